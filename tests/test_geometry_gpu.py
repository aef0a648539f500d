"""GRE lattice occupancy on the GPU (bdda_gre_occupancy) against the reference.

The golden geometry records were produced by the reference's shape model
(tests/golden/make_golden.py); the GPU near-surface and inside kernels must
reproduce their masks bit for bit.  The host binning is checked on the CPU."""
import os

import numpy as np
import pytest

from bdda_b200.inputs import load_geometry
from bdda_b200.shapes import gre_particle, gre_geometry, gre_surface, host_near_surface, inside_mask, lattice_axes
from conftest import load_golden

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_surface_bins_hold_every_point_once():
    from bdda_b200.geometry import _bins
    rng = np.random.default_rng(5)
    surf = gre_surface(0.3, 0.8, 0.9, 0.1, rng, coarse=(13, 50))
    thr = 0.02
    pts, start, nb, origin, h = _bins(surf, thr)
    assert h >= thr and start[0] == 0 and start[-1] == len(surf) and np.all(np.diff(start) >= 0)
    assert sorted(map(tuple, pts)) == sorted(map(tuple, surf))
    b = np.floor((pts - origin) / h).astype(np.int64)
    flat = (b[:, 0] * nb[1] + b[:, 1]) * nb[2] + b[:, 2]
    assert np.all((flat >= 0) & (flat < np.prod(nb)))
    assert np.all(start[flat] <= np.arange(len(pts))) and np.all(np.arange(len(pts)) < start[flat + 1])


@pytest.mark.gpu
@pytest.mark.parametrize("name,args", [
    ("geometry_cfg1", dict(x=5, ab=1.0, bc=1.0, beta=0.0, seed=0, wl_0=1.0, m_m=1.0)),
    ("geometry_cfg2", dict(x=20, ab=0.7, bc=0.8, beta=0.1, seed=1, wl_0=1.0, m_m=1.33)),
])
def test_gpu_occupancy_matches_reference_lattice(name, args):
    from bdda_b200.geometry import inside_from_gpu
    rec = load_geometry(os.path.join(GOLDEN, name + ".npz"))
    g = gre_particle(**args, mask_fn=inside_from_gpu)
    assert np.array_equal(g["lattice_n"], rec["lattice_n"])
    assert np.array_equal(g["is_in"], rec["is_in"])


@pytest.mark.gpu
def test_gpu_occupancy_of_sweep_shapes_matches_reference_r_ve():
    """The reference-default spacing pipeline (run_dda.py:21-35) with the GPU mask gives the
    reference's r_ve for the shapes of the small sweep."""
    from bdda_b200.geometry import inside_from_gpu
    g = load_golden("sweep_small")
    for i, rv in enumerate(g["r_v_base_list"]):
        geo = gre_geometry(float(rv), float(g["bc_ratio_list"][0]), float(g["ab_ratio_list"][0]),
                           float(g["gre_beta_list"][0]), int(g["rng_seed"]), mask_fn=inside_from_gpu)
        assert geo["r_ve"] == g["r_ve"][i, 0, 0, 0]


@pytest.mark.gpu
def test_gpu_near_and_inside_match_host_on_random_shapes():
    from bdda_b200.geometry import occupancy
    rng = np.random.default_rng(17)
    for trial in range(6):
        ab, bc, beta = rng.uniform(0.5, 1.0), rng.uniform(0.5, 1.0), rng.uniform(0.0, 0.3)
        r_v = rng.uniform(0.1, 0.5)
        surf = gre_surface(r_v, ab, bc, beta, np.random.default_rng(trial), coarse=(13, 50))
        lf = r_v / rng.uniform(6, 20)
        thr = lf * rng.uniform(0.6, 1.5)
        axes = lattice_axes(surf, lf)
        near, inside = occupancy(axes, surf, thr)
        near_h = host_near_surface(axes, surf, thr)
        assert np.array_equal(near, near_h), trial
        assert np.array_equal(inside, inside_mask(near_h)), trial
