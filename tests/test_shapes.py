"""The GRE shape generator reproduces the reference's lattices (CPU).

The golden geometry records were produced by the reference's own shape model
(tests/golden/make_golden.py); the restatement must give the same lattice,
spacing and occupancy mask bit for bit from the same seed."""
import os

import numpy as np
import pytest

from bdda_b200.inputs import load_geometry
from bdda_b200.shapes import gre_particle, inside_mask

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("name,args", [
    ("geometry_cfg1", dict(x=5, ab=1.0, bc=1.0, beta=0.0, seed=0, wl_0=1.0, m_m=1.0)),
    ("geometry_cfg2", dict(x=20, ab=0.7, bc=0.8, beta=0.1, seed=1, wl_0=1.0, m_m=1.33)),
])
def test_gre_matches_reference_lattice(name, args):
    rec = load_geometry(os.path.join(GOLDEN, name + ".npz"))
    g = gre_particle(**args)
    assert np.array_equal(g["lattice_n"], rec["lattice_n"])
    assert g["lattice_lf"] == rec["lattice_lf"]
    for ax in ("x_axis", "y_axis", "z_axis"):
        assert np.array_equal(g[ax], rec[ax])
    assert np.array_equal(g["is_in"], rec["is_in"])


def test_inside_mask_excludes_the_surface_shell():
    near = np.zeros((7, 7, 7), bool)
    near[1, 1:6, 1:6] = near[5, 1:6, 1:6] = True
    near[1:6, 1, 1:6] = near[1:6, 5, 1:6] = True
    near[1:6, 1:6, 1] = near[1:6, 1:6, 5] = True
    ins = inside_mask(near)
    assert ins[2:5, 2:5, 2:5].all() and ins.sum() == 27


def test_coarse_field_is_seeded_and_sized():
    a = gre_particle(8, 0.8, 0.9, 0.1, seed=4, coarse=(13, 50))
    b = gre_particle(8, 0.8, 0.9, 0.1, seed=4, coarse=(13, 50))
    assert np.array_equal(a["is_in"], b["is_in"]) and a["address"].size > 1000
