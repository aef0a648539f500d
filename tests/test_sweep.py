"""Sweep driver (the reference's run_dda.py): retries, NaN fill, resumable shards.

CPU tests drive the sweep logic with a stand-in solver and geometry; the GPU
test runs a small sweep end to end and compares it with the same sweep run
by the reference's own classes (tests/golden/sweep_small.npz, made by
tests/golden/make_golden.py)."""
import os

import numpy as np
import pytest

from bdda_b200 import sweep as S
from bdda_b200.mie import mie_q_and_s
from conftest import load_golden


def _spec(**kw):
    g = load_golden("sweep_small")
    args = dict(wl_m_m_pairs=g["wl_m_m_pairs"], m_p_xyz_list=g["m_p_xyz_list"], r_v_base_list=g["r_v_base_list"],
                bc_ratio_list=g["bc_ratio_list"], ab_ratio_list=g["ab_ratio_list"],
                gre_beta_list=g["gre_beta_list"], num_orientations=int(g["num_orientations"]),
                rng_seed=int(g["rng_seed"]), max_try=int(g["max_try"]))
    args.update(kw)
    return S.SweepSpec(**args)


def test_euler_tries_follow_the_reference_draws():
    g = load_golden("sweep_small")
    tries = S.euler_tries(int(g["num_orientations"]), int(g["rng_seed"]) + 1, int(g["max_try"]))
    # every golden condition converged on its first try: its angles are try 1's
    assert (g["tries"] == 1).all()
    for idx in np.ndindex(g["tries"].shape):
        assert np.array_equal(g["Euler_angles"][idx], tries[0])
    assert len(tries) == 4 and not np.array_equal(tries[0], tries[1])
    assert (tries[1][:, 1] >= 0).all() and (tries[1][:, 1] < np.pi).all()   # beta ~ U[0, pi), as run_dda.py:51


def test_mie_matches_reference_routine():
    m = load_golden("mie_small")
    for row, q, s in zip(m["cases"], m["Q_sca_abs_ext"], m["S_fw_bk"]):
        wl, mm, r, a, b = row
        qs, qa, qe, sf, sb = mie_q_and_s(wl, mm, r, complex(a, b))
        assert np.allclose([qs, qa, qe], q, rtol=1e-12, atol=1e-13 * abs(q[2])), (row, [qs, qa, qe], q)
        # the reference rounds the amplitudes to complex64
        assert abs(sf - s[0]) <= 1e-7 * abs(s[0]) and abs(sb - s[1]) <= 1e-7 * abs(s[1]), row


class _FakeSolver:
    """Observables derived from the angles; (pair 0, m_p 1) converges on try 3, (pair 1, m_p 1) never."""

    def __init__(self):
        self.calls = []

    def __call__(self, items):
        out = []
        for target, wl_0, m_m, euler in items:
            key = (wl_0, complex(target.m_p_xyz[0]))
            self.calls.append((key, float(euler[0, 0])))
            n_try = sum(1 for k, _ in self.calls if k == key)
            L = euler.shape[0]
            obs = np.zeros((L, 12))
            obs[:, 1] = euler[:, 0] * wl_0
            obs[:, 2] = euler[:, 1]
            obs[:, 10] = euler[:, 2]
            fails = {(0.633, 1.55 + 0.01j): 2, (0.8337, 1.55 + 0.01j): 99}.get(key, 0)
            out.append((n_try > fails, obs, 3))
        return out


def _fake_geometry(r_v_base, bc, ab, beta, seed, lattice_lf=None, mask_fn=None):
    n = np.array([4, 3, 2])
    grid = np.stack(np.meshgrid(*[np.arange(k) * 0.01 for k in n], indexing="ij"), -1).reshape(-1, 3)
    is_in = np.ones(24, bool)
    return dict(name="fake%.2f" % r_v_base, lattice_n=n, lattice_lf=0.01, is_in=is_in, address=np.arange(24),
                grid=grid, r_ve=r_v_base)


def test_sweep_retries_fills_nan_and_resumes(tmp_path, monkeypatch):
    monkeypatch.setattr(S, "gre_geometry", _fake_geometry)
    spec = _spec()
    out = str(tmp_path / "sweep")
    fake = _FakeSolver()
    sw = S.Sweep(spec, out, solve=fake, verbose=False)
    assert len(sw.pending()) == 8
    # interrupted after 3 conditions: only whole shards exist
    assert sw.run(max_conditions=3) == 3
    assert len(sw.pending()) == 5
    # a shard half-written by a crash is not taken as done
    open(os.path.join(out, S.shard_name((1, 1, 1, 0, 0, 0)) + ".part.npz"), "wb").write(b"partial")
    fake2 = _FakeSolver()
    sw2 = S.Sweep(spec, out, solve=fake2, verbose=False)
    assert len(sw2.pending()) == 5
    assert sw2.run() == 5
    assert sw2.pending() == []
    # nothing done before was solved again: shape 0's last condition (4 failed
    # tries) and shape 1's four (1 + 3 + 1 + 4 tries)
    assert len(fake2.calls) == 4 + 9
    r = S.load_results(out)
    assert r["done"].all()
    tries = S.euler_tries(spec.num_orientations, spec.rng_seed + 1, spec.max_try)
    for idx in np.ndindex(r["done"].shape):
        p, m = idx[:2]
        wl = spec.wl_m_m_pairs[p, 0]
        if (p, m) == (1, 1):   # never converged: NaN with the last try's angles (run_dda.py:68-70)
            assert not r["converged"][idx]
            assert np.isnan(r["C_ext"][idx]).all() and np.isnan(r["S_bk_OCBS"][idx]).all()
            assert np.array_equal(r["Euler_angles"][idx], tries[-1])
        else:
            t = 2 if (p, m) == (0, 1) else 0
            assert r["converged"][idx]
            assert np.array_equal(r["Euler_angles"][idx], tries[t])
            assert np.allclose(r["C_ext"][idx], tries[t][:, 0] * wl)
            assert np.allclose(r["S_bk_OCBS"][idx].real, tries[t][:, 2])
        assert np.isfinite(r["C_ext_mie"][idx])
    assert np.allclose(r["r_ve"][:, 0, 0, 0], spec.r_v_base_list)
    # a third run finds nothing to do and builds no geometry
    monkeypatch.setattr(S, "gre_geometry", lambda *a, **k: pytest.fail("geometry rebuilt for a finished shape"))
    assert S.Sweep(spec, out, solve=_FakeSolver(), verbose=False).run() == 0


def test_sweep_refuses_a_folder_of_another_sweep(tmp_path, monkeypatch):
    monkeypatch.setattr(S, "gre_geometry", _fake_geometry)
    out = str(tmp_path / "sweep")
    S.Sweep(_spec(), out, solve=_FakeSolver(), verbose=False)
    with pytest.raises(ValueError):
        S.Sweep(_spec(num_orientations=16), out, solve=_FakeSolver(), verbose=False)


def _golden_geometry(g):
    """gre_geometry stand-in serving the reference's own lattices of the small sweep
    (the GRE surface depends on the host's LAPACK eigh, so it is not redrawn here)."""
    from bdda_b200.inputs import lattice_points

    def geometry(r_v_base, bc, ab, beta, seed, lattice_lf=None, mask_fn=None):
        i = int(np.flatnonzero(np.isclose(g["r_v_base_list"], r_v_base))[0])
        tag = "shape_%d_0_0_0_" % i
        n = g[tag + "lattice_n"]
        is_in = np.unpackbits(g[tag + "mask_bits"])[:int(np.prod(n))].astype(bool)
        lf = float(g[tag + "lattice_lf"])
        return dict(name=str(g[tag + "name"]), lattice_n=n, lattice_lf=lf, is_in=is_in,
                    address=np.flatnonzero(is_in),
                    grid=lattice_points(g[tag + "x_axis"], g[tag + "y_axis"], g[tag + "z_axis"]),
                    r_ve=float(np.cbrt(3.0 * lf ** 3 * int(is_in.sum()) / (4 * np.pi))))
    return geometry


@pytest.mark.gpu
def test_small_sweep_matches_reference_run(tmp_path, monkeypatch):
    """The sweep on the GPU (batched solves, Green's spectra shared across m_p)
    on the reference's own lattices, against the same sweep run with the
    reference's classes: same angles and r_ve, observables of these short
    solves (tol 1e-2, a few iterations) to 1e-8, Mie values to the
    reference's complex64 rounding."""
    g = load_golden("sweep_small")
    monkeypatch.setattr(S, "gre_geometry", _golden_geometry(g))
    out = str(tmp_path / "sweep")
    sw = S.Sweep(_spec(), out, verbose=False)
    assert sw.run() == 8
    r = S.load_results(out)
    assert r["done"].all() and r["converged"].all()
    assert np.array_equal(r["r_ve"], g["r_ve"])
    assert np.array_equal(r["Euler_angles"], g["Euler_angles"])
    for k in ("C_ext", "S_fw_PCAS_theta", "S_fw_PCAS_phi", "S_bk_OCBS"):
        err = np.max(np.abs(r[k] - g[k])) / np.max(np.abs(g[k]))
        assert err < 1e-8, (k, err)
    assert np.max(np.abs(r["C_abs"] - g["C_abs"])) <= 1e-8 * np.max(np.abs(g["C_abs"]))
    for k in ("S_fw_PCAS_mie", "S_bk_OCBS_mie"):
        assert np.max(np.abs(r[k] - g[k]) / np.abs(g[k])) < 1e-6
    for k in ("C_abs_mie", "C_ext_mie"):
        assert np.allclose(r[k], g[k], rtol=1e-10, atol=1e-12 * np.max(np.abs(g["C_ext_mie"])))
