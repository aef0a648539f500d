"""GPU block solvers against the reference's golden runs and the oracle.

Parity levels (see the oracle tests for the reference's own sensitivity):
* short solves (<= 13 iterations) follow the reference's trajectory: same
  iteration count, same printed history, X within 1e-9;
* at tol 1e-5 the iterate is rounding-dependent in the reference itself, so
  iterations agree within 1 and outputs within 1e-4;
* converged to 1e-11 the outputs agree within 1e-8.
"""
import os

import numpy as np
import pytest
import torch

from conftest import load_golden
from oracle import dda_oracle as O
from bdda_b200.inputs import load_geometry

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def rel(a, b):
    a = a.cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a)
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


@pytest.fixture(scope="module")
def mods():
    from mvp_fft import mvp_fft
    from bl_krylov import bl_krylov
    return mvp_fft, bl_krylov


def solver_fn(bk, name):
    return bk.bl_bicgstab_jacobi_mvp_fft if name == "bicgstab" else bk.bl_cocg_rq_jacobi_mvp_fft


@pytest.mark.parametrize("solver", ["bicgstab", "cocg"])
def test_small_solve_follows_reference_trajectory(mods, solver):
    mf, bk = mods
    g = load_golden("solver_small")
    til = mf.fft_init(g["n"], 3, float(g["lf"]), float(g["k"]))
    hist = []
    X, it, err = solver_fn(bk, solver)(g["n"], 3, g["address"], til, g["diag_A"], g["B"], 1e-5, 200,
                                       history=hist)
    assert it == int(g[solver + "_iter_fin"])
    assert np.array_equal(np.round(hist, 4), g[solver + "_history"])
    assert abs(err - float(g[solver + "_err_fin"])) < 1e-8 * abs(float(g[solver + "_err_fin"])) + 1e-13
    assert rel(X, g[solver + "_X"]) < 1e-9


def _case(rec):
    n = rec["lattice_n"]
    lf = rec["lattice_lf"]
    address = rec["address"]
    pos = rec["grid"][address]
    geom = O.incident_geometry(float(rec["wl_0"]), float(rec["m_m"]), rec["euler"])
    eper_r, _, diag = O.polarizability(rec["m_p_xyz"], float(rec["m_m"]), lf, geom["k"], address.size)
    B = O.rhs(geom["k"], geom["u_inc"], geom["e0_inc"], pos)
    return n, lf, address, pos, geom, eper_r, diag, B


def test_test_dda_notebook_known_answers(mods):
    mf, bk = mods
    rec = load_geometry(os.path.join(GOLDEN, "kat_test_dda.npz"))
    n, lf, address, pos, geom, eper_r, diag, B = _case(rec)
    til = mf.fft_init(n, 3, lf, geom["k"])
    hist = []
    X, it, err = bk.bl_bicgstab_jacobi_mvp_fft(n, 3, address, til, diag, B, 1e-2, 25, history=hist)
    assert it == 1 and [round(h, 4) for h in hist] == [0.0156, 0.0002]   # test_dda.ipynb:189-191
    obs = O.observables(X, geom, pos, eper_r, lf)
    for key in ("C_abs", "C_ext", "S_fw_theta", "S_fw_phi", "S_bk"):
        assert rel(obs[key], rec[key]) < 1e-10, key


CFG1 = [("cocg", 1e-5, ""), ("bicgstab", 1e-5, "bicgstab_tol5_"),
        ("cocg", 1e-11, "cocg_tight_"), ("bicgstab", 1e-11, "bicgstab_tight_")]


@pytest.mark.parametrize("solver,tol,tag", CFG1)
def test_config1_sphere_matches_reference(mods, solver, tol, tag):
    mf, bk = mods
    rec = load_geometry(os.path.join(GOLDEN, "geometry_cfg1.npz"))
    n, lf, address, pos, geom, eper_r, diag, B = _case(rec)
    til = mf.fft_init(n, 3, lf, geom["k"])
    X, it, err = solver_fn(bk, solver)(n, 3, address, til, diag, B, tol, 300)
    assert err < tol
    # +-1 iteration at tol 1e-5; at 1e-11 the recursive residual sits at the
    # FP64 floor, where a different (CholeskyQR vs Householder) rounding moves
    # COCG-rq's stopping iteration by a few
    assert abs(it - int(rec[tag + "iter_fin"])) <= (1 if tol > 1e-6 else 3)
    obs = O.observables(X, geom, pos, eper_r, lf)
    bound = 1e-4 if tol > 1e-6 else 1e-8
    for key in ("C_abs", "C_ext", "S_fw_theta", "S_fw_phi", "S_bk"):
        assert rel(obs[key], rec[tag + key]) < bound, key
    # the recursive residual tracks the true one
    true = O.true_residual(n, 3, address, O.fft_init(n, 3, lf, geom["k"]), diag, B, X)
    assert true < 3 * tol


def test_fp32_solve_reaches_fp32_accuracy(mods):
    mf, bk = mods
    rec = load_geometry(os.path.join(GOLDEN, "geometry_cfg1.npz"))
    n, lf, address, pos, geom, eper_r, diag, B = _case(rec)
    til = mf.fft_init(n, 3, lf, geom["k"])
    X, it, err = bk.bl_bicgstab_jacobi_mvp_fft(n, 3, address, til, diag, B, 1e-4, 300, precision="c64")
    assert err < 1e-4
    true = O.true_residual(n, 3, address, O.fft_init(n, 3, lf, geom["k"]), diag, B, X)
    assert true < 5e-4


def test_warm_start_from_solution_converges_immediately(mods):
    mf, bk = mods
    g = load_golden("solver_small")
    til = mf.fft_init(g["n"], 3, float(g["lf"]), float(g["k"]))
    X, it, err = bk.bl_bicgstab_jacobi_mvp_fft(g["n"], 3, g["address"], til, g["diag_A"], g["B"],
                                                1e-6, 200, X0=g["bicgstab_X"])
    assert it == 0 and err < 1e-5
    Xr, itr, errr = O.bicgstab(g["n"], 3, g["address"], O.fft_init(g["n"], 3, float(g["lf"]), float(g["k"])),
                               g["diag_A"], g["B"], 1e-6, 200, X0=g["bicgstab_X"])
    assert itr == 0 and rel(X, Xr) < 1e-9


@pytest.mark.parametrize("solver", ["bicgstab", "cocg"])
def test_errors_and_edge_cases(mods, solver):
    mf, bk = mods
    g = load_golden("solver_small")
    fn = solver_fn(bk, solver)
    til = mf.fft_init(g["n"], 3, float(g["lf"]), float(g["k"]))
    args = (g["n"], 3, g["address"], til, g["diag_A"])
    with pytest.raises(ValueError):
        fn(g["n"], 2, g["address"], til, g["diag_A"], g["B"], 1e-5, 10)
    # itermax = 0: X = 0, iter_fin = 0, err_fin = inf (bl_krylov.py:95-96)
    X, it, err = fn(*args, g["B"], 1e-5, 0)
    assert it == 0 and err == float("inf") and not np.any(X)
    # itermax reached: not an error
    X, it, err = fn(*args, g["B"], 1e-14, 2)
    assert it == 1 and err > 1e-14
    # a NaN right-hand side stops with a NaN residual, not an exception
    Bn = g["B"].copy()
    Bn[5, 1] = np.nan
    X, it, err = fn(*args, Bn, 1e-5, 50)
    assert not np.isfinite(err)


def test_duplicate_columns_raise_linalgerror(mods):
    """Linearly dependent right-hand sides make R0^H V exactly singular (numpy raises too)."""
    mf, bk = mods
    g = load_golden("solver_small")
    B = g["B"].copy()
    B[:, 2] = B[:, 0]
    til = mf.fft_init(g["n"], 3, float(g["lf"]), float(g["k"]))
    with pytest.raises(np.linalg.LinAlgError):
        bk.bl_bicgstab_jacobi_mvp_fft(g["n"], 3, g["address"], til, g["diag_A"], B, 1e-5, 50)
    with pytest.raises(np.linalg.LinAlgError):
        O.bicgstab(g["n"], 3, g["address"], O.fft_init(g["n"], 3, float(g["lf"]), float(g["k"])),
                   g["diag_A"], B, 1e-5, 50)


@pytest.mark.parametrize("L", [16, 32, 64])
@pytest.mark.parametrize("solver", ["bicgstab", "cocg"])
def test_specialised_block_kernels_match_generic(mods, L, solver):
    """The L-specialised Gram / update kernels and the generic ones give the same solve."""
    from bdda_b200 import _lib
    mf, bk = mods
    rec = load_geometry(os.path.join(GOLDEN, "kat_test_dda.npz"))
    n, lf, address, pos, geom, eper_r, diag, B = _case(rec)
    rng = np.random.default_rng(L)
    Bl = rng.standard_normal((B.shape[0], L)) + 1j * rng.standard_normal((B.shape[0], L))
    til = mf.fft_init(n, 3, lf, geom["k"])
    fn = solver_fn(bk, solver)
    X1, it1, err1 = fn(n, 3, address, til, diag, Bl, 1e-6, 60)
    _lib.load().bdda_tune_fixed(0)
    try:
        X2, it2, err2 = fn(n, 3, address, til, diag, Bl, 1e-6, 60)
    finally:
        _lib.load().bdda_tune_fixed(1)
    assert err1 < 1e-6 and err2 < 1e-6 and abs(it1 - it2) <= 1
    assert rel(X1, X2) < 1e-5


@pytest.mark.parametrize("precision", ["mixed", "mixed-fp32"])
@pytest.mark.parametrize("solver", ["bicgstab", "cocg"])
def test_mixed_precision_refinement_meets_fp64_accuracy(mods, solver, precision):
    """Both mixed forms (complex64 products in complex128 Krylov; complex64
    block solves inside FP64 refinement) reach the true residual 1e-5 and the
    observables agree with the FP64 solve within 1e-4 (the metric's bound)."""
    mf, bk = mods
    rec = load_geometry(os.path.join(GOLDEN, "geometry_cfg1.npz"))
    n, lf, address, pos, geom, eper_r, diag, B = _case(rec)
    til = mf.fft_init(n, 3, lf, geom["k"])
    fn = solver_fn(bk, solver)
    hist = []
    Xm, itm, errm = fn(n, 3, address, til, diag, B, 1e-5, 400, precision=precision, history=hist)
    assert errm < 1e-5 and len(hist) == itm + 1
    true = O.true_residual(n, 3, address, O.fft_init(n, 3, lf, geom["k"]), diag, B, Xm)
    assert abs(true - errm) < 1e-3 * errm + 1e-9      # err_fin is the true residual
    X64, it64, err64 = fn(n, 3, address, til, diag, B, 1e-5, 400)
    om = O.observables(Xm, geom, pos, eper_r, lf)
    o64 = O.observables(X64, geom, pos, eper_r, lf)
    for key in ("C_ext", "S_fw_theta", "S_fw_phi", "S_bk"):
        assert rel(om[key], o64[key]) < 1e-4, key


def test_reliable_update_variant_small_block(mods):
    """One FP32 BiCGSTAB recursion with FP64 residual replacement (L = 8)."""
    mf, bk = mods
    rec = load_geometry(os.path.join(GOLDEN, "geometry_cfg1.npz"))
    n, lf, address, pos, geom, eper_r, diag, B = _case(rec)
    til = mf.fft_init(n, 3, lf, geom["k"])
    X, it, err = bk.bl_bicgstab_jacobi_mvp_fft(n, 3, address, til, diag, B, 1e-5, 300, precision="mixed-reliable")
    assert err < 1e-5
    true = O.true_residual(n, 3, address, O.fft_init(n, 3, lf, geom["k"]), diag, B, X)
    assert abs(true - err) < 1e-3 * err + 1e-9
    assert it + 1 <= 2 * (int(rec["bicgstab_tol5_iter_fin"]) + 1)


def test_mixed_fallback_after_divergence_warm_starts_from_the_best_iterate(mods):
    """With a divergence factor of 1.2 the mixed recursion counts as diverged at
    its first 1.2-fold residual rise above its reference (x=20 particle, 16
    orientations: block BiCGSTAB's residual is not monotone there).  The complex128 fallback then
    starts from the X of the smallest residual so far, watched by the same
    test (and restarted from zero once if that trips too): the solve converges
    to tol on the true residual, to the complex128 solution, its complex128
    phase starts below a zero start's first residual, and it needs no more
    iterations than the recursion plus two complex128 solves from zero."""
    from bdda_b200 import _lib
    mf, bk = mods
    rec = load_geometry(os.path.join(GOLDEN, "geometry_cfg2.npz"))
    rec = dict(rec, euler=rec["euler"][:16])
    n, lf, address, pos, geom, eper_r, diag, B = _case(rec)
    til = mf.fft_init(n, 3, lf, geom["k"])
    h64 = []
    X64, it64, err64 = bk.bl_bicgstab_jacobi_mvp_fft(n, 3, address, til, diag, B, 1e-5, 400, history=h64)
    lib = _lib.load()
    import ctypes as C
    d, sw, f = C.c_double(), C.c_double(), C.c_double()
    assert lib.bdda_tune_mixed_get(C.byref(d), C.byref(sw), C.byref(f)) == 0
    hm = []
    try:
        assert lib.bdda_tune_mixed(d.value, sw.value, 1.2) == 0
        Xm, itm, errm = bk.bl_bicgstab_jacobi_mvp_fft(n, 3, address, til, diag, B, 1e-5, 400, precision="mixed",
                                                      history=hm)
    finally:
        lib.bdda_tune_mixed(d.value, sw.value, f.value)
    # the fallback ran at the first 1.2-fold rise: above the first iteration's
    # residual in the first 8 iterations before the first residual replacement
    # (a 10-fold drop below the largest residual), above the smallest after
    replaced, rmax, k_div = False, 0.0, None
    for k in range(len(hm)):
        if k and hm[k] < 0.1 * rmax:
            replaced, rmax = True, hm[k]
        rmax = max(rmax, hm[k])
        if k and hm[k] > 1.2 * (min(hm[:k + 1]) if (replaced or k >= 8) else hm[0]):
            k_div = k
            break
    assert k_div is not None
    assert errm < 1e-5 and err64 < 1e-5
    true = O.true_residual(n, 3, address, O.fft_init(n, 3, lf, geom["k"]), diag, B, Xm)
    assert true < 1e-5
    assert rel(Xm, X64) < 1e-3
    assert itm + 1 <= (k_div + 1) + 2 * (it64 + 1)
    # the complex128 phase starts below where a zero start begins
    assert hm[k_div + 1] < h64[0]


def test_mixed_form_recovers_where_a_warm_complex128_restart_stagnates():
    """A small strongly scattering GRE (x = 4.4, m = 1.53 + 0.005i, 24 x 28 x 35
    lattice, 32 orientations, built as the batched sweep builds it): the
    complex64 recursion stagnates near 1e-3 and counts as diverged; a
    complex128 restart from its best X stagnated for 480 iterations, so that
    restart is watched and replaced by a zero start.  The mixed solve converges
    and gives the complex128 observables."""
    from bdda_b200.inputs import so3_euler
    from bdda_b200.shapes import gre_particle
    from bl_dda import scatterer as sc
    wl, mp = 0.85, 1.53 + 0.005j
    g = gre_particle(4.403823395619191, 0.7398419617561375, 0.7475936957677011, 0.029412861486646926, 3002,
                     wl_0=1.0, m_m=1.0, workers=1)
    sc.DiscreteDipoles.verbose = False
    out = {}
    for prec, tol in ((None, 1e-5), ("mixed", 1e-5), (None, 1e-10)):
        t = sc.Target("gre2", g["lattice_n"], g["lattice_lf"] * wl, g["grid"] * wl, g["is_in"], [mp] * 3)
        d = sc.DiscreteDipoles(t, sc.IncidentField(wl, 1.0, so3_euler(32, 308)))
        d.tol, d.itermax, d.precision = tol, 800, prec
        d.set_interaction_matrix()
        d.solve_matrix_equation()
        assert d.converge and d.err_fin < tol, (prec, d.iter_fin, d.err_fin)
        out[(prec, tol)] = (d.iter_fin, d.observables())
    assert out[("mixed", 1e-5)][0] <= 120
    o64, om, oc = out[(None, 1e-5)][1], out[("mixed", 1e-5)][1], out[(None, 1e-10)][1]

    def err(o, r, cols):
        a = o[:, cols[0]] + (1j * o[:, cols[1]] if len(cols) > 1 else 0)
        b = r[:, cols[0]] + (1j * r[:, cols[1]] if len(cols) > 1 else 0)
        return np.max(np.abs(a - b)) / np.max(np.abs(b))
    # C_ext and S_fw within 1e-4 of the complex128 path; S_bk (the most
    # rounding-sensitive amplitude) as close to the converged solution as the
    # complex128 path at the same tolerance is (within 3x, or 1e-4)
    for cols in ((1,), (2, 3), (4, 5)):
        assert err(om, o64, cols) < 1e-4, cols
    assert err(om, oc, (10, 11)) < max(3 * err(o64, oc, (10, 11)), 1e-4)


def test_mixed_form_converges_where_fp32_krylov_diverges(mods):
    """A strongly scattering GRE (x = 9.2, m = 1.53 + 0.005i, 34 x 65 x 69
    lattice): complex64 Krylov vectors diverge here, the mixed form (complex64
    products only) converges and gives complex128's observables.  It needs
    more iterations here: under 1e-7 perturbations of B, complex128 took
    86-90 and the mixed form 106-120 (replacement after each 10-fold drop)."""
    from bdda_b200.inputs import so3_euler
    from bdda_b200.shapes import gre_particle
    mf, bk = mods
    g = gre_particle(9.197523282837686, 0.6459893079939255, 0.7681224627849057, 0.04502319853187231, seed=3005,
                     wl_0=0.55)
    rec = dict(g, euler=so3_euler(8, 16), m_p_xyz=np.array([1.53 + 0.005j] * 3))
    n, lf, address, pos, geom, eper_r, diag, B = _case(rec)
    til = mf.fft_init(n, 3, lf, geom["k"])
    X64, it64, err64 = bk.bl_bicgstab_jacobi_mvp_fft(n, 3, address, til, diag, B, 1e-5, 400)
    Xm, itm, errm = bk.bl_bicgstab_jacobi_mvp_fft(n, 3, address, til, diag, B, 1e-5, 400, precision="mixed")
    Xc, _, errc = bk.bl_bicgstab_jacobi_mvp_fft(n, 3, address, til, diag, B, 1e-10, 600)
    assert err64 < 1e-5 and errm < 1e-5 and errc < 1e-10
    assert itm <= 1.4 * it64 + 5
    o64 = O.observables(X64, geom, pos, eper_r, lf)
    om = O.observables(Xm, geom, pos, eper_r, lf)
    oc = O.observables(Xc, geom, pos, eper_r, lf)
    # against the converged solution the mixed form is as accurate as complex128 at the same tolerance
    for key in ("C_ext", "S_fw_theta", "S_fw_phi", "S_bk"):
        assert rel(om[key], oc[key]) < max(3 * rel(o64[key], oc[key]), 1e-5), key


@pytest.mark.parametrize("solver", ["bicgstab", "cocg"])
@pytest.mark.parametrize("prec", [None, "c64"])
def test_graph_driven_loop_matches_the_host_loop(mods, solver, prec):
    """Small solves run their iterations as a CUDA graph while node (the loop
    condition set on the device at the residual test); the same solve with the
    host-driven loop gives the same iterates, residual history and count."""
    from bdda_b200 import _lib
    mf, bk = mods
    g = load_golden("solver_small")
    til = mf.fft_init(g["n"], 3, float(g["lf"]), float(g["k"]))
    lib = _lib.load()
    res = {}
    try:
        for on in (1, 0):
            assert lib.bdda_tune_solver_graphs(on) == 0
            h = []
            n0 = lib.bdda_launch_count()
            X, it, err = solver_fn(bk, solver)(g["n"], 3, g["address"], til, g["diag_A"], g["B"], 1e-9, 300,
                                               precision=prec, history=h)
            res[on] = (X, it, err, h, lib.bdda_launch_count() - n0)
    finally:
        lib.bdda_tune_solver_graphs(1)
    assert res[1][1] == res[0][1] and res[1][1] > 5
    assert res[1][2] == res[0][2]
    assert res[1][3] == res[0][3]
    assert np.array_equal(res[1][0], res[0][0])
    # the launch counter counts the kernels the graph ran: the host loop's,
    # plus the loop-condition kernel once per iteration (the host loop reads
    # the residual instead; COCG's in-place copy of the new Q is no kernel)
    assert abs((res[1][4] - res[0][4]) - (res[1][1] + 1)) <= 2, (res[1][4], res[0][4], res[1][1])


def test_graph_driven_loop_stops_at_itermax(mods):
    """A solve that cannot converge stops after exactly itermax iterations in
    the graph-driven loop, with the host loop's count and residual."""
    from bdda_b200 import _lib
    mf, bk = mods
    g = load_golden("solver_small")
    til = mf.fft_init(g["n"], 3, float(g["lf"]), float(g["k"]))
    lib = _lib.load()
    out = {}
    try:
        for on in (1, 0):
            lib.bdda_tune_solver_graphs(on)
            h = []
            X, it, err = bk.bl_bicgstab_jacobi_mvp_fft(g["n"], 3, g["address"], til, g["diag_A"], g["B"], 1e-30, 7,
                                                       history=h)
            out[on] = (it, err, len(h))
    finally:
        lib.bdda_tune_solver_graphs(1)
    assert out[1] == out[0] == (6, out[0][1], 7)
