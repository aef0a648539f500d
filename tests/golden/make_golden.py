"""Generate the golden fixtures in this folder from the live reference.

Run in a container where the reference block-DDA_Py v0.3.0 is checked out,
naming its folder with ``--reference`` or the ``BDDA_REFERENCE`` variable:

    python tests/golden/make_golden.py --reference PATH [fixture ...]

With no fixture names the small fixtures are written; ``solve_cfg2_chunk``
(minutes of CPU and ~14 GB of RAM), ``sweep_small`` and ``mie_small`` are
written when named.

The reference is imported as-is; ``matplotlib`` (absent in this image, used
only for plotting in shape_model/gaussian_ellipsoid.py:4-8,41) is replaced by
an inert stub.  Nothing here runs at test time: the tests read only the
``.npz`` files written below.

Fixtures
--------
green_small.npz      build_interaction_tensor + fft_init, n=(3,4,5)
fft_mvp_small.npz    fft_mvp on (5,6,7), L=3 and a 1-D column
block_mvp_small.npz  _block_mvp on a ragged occupancy of a (6,5,7) cuboid, L=4
solver_small.npz     both block solvers to 1e-5 on a small blob (L=3),
                     full X and the per-iteration residual history
kat_test_dda.npz     inputs and reference outputs of test_dda.ipynb
                     (sphere r_v=0.2 um, 17^3 lattice, L=10, tol 1e-2)
geometry_cfg1.npz    sphere x=5, wl=1, m_m=1, spacing 1/16 -> 28^3 lattice,
                     plus the reference's COCG-rq solution to 1e-5 at L=8
geometry_cfg2.npz    GRE x=20 (m_m=1.33, wl=1), ab 0.7, bc 0.8, beta 0.1,
                     surface seed 1, spacing lambda_m/16 -> 93x112x174
solve_cfg2_chunk.npz the reference's block-BiCGSTAB solve of that particle,
                     orientations 0-7 of the seed-2 set, to 1e-5: iteration
                     count, residual history, observables, sampled rows of X
sweep_small.npz      a 2 x 2 x 2-shape sweep run as run_dda.py runs it (shape
                     seed 12345, angle seed 12346, retries, Mie values), in
                     the reference's 7-D layout
mie_small.npz        the reference's Mie routine on six spheres
"""
from __future__ import annotations

import argparse
import contextlib
import io
import os
import sys
import time
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.environ.get("BDDA_REFERENCE")


def _stub_matplotlib() -> None:
    """Register inert stand-ins for the plotting imports of the shape model."""
    class _Any:  # accepts any construction / attribute access
        def __init__(self, *a, **k):
            pass

    names = ["matplotlib", "matplotlib.pyplot", "matplotlib.patches",
             "mpl_toolkits", "mpl_toolkits.mplot3d", "mpl_toolkits.mplot3d.proj3d"]
    for name in names:
        sys.modules.setdefault(name, types.ModuleType(name))
    sys.modules["matplotlib.patches"].FancyArrowPatch = _Any
    sys.modules["mpl_toolkits.mplot3d"].Axes3D = _Any
    sys.modules["mpl_toolkits.mplot3d.proj3d"].proj_transform = lambda *a, **k: None


def _import_reference():
    if not REF or not os.path.isdir(os.path.join(REF, "bl_krylov")):
        raise SystemExit("make_golden: pass --reference PATH (or set BDDA_REFERENCE) to the "
                         "block-DDA_Py checkout; got %r" % (REF,))
    _stub_matplotlib()
    sys.path.insert(0, REF)
    from mvp_fft import mvp_fft
    from bl_krylov import bl_krylov
    from bl_dda import scatterer
    from shape_model import gaussian_ellipsoid
    return mvp_fft, bl_krylov, scatterer, gaussian_ellipsoid


def _quiet_call(fn, *args):
    """Call fn, capturing its per-iteration prints; return (result, history)."""
    buf = io.StringIO()
    with contextlib.redirect_stdout(buf):
        res = fn(*args)
    hist = [float(line.split("err=")[1]) for line in buf.getvalue().splitlines()
            if line.startswith("iter=")]
    return res, hist


def so3_euler(L: int, seed: int) -> np.ndarray:
    """SO(3)-uniform ZYZ Euler angles: alpha, gamma ~ U[0, 2pi), beta = arccos U[-1, 1]."""
    rng = np.random.default_rng(seed)
    a = rng.uniform(0.0, 2 * np.pi, L)
    b = np.arccos(rng.uniform(-1.0, 1.0, L))
    g = rng.uniform(0.0, 2 * np.pi, L)
    return np.column_stack([a, b, g])


def gre_geometry(ge, r_v_base, bc, ab, beta, seed, lattice_lf=None):
    """The reference's geometry pipeline (run_dda.py:21-35) with an optional spacing override."""
    rng = np.random.default_rng(seed)
    gre = ge.gaussian_ellipsoid_shape_model(r_v_base, bc, ab, beta)
    if lattice_lf is not None:
        gre.lattice_lf = lattice_lf
    r_pts, _ = gre.compute_r_points_on_GRE(rng)
    _, lattice_n, grid = gre.create_cuboid_lattice_that_encloses_GRE_shape(r_pts)
    dist = gre.find_nearest_distance_from_the_GRE_surf(grid, r_pts)
    is_in = gre.extract_lattice_address_in_GRE_volume(
        gre.lattice_lf, gre.distance_factor, lattice_n, dist)
    nx, ny, nz = (int(v) for v in lattice_n)
    g3 = grid.reshape(nx, ny, nz, 3)
    axes = (g3[:, 0, 0, 0].copy(), g3[0, :, 0, 1].copy(), g3[0, 0, :, 2].copy())
    return dict(name=gre.name, lattice_n=np.asarray(lattice_n, dtype=np.int64),
                lattice_lf=float(gre.lattice_lf), grid=grid, is_in=np.asarray(is_in, bool),
                x_axis=axes[0], y_axis=axes[1], z_axis=axes[2], surface=r_pts,
                thr=float(gre.distance_factor * gre.lattice_lf))


def geometry_record(geo) -> dict:
    return dict(lattice_n=geo["lattice_n"], lattice_lf=geo["lattice_lf"],
                mask_bits=np.packbits(geo["is_in"]), n_cells=geo["is_in"].size,
                x_axis=geo["x_axis"], y_axis=geo["y_axis"], z_axis=geo["z_axis"])


def run_reference_solve(sc, bk, geo, m_p_xyz, wl_0, m_m, euler, solver, tol, itermax):
    target = sc.Target(geo["name"] or "gre", geo["lattice_n"], geo["lattice_lf"],
                       geo["grid"], geo["is_in"], m_p_xyz)
    inc = sc.IncidentField(wl_0, m_m, euler)
    with contextlib.redirect_stdout(io.StringIO()):
        dd = sc.DiscreteDipoles(target, inc)
    dd.set_interaction_matrix()
    fn = bk.bl_cocg_rq_jacobi_mvp_fft if solver == "cocg" else bk.bl_bicgstab_jacobi_mvp_fft
    (X, it_fin, err_fin), hist = _quiet_call(
        fn, dd.lattice_n, dd.f, dd.lattice_address_in_target, dd.Au_til,
        dd.diag_A, dd.B, tol, itermax)
    # observables exactly as solve_matrix_equation + compute_* do (scatterer.py:164-227)
    dd.X = X
    dd.P = X.T.reshape(dd.L, dd.num_element_occupy, 3)
    dd.E = dd.P * (4 * np.pi) / ((dd.eper_r[np.newaxis, :, :] - 1) * dd.element_vol)
    c_abs = dd.compute_C_abs()
    c_ext = dd.compute_C_ext()
    s_fw_t, s_fw_p = dd.compute_PCAS_observable_S_fw()
    s_bk = dd.compute_OCBS_observable_S_bk()
    return dict(X=X, iter_fin=it_fin, err_fin=err_fin, history=np.array(hist),
                C_abs=c_abs, C_ext=c_ext, S_fw_theta=s_fw_t, S_fw_phi=s_fw_p,
                S_bk=s_bk, S_bk_theta=dd.S_bk_OCBS_theta, S_bk_phi=dd.S_bk_OCBS_phi,
                diag_A=dd.diag_A, B=dd.B, ve_radius=dd.ve_radius, dpl=dd.dpl)


CFG2_M_P = np.array([1.55 + 0.001j, 1.60 + 0.001j, 1.52 + 0.002j])


def cfg2_geometry(ge):
    """Config 2 particle: GRE x=20 (m_m=1.33, wl=1), ab 0.7, bc 0.8, beta 0.1, seed 1, lambda_m/16."""
    m_m, wl_0 = 1.33, 1.0
    lam_m = wl_0 / m_m
    r_v = 20.0 * lam_m / (2 * np.pi)
    return gre_geometry(ge, r_v, 0.8, 0.7, 0.1, 1, lattice_lf=lam_m / 16), wl_0, m_m


def cfg2_chunk_fixture(bk, sc, ge) -> dict:
    """The reference's own block-BiCGSTAB solve of config 2, orientations 0-7, to 1e-5.

    The solve runs through the reference's DiscreteDipoles + bl_bicgstab_jacobi_mvp_fft
    on all host threads (DDA_FFT_WORKERS as set by the caller); its wall time is
    recorded beside the results.  X (168 MB) is kept only at 96 evenly spaced
    dipoles.
    """
    geo, wl_0, m_m = cfg2_geometry(ge)
    euler = so3_euler(64, 2)[:8]
    t0 = time.perf_counter()
    res = run_reference_solve(sc, bk, geo, CFG2_M_P, wl_0, m_m, euler, "bicgstab", 1e-5, 300)
    wall = time.perf_counter() - t0
    n_occ = int(geo["is_in"].sum())
    dip = np.unique(np.linspace(0, n_occ - 1, 96).astype(np.int64))
    rows = (3 * dip[:, None] + np.arange(3)[None, :]).ravel()
    from mvp_fft import mvp_fft as _mf
    rec = dict(lattice_n=geo["lattice_n"], n_occ=n_occ, mask_bits=np.packbits(geo["is_in"]),
               euler=euler, m_p_xyz=CFG2_M_P, wl_0=wl_0, m_m=m_m, tol=1e-5, itermax=300,
               sample_dipoles=dip, X_rows=res["X"][rows],
               wall_s=wall, cpu_count=os.cpu_count() or 1, fft_workers=int(_mf._FFT_WORKERS))
    rec.update({k2: res[k2] for k2 in ("iter_fin", "err_fin", "history", "C_abs", "C_ext",
                                       "S_fw_theta", "S_fw_phi", "S_bk")})
    return rec


def small_fixtures(mf, bk, sc, ge) -> dict:
    rng = np.random.default_rng(20261203)
    out = {}

    # --- L1 Green's tensor ----------------------------------------------------
    n, lf, k = [3, 4, 5], 0.05, 2 * np.pi * 1.33 / 0.8
    out["green_small"] = dict(n=np.array(n), lf=lf, k=k,
                              A=mf.build_interaction_tensor(n, lf, k),
                              A_til=mf.fft_init(n, 3, lf, k))

    # --- L1 fft_mvp -----------------------------------------------------------
    n, lf, k = [5, 6, 7], 0.04, 2 * np.pi / 0.55
    Nc = int(np.prod(n))
    P = rng.standard_normal((3 * Nc, 3)) + 1j * rng.standard_normal((3 * Nc, 3))
    p1 = rng.standard_normal(3 * Nc) + 1j * rng.standard_normal(3 * Nc)
    til = mf.fft_init(n, 3, lf, k)
    out["fft_mvp_small"] = dict(n=np.array(n), lf=lf, k=k, P=P, Y=mf.fft_mvp(n, 3, til, P),
                                p1=p1, y1=mf.fft_mvp(n, 3, til, p1))

    # --- L2 block MVP on a ragged occupancy --------------------------------------
    n, lf, k = [6, 5, 7], 0.05, 2 * np.pi * 1.2 / 0.6
    Nc = int(np.prod(n))
    occ = rng.random(Nc) < 0.55
    address = np.where(occ)[0]
    N = address.size
    diag = (rng.standard_normal(3 * N) + 5.0) + 1j * rng.standard_normal(3 * N)
    S = rng.standard_normal((3 * N, 4)) + 1j * rng.standard_normal((3 * N, 4))
    til = mf.fft_init(n, 3, lf, k)
    full_idx = bk._build_scatter_index(address, 3)
    out["block_mvp_small"] = dict(n=np.array(n), lf=lf, k=k, address=address, diag_A=diag,
                                  S=S, full_idx=full_idx,
                                  AS=bk._block_mvp(n, 3, til, full_idx, diag, S, 1.0 / diag))

    # --- L2 solvers on a small blob --------------------------------------------
    n = [8, 7, 6]
    I, J, K = np.meshgrid(*[np.arange(v) for v in n], indexing="ij")
    blob = ((I - 3.5) / 4.2) ** 2 + ((J - 3.0) / 3.6) ** 2 + ((K - 2.5) / 3.1) ** 2 <= 1.0
    address = np.where(blob.ravel())[0]
    N = address.size
    lf, wl_0, m_m = 0.03, 0.6, 1.1
    kk = 2 * np.pi * m_m / wl_0
    m_p = np.array([1.45 + 0.02j, 1.5 + 0.01j, 1.55 + 0.03j])
    vol = lf ** 3
    eper_r = (np.ones((N, 3)) * m_p) ** 2 / m_m ** 2
    a0 = (3 / (4 * np.pi)) * ((eper_r - 1) / (eper_r + 2)) * vol
    arad = (3 * vol / (4 * np.pi)) ** (1 / 3)
    Mt = (8 * np.pi / 3) * ((1 - 1j * kk * arad) * np.exp(1j * kk * arad) - 1)
    diag = (1.0 / (a0 / (1 - Mt * a0 / vol))).ravel()
    B = rng.standard_normal((3 * N, 3)) + 1j * rng.standard_normal((3 * N, 3))
    til = mf.fft_init(n, 3, lf, kk)
    rec = dict(n=np.array(n), lf=lf, k=kk, address=address, diag_A=diag, B=B)
    for name, fn in (("bicgstab", bk.bl_bicgstab_jacobi_mvp_fft),
                     ("cocg", bk.bl_cocg_rq_jacobi_mvp_fft)):
        (X, it, err), hist = _quiet_call(fn, n, 3, address, til, diag, B, 1e-5, 200)
        rec[name + "_X"] = X
        rec[name + "_iter_fin"] = it
        rec[name + "_err_fin"] = err
        rec[name + "_history"] = np.array(hist)
    out["solver_small"] = rec

    # --- test_dda.ipynb known-answer case ----------------------------------------
    geo = gre_geometry(ge, 0.2, 1, 1, 0.0, 1234)          # test_dda.ipynb cells 1-2
    r2 = np.random.default_rng(12345)                      # test_dda.ipynb cell 5
    a_deg = r2.uniform(0, 360, 10).reshape(10, 1)
    b_deg = r2.uniform(0, 180, 10).reshape(10, 1)
    g_deg = r2.uniform(0, 360, 10).reshape(10, 1)
    euler = np.radians(np.hstack((a_deg, b_deg, g_deg)))
    m_p = np.array([1.5 + 0.01j] * 3, dtype=np.complex64)  # test_dda.ipynb cell 3
    res = run_reference_solve(sc, bk, geo, m_p, 0.834, 1.329, euler, "bicgstab", 1e-2, 25)
    rec = geometry_record(geo)
    rec.update(euler=euler, m_p_xyz=m_p, wl_0=0.834, m_m=1.329, tol=1e-2, itermax=25)
    rec.update({k2: v for k2, v in res.items() if k2 not in ("B", "X")})
    out["kat_test_dda"] = rec

    # --- config 1: sphere x=5, spacing lambda/16, COCG-rq to 1e-5, L=8 ----------
    r_v = 5.0 / (2 * np.pi)
    geo = gre_geometry(ge, r_v, 1.0, 1.0, 0.0, 0, lattice_lf=1.0 / 16)
    euler = so3_euler(8, 0)
    m_p = np.array([1.5 + 0.01j] * 3)
    res = run_reference_solve(sc, bk, geo, m_p, 1.0, 1.0, euler, "cocg", 1e-5, 300)
    rec = geometry_record(geo)
    rec.update(euler=euler, m_p_xyz=m_p, wl_0=1.0, m_m=1.0, tol=1e-5, itermax=300)
    rec.update({k2: v for k2, v in res.items() if k2 not in ("X", "B", "diag_A")})
    # the same case with BiCGSTAB, and both solvers converged to 1e-11: at 1e-5
    # the iterate depends on rounding (a 1e-16 change of B moves S_bk by ~1e-5),
    # at 1e-11 the outputs are fixed by the problem to ~1e-11
    for solver, tol in (("bicgstab", 1e-5), ("cocg", 1e-11), ("bicgstab", 1e-11)):
        r = run_reference_solve(sc, bk, geo, m_p, 1.0, 1.0, euler, solver, tol, 300)
        tag = "%s_%s_" % (solver, "tight" if tol < 1e-6 else "tol5")
        for key in ("iter_fin", "err_fin", "history", "C_abs", "C_ext", "S_fw_theta",
                    "S_fw_phi", "S_bk"):
            rec[tag + key] = r[key]
    out["geometry_cfg1"] = rec

    # --- config 2 geometry --------------------------------------------------------
    geo, wl_0, m_m = cfg2_geometry(ge)
    rec = geometry_record(geo)
    # the reference's surface points and near-surface threshold: the surface
    # comes from LAPACK's eigh, whose last bits vary with the CPU's code path,
    # so the lattice occupancy is checked from these on any machine
    rec.update(euler=so3_euler(64, 2), wl_0=wl_0, m_m=m_m, m_p_xyz=CFG2_M_P, surface=geo["surface"],
               thr=geo["thr"])
    out["geometry_cfg2"] = rec
    return out


SWEEP_SMALL = dict(wl_m_m_pairs=np.array([[0.633, 1.330], [0.8337, 1.329]]),
                   m_p_xyz_list=np.array([[1.5 + 0j] * 3, [1.55 + 0.01j, 1.5 + 0.01j, 1.6 + 0.02j]]),
                   r_v_base_list=np.array([0.08, 0.12]), bc_ratio_list=np.array([1.5]),
                   ab_ratio_list=np.array([1.2]), gre_beta_list=np.array([0.1]), num_orientations=8,
                   rng_seed=12345, max_try=4)


def sweep_small_fixture(sc, ge, mie) -> dict:
    """A small sweep run the way run_dda.py runs one (run_dda.py:21-146), with the
    reference's own classes; run_dda.py itself opens an HDF5 file at import
    time, so its loop is restated here step for step."""
    sp = SWEEP_SMALL
    P, M = len(sp["wl_m_m_pairs"]), len(sp["m_p_xyz_list"])
    geo_shape = (len(sp["r_v_base_list"]), len(sp["bc_ratio_list"]), len(sp["ab_ratio_list"]),
                 len(sp["gre_beta_list"]))
    L = sp["num_orientations"]
    cond = (P, M) + geo_shape
    out = {k: v for k, v in sp.items()}
    out["r_ve"] = np.zeros(geo_shape)
    out["Euler_angles"] = np.zeros(cond + (L, 3))
    for k in ("C_abs", "C_ext"):
        out[k] = np.zeros(cond + (L,))
    for k in ("S_fw_PCAS_theta", "S_fw_PCAS_phi", "S_bk_OCBS"):
        out[k] = np.zeros(cond + (L,), dtype=np.complex128)
    for k in ("C_abs_mie", "C_ext_mie"):
        out[k] = np.zeros(cond)
    for k in ("S_fw_PCAS_mie", "S_bk_OCBS_mie"):
        out[k] = np.zeros(cond, dtype=np.complex128)
    out["tries"] = np.zeros(cond, dtype=np.int64)
    for i_rv, rv in enumerate(sp["r_v_base_list"]):
        for i_bc, bc in enumerate(sp["bc_ratio_list"]):
            for i_ab, ab in enumerate(sp["ab_ratio_list"]):
                for i_bt, bt in enumerate(sp["gre_beta_list"]):
                    s4 = (i_rv, i_bc, i_ab, i_bt)
                    rng = np.random.default_rng(sp["rng_seed"])
                    gre = ge.gaussian_ellipsoid_shape_model(rv, bc, ab, bt)
                    r_pts, _ = gre.compute_r_points_on_GRE(rng)
                    _, lattice_n, grid = gre.create_cuboid_lattice_that_encloses_GRE_shape(r_pts)
                    dist = gre.find_nearest_distance_from_the_GRE_surf(grid, r_pts)
                    is_in = gre.extract_lattice_address_in_GRE_volume(gre.lattice_lf, gre.distance_factor,
                                                                      lattice_n, dist)
                    r_ve = np.cbrt(3.0 * gre.lattice_lf ** 3 * int(is_in.sum()) / (4 * np.pi))
                    out["r_ve"][s4] = r_ve
                    nx, ny, nz = (int(v) for v in lattice_n)
                    g3 = grid.reshape(nx, ny, nz, 3)
                    tag = "shape_%d_%d_%d_%d_" % s4
                    out[tag + "lattice_n"] = np.asarray(lattice_n, dtype=np.int64)
                    out[tag + "lattice_lf"] = float(gre.lattice_lf)
                    out[tag + "x_axis"] = g3[:, 0, 0, 0].copy()
                    out[tag + "y_axis"] = g3[0, :, 0, 1].copy()
                    out[tag + "z_axis"] = g3[0, 0, :, 2].copy()
                    out[tag + "mask_bits"] = np.packbits(np.asarray(is_in, bool))
                    out[tag + "name"] = gre.name
                    for i_pair, (wl_0, m_m) in enumerate(sp["wl_m_m_pairs"]):
                        for i_mp, m_p_xyz in enumerate(sp["m_p_xyz_list"]):
                            idx6 = (i_pair, i_mp) + s4
                            target = sc.Target(gre.name, lattice_n, gre.lattice_lf, grid, is_in, m_p_xyz)
                            rng2 = np.random.default_rng(sp["rng_seed"] + 1)
                            res = None
                            for i_try in range(1, sp["max_try"] + 1):
                                euler = np.column_stack([rng2.uniform(0, 2 * np.pi, L), rng2.uniform(0, np.pi, L),
                                                         rng2.uniform(0, 2 * np.pi, L)])
                                with contextlib.redirect_stdout(io.StringIO()):
                                    dd = sc.DiscreteDipoles(target, sc.IncidentField(wl_0, m_m, euler))
                                    dd.set_interaction_matrix()
                                    dd.solve_matrix_equation()
                                if dd.converge:
                                    res = (dd.compute_C_abs(), dd.compute_C_ext(),
                                           *dd.compute_PCAS_observable_S_fw(), dd.compute_OCBS_observable_S_bk())
                                    break
                            if res is None:
                                res = tuple(np.full(L, np.nan) for _ in range(5))
                            out["Euler_angles"][idx6] = euler
                            out["tries"][idx6] = i_try
                            for k, v in zip(("C_abs", "C_ext", "S_fw_PCAS_theta", "S_fw_PCAS_phi", "S_bk_OCBS"),
                                            res):
                                out[k][idx6] = v
                            _, q_abs, q_ext, s_fw, s_bk = mie.mie_compute_q_and_s(
                                wl_0, m_m, r_ve, complex(np.mean(m_p_xyz)), nang=3)
                            out["C_abs_mie"][idx6] = q_abs * np.pi * r_ve ** 2
                            out["C_ext_mie"][idx6] = q_ext * np.pi * r_ve ** 2
                            out["S_fw_PCAS_mie"][idx6] = s_fw
                            out["S_bk_OCBS_mie"][idx6] = s_bk
    return out


def mie_fixture(mie) -> dict:
    """The reference's Mie routine on a spread of sizes and indices (complex64 amplitudes)."""
    cases = [(0.633, 1.33, 0.05, 1.5 + 0j), (0.8337, 1.329, 0.2027, 1.5 + 0.05j), (0.55, 1.0, 0.5, 1.53 + 0.005j),
             (1.0, 1.0, 5 / (2 * np.pi), 1.5 + 0.01j), (0.45, 1.0, 1.2, 1.6 + 0.1j), (0.532, 1.331, 0.01, 2.0 + 1.0j)]
    rows = np.array([[wl, mm, r, mp.real, mp.imag] for wl, mm, r, mp in cases])
    q = np.array([mie.mie_compute_q_and_s(wl, mm, r, mp, nang=3)[:3] for wl, mm, r, mp in cases])
    s = np.array([mie.mie_compute_q_and_s(wl, mm, r, mp, nang=3)[3:] for wl, mm, r, mp in cases])
    return dict(cases=rows, Q_sca_abs_ext=q, S_fw_bk=s.astype(np.complex128))


SMALL = ("green_small", "fft_mvp_small", "block_mvp_small", "solver_small", "kat_test_dda",
         "geometry_cfg1", "geometry_cfg2")


def main(argv=None) -> None:
    global REF
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--reference", default=None, help="block-DDA_Py checkout (else $BDDA_REFERENCE)")
    ap.add_argument("fixtures", nargs="*", help="fixture names (default: all small ones)")
    a = ap.parse_args(argv)
    REF = a.reference or REF
    names = a.fixtures or list(SMALL)
    unknown = set(names) - set(SMALL) - {"solve_cfg2_chunk", "sweep_small", "mie_small"}
    if unknown:
        raise SystemExit("unknown fixture(s): %s" % sorted(unknown))
    mf, bk, sc, ge = _import_reference()
    out = {}
    if set(names) & set(SMALL):
        out.update({k: v for k, v in small_fixtures(mf, bk, sc, ge).items() if k in names})
    if "sweep_small" in names or "mie_small" in names:
        from analytical_scattering_theories import homogeneous_sphere as mie
        if "sweep_small" in names:
            out["sweep_small"] = sweep_small_fixture(sc, ge, mie)
        if "mie_small" in names:
            out["mie_small"] = mie_fixture(mie)
    if "solve_cfg2_chunk" in names:
        out["solve_cfg2_chunk"] = cfg2_chunk_fixture(bk, sc, ge)
    for name, rec in out.items():
        path = os.path.join(HERE, name + ".npz")
        np.savez_compressed(path, **rec)
        print("%-18s %8.1f KB" % (name, os.path.getsize(path) / 1024))


if __name__ == "__main__":
    main()
