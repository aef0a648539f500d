"""Generate the golden fixtures in this folder from the live reference.

Run in a container where the reference block-DDA_Py v0.3.0 is checked out
(default ``/root/reference``, override with ``BDDA_REFERENCE``):

    python tests/golden/make_golden.py

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
                     surface seed 1, spacing lambda_m/16 -> 96x111x160
"""
from __future__ import annotations

import contextlib
import io
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.environ.get("BDDA_REFERENCE", "/root/reference")


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
                x_axis=axes[0], y_axis=axes[1], z_axis=axes[2])


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


def main() -> None:
    mf, bk, sc, ge = _import_reference()
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

    # --- config 2 geometry only (the solve is GPU-scale) ---------------------------
    m_m, wl_0 = 1.33, 1.0
    lam_m = wl_0 / m_m
    r_v = 20.0 * lam_m / (2 * np.pi)
    geo = gre_geometry(ge, r_v, 0.8, 0.7, 0.1, 1, lattice_lf=lam_m / 16)
    rec = geometry_record(geo)
    rec.update(euler=so3_euler(64, 2), wl_0=wl_0, m_m=m_m,
               m_p_xyz=np.array([1.55 + 0.001j, 1.60 + 0.001j, 1.52 + 0.002j]))
    out["geometry_cfg2"] = rec

    for name, rec in out.items():
        path = os.path.join(HERE, name + ".npz")
        np.savez_compressed(path, **rec)
        print("%-18s %8.1f KB" % (name, os.path.getsize(path) / 1024))


if __name__ == "__main__":
    main()
