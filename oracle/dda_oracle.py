"""CPU oracle for the block-DDA hot path -- TEST INFRASTRUCTURE ONLY.

This module restates, in NumPy/SciPy, the algorithm of the reference
block-DDA_Py v0.3.0 for the path that the CUDA library replaces:

* the Goodman doubled-grid Green's tensor and its FFT  (mvp_fft/mvp_fft.py:13-119)
* the FFT off-diagonal matrix-vector product            (mvp_fft/mvp_fft.py:122-173)
* the sparse<->cuboid scatter index and block MVP       (bl_krylov/bl_krylov.py:5-55)
* block-COCG-rq and block-BiCGSTAB (Jacobi-preconditioned) (bl_krylov/bl_krylov.py:58-187)
* the CR2009 polarizability, incident field, RHS and the
  observables C_abs, C_ext, S_fw (PCAS), S_bk (OCBS)    (bl_dda/scatterer.py:33-227)

It is the checker, never the product: only ``tests/``, ``__graft_entry__.smoke``
and the ``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` may import
it.  The CUDA product path never routes through here.

Pinning: every function is checked against golden vectors produced by the
live reference (``tests/golden/make_golden.py``) and against the recorded
outputs of the reference's ``test_dda.ipynb`` (lines 92, 162, 189-191,
231-232, 316-321).  Third-party arithmetic follows the reference's pins:
FFTs are scipy.fft (pocketfft; scipy==1.17.1 in requirements.txt:99), dense
linear algebra is numpy.linalg (LAPACK; numpy==2.4.2, requirements.txt:73).
"""
from __future__ import annotations

import os

import numpy as np
import scipy.fft

# Thread count for scipy.fft, same environment knob and default as the
# reference (mvp_fft/mvp_fft.py:9-10): DDA_FFT_WORKERS, else cpu_count-2.
FFT_WORKERS = int(os.environ.get("DDA_FFT_WORKERS", max(1, (os.cpu_count() or 1) - 2)))

# Order of the six unique entries of the symmetric 3x3 Green's tensor.
SYM6 = ((0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (2, 2))


# ----------------------------------------------------------------------------
# L1: Green's tensor and the FFT matrix-vector product
# ----------------------------------------------------------------------------
def _displacements(N: int, M: int) -> tuple[np.ndarray, np.ndarray]:
    """Integer displacement carried by each index of a cyclic axis of length M.

    Index I holds displacement I for I <= N-1 and I-M for I >= M-(N-1); the
    remaining indices carry no pair of cuboid points and are marked invalid.
    With M = 2N this is exactly the reference's map (mvp_fft.py:49-51) with
    its Nyquist plane I = N zeroed (mvp_fft.py:89-92).
    """
    idx = np.arange(M)
    disp = np.where(idx <= N - 1, idx, idx - M).astype(np.float64)
    valid = (idx <= N - 1) | (idx >= M - (N - 1))
    return disp, valid


def green_components(n, lf: float, k: float, m=None) -> np.ndarray:
    """A'(r) = e^{ikr}/r [k^2 (r^ r^ - I) + (1 - ikr)/r^2 (I - 3 r^ r^)].

    Returns the six unique components (order ``SYM6``) on a cyclic grid of
    size ``m`` (default: the reference's doubled grid 2n), shape
    (Mx, My, Mz, 6) complex128.  Origin and non-physical positions are zero.
    Formula: mvp_fft.py:77-84; origin zeroing: mvp_fft.py:86-87.
    """
    n = [int(v) for v in n]
    m = [2 * v for v in n] if m is None else [int(v) for v in m]
    axes = [_displacements(n[a], m[a]) for a in range(3)]
    d = [axes[a][0] * lf for a in range(3)]
    X, Y, Z = np.meshgrid(d[0], d[1], d[2], indexing="ij", sparse=True)
    r = np.sqrt(X * X + Y * Y + Z * Z)
    rr = np.where(r == 0.0, 1.0, r)
    unit = (X / rr, Y / rr, Z / rr)
    phase = np.exp(1j * k * rr) / rr
    near = (1.0 - 1j * k * rr) / (rr * rr)
    out = np.empty(tuple(m) + (6,), dtype=np.complex128)
    for c, (a, b) in enumerate(SYM6):
        uu = unit[a] * unit[b]
        delta = 1.0 if a == b else 0.0
        out[..., c] = phase * (k * k * (uu - delta) + near * (delta - 3.0 * uu))
    valid = (axes[0][1][:, None, None] & axes[1][1][None, :, None]
             & axes[2][1][None, None, :])
    out[~valid] = 0.0
    out[0, 0, 0] = 0.0
    return out


def sym6_to_full(g6: np.ndarray) -> np.ndarray:
    """(..., 6) symmetric storage -> (..., 3, 3)."""
    full = np.empty(g6.shape[:-1] + (3, 3), dtype=g6.dtype)
    for c, (a, b) in enumerate(SYM6):
        full[..., a, b] = g6[..., c]
        full[..., b, a] = g6[..., c]
    return full


def build_interaction_tensor(n, lf, k) -> np.ndarray:
    """Reference layout (2Nx, 2Ny, 2Nz, 3, 3) c128 (mvp_fft.py:13-94)."""
    return sym6_to_full(green_components(n, lf, k))


def fft_init(n, f, lf, k) -> np.ndarray:
    """FFT of the interaction tensor over the three grid axes (mvp_fft.py:97-119)."""
    if f != 3:
        raise ValueError("fft_init: only f=3 (electric dipoles) is supported.")
    return scipy.fft.fftn(build_interaction_tensor(n, lf, k), axes=(0, 1, 2),
                          workers=FFT_WORKERS)


def fft_mvp(n, f, Ghat, P) -> np.ndarray:
    """Off-diagonal product A_off @ P via the doubled grid (mvp_fft.py:122-173).

    ``P`` is (f*Nc,) or (f*Nc, L) on the full cuboid (C-order x,y,z then
    component).  Zero-pad, forward FFT, per-frequency 3x3 @ 3xL product,
    inverse FFT, crop.
    """
    Nx, Ny, Nz = (int(v) for v in n)
    one_col = P.ndim == 1
    cols = P[:, None] if one_col else P
    L = cols.shape[1]
    grid = np.zeros((2 * Nx, 2 * Ny, 2 * Nz, f, L), dtype=np.complex128)
    grid[:Nx, :Ny, :Nz] = cols.reshape(Nx, Ny, Nz, f, L)
    spec = scipy.fft.fftn(grid, axes=(0, 1, 2), workers=FFT_WORKERS)
    spec = np.matmul(Ghat, spec)
    back = scipy.fft.ifftn(spec, axes=(0, 1, 2), workers=FFT_WORKERS)
    out = back[:Nx, :Ny, :Nz].reshape(f * Nx * Ny * Nz, L)
    return out[:, 0] if one_col else out


# ----------------------------------------------------------------------------
# L2: block MVP and block Krylov solvers
# ----------------------------------------------------------------------------
def scatter_index(address, f: int) -> np.ndarray:
    """full_idx[f*m + c] = f*address[m] + c (bl_krylov.py:5-24)."""
    address = np.asarray(address, dtype=np.int64)
    return (address[:, None] * f + np.arange(f)[None, :]).ravel()


def block_mvp(n, f, Ghat, full_idx, diag_a, S, jpre) -> np.ndarray:
    """jpre * (diag_a * S + gather(A_off scatter(S)))  (bl_krylov.py:27-55)."""
    nc = int(np.prod(n))
    full = np.zeros((f * nc, S.shape[1]), dtype=np.complex128)
    full[full_idx] = S
    off = fft_mvp(n, f, Ghat, full)
    return (diag_a[:, None] * S + off[full_idx]) * jpre[:, None]


def cocg_rq(n, f, address, Ghat, diag_a, B, tol, itermax, history=None):
    """Block-COCG-rq, Jacobi-preconditioned (bl_krylov.py:58-118).

    Returns (X, iter_fin, err_fin) with iter_fin the 0-based index of the last
    iteration run.  Bilinear (unconjugated) transposes throughout.  When
    ``history`` is a list, the per-iteration relative residual is appended.
    """
    jpre = 1.0 / diag_a
    idx = scatter_index(address, f)
    Bj = B * jpre[:, None]
    bnorm = np.linalg.norm(Bj)
    X = np.zeros_like(B)
    Q, xi = np.linalg.qr(Bj, mode="reduced")
    S = Q
    it_last, err_last = 0, float("inf")
    for it in range(itermax):
        AS = block_mvp(n, f, Ghat, idx, diag_a, S, jpre)
        alpha = np.linalg.solve(S.T @ AS, Q.T @ Q)
        X = X + S @ (alpha @ xi)
        Qn, tau = np.linalg.qr(Q - AS @ alpha, mode="reduced")
        xi = tau @ xi
        err = np.linalg.norm(xi) / bnorm
        if history is not None:
            history.append(err)
        it_last, err_last = it, err
        if err < tol:
            break
        beta = np.linalg.solve(Q.T @ Q, tau.T @ (Qn.T @ Qn))
        Q = Qn
        S = Q + S @ beta
    return X, it_last, err_last


def bicgstab(n, f, address, Ghat, diag_a, B, tol, itermax, history=None, X0=None):
    """Block-BiCGSTAB, Jacobi-preconditioned (bl_krylov.py:121-187).

    The stopping test is the recursively updated global Frobenius residual
    ||R||_F / ||M^-1 B||_F (bl_krylov.py:177).  ``X0`` (default zero, as in
    the reference) seeds the iterate; R starts at M^-1 (B - A X0).
    """
    jpre = 1.0 / diag_a
    idx = scatter_index(address, f)
    Bj = B * jpre[:, None]
    bnorm = np.linalg.norm(Bj)
    if X0 is None:
        X = np.zeros_like(B)
        R = Bj.copy()
    else:
        X = np.array(X0, dtype=np.complex128)
        R = Bj - block_mvp(n, f, Ghat, idx, diag_a, X, jpre)
    P = R.copy()
    R0h = R.conj().T
    it_last, err_last = 0, float("inf")
    for it in range(itermax):
        V = block_mvp(n, f, Ghat, idx, diag_a, P, jpre)
        RV = R0h @ V
        alpha = np.linalg.solve(RV, R0h @ R)
        T = R - V @ alpha
        Z = block_mvp(n, f, Ghat, idx, diag_a, T, jpre)
        zeta = np.trace(Z.conj().T @ T) / np.trace(Z.conj().T @ Z)
        X = X + P @ alpha + zeta * T
        R = T - zeta * Z
        err = np.linalg.norm(R) / bnorm
        if history is not None:
            history.append(err)
        it_last, err_last = it, err
        if err < tol:
            break
        beta = np.linalg.solve(RV, -(R0h @ Z))
        P = R + (P - zeta * V) @ beta
    return X, it_last, err_last


def true_residual(n, f, address, Ghat, diag_a, B, X) -> float:
    """||M^-1 (B - A X)||_F / ||M^-1 B||_F with M = diag(A) (the Jacobi residual)."""
    jpre = 1.0 / diag_a
    idx = scatter_index(address, f)
    Bj = B * jpre[:, None]
    R = Bj - block_mvp(n, f, Ghat, idx, diag_a, X, jpre)
    return float(np.linalg.norm(R) / np.linalg.norm(Bj))


# ----------------------------------------------------------------------------
# L3: incident field, polarizability, RHS, observables
# ----------------------------------------------------------------------------
def _rot_z(t):
    c, s = np.cos(t), np.sin(t)
    R = np.zeros(t.shape + (3, 3))
    R[..., 0, 0] = c; R[..., 0, 1] = -s
    R[..., 1, 0] = s; R[..., 1, 1] = c
    R[..., 2, 2] = 1.0
    return R


def _rot_y(t):
    c, s = np.cos(t), np.sin(t)
    R = np.zeros(t.shape + (3, 3))
    R[..., 0, 0] = c; R[..., 0, 2] = s
    R[..., 1, 1] = 1.0
    R[..., 2, 0] = -s; R[..., 2, 2] = c
    return R


def lab_to_particle(euler) -> np.ndarray:
    """Rotation taking lab vectors into the particle frame, one per orientation.

    The particle is oriented by intrinsic ZYZ Euler angles (alpha, beta,
    gamma); lab -> particle is the inverse, intrinsic ZYZ(-gamma, -beta,
    -alpha) = Rz(-gamma) Ry(-beta) Rz(-alpha)  (scatterer.py:67-70).
    """
    e = np.asarray(euler, dtype=np.float64)
    return _rot_z(-e[:, 2]) @ _rot_y(-e[:, 1]) @ _rot_z(-e[:, 0])


def incident_geometry(wl_0, m_m, euler) -> dict:
    """Wavenumber and lab-frame unit vectors rotated into the particle frame.

    Lab geometry: incidence +z with theta=+x, phi=+y; forward scattering the
    same; backscattering -z with theta=-x, phi=+y; circular incident
    polarisation e0 = theta/sqrt2 + i phi/sqrt2  (scatterer.py:46-85).
    """
    R = lab_to_particle(euler)
    ez = np.array([0.0, 0.0, 1.0]); ex = np.array([1.0, 0.0, 0.0]); ey = np.array([0.0, 1.0, 0.0])
    g = {"k": 2 * np.pi * m_m / wl_0, "eper_m": m_m ** 2}
    g["u_inc"] = R @ ez
    g["theta_inc"] = R @ ex
    g["phi_inc"] = R @ ey
    g["e0_inc"] = g["theta_inc"] / np.sqrt(2) + 1j * g["phi_inc"] / np.sqrt(2)
    g["u_fw"], g["theta_fw"], g["phi_fw"] = R @ ez, R @ ex, R @ ey
    g["u_bk"], g["theta_bk"], g["phi_bk"] = -(R @ ez), -(R @ ex), R @ ey
    return g


def polarizability(m_p_xyz, m_m, lf, k, n_occ):
    """CR2009-corrected Clausius-Mossotti polarizability (scatterer.py:137-148).

    Returns (eper_r (N,3), alpha (N,3), diag_A (3N,)) with diag_A ordered
    [x0, y0, z0, x1, ...].
    """
    vol = lf ** 3
    # m_p is promoted to complex128 before squaring, as the reference's
    # ones_like(float64) * m_p_xyz does (scatterer.py:24-25).
    mp = np.asarray(m_p_xyz).astype(np.complex128)
    eper_r = (np.ones((n_occ, 3)) * mp) ** 2 / (m_m ** 2)
    cm = (3 / (4 * np.pi)) * ((eper_r - 1) / (eper_r + 2)) * vol
    a = (3 * vol / (4 * np.pi)) ** (1 / 3)
    corr = (8 * np.pi / 3) * ((1 - 1j * k * a) * np.exp(1j * k * a) - 1)
    alpha = cm / (1 - corr * cm / vol)
    return eper_r, alpha, (1.0 / alpha).ravel()


def incident_field(k, u_inc, e0_inc, pos) -> np.ndarray:
    """E_inc[l, n, c] = e0[l, c] exp(i k u_l . r_n)  (scatterer.py:155-158)."""
    phase = np.exp(1j * k * (u_inc @ pos.T))
    return phase[:, :, None] * e0_inc[:, None, :]


def rhs(k, u_inc, e0_inc, pos) -> np.ndarray:
    """B (3N, L) with B[3n+c, l] = E_inc[l, n, c]  (scatterer.py:160-161)."""
    E = incident_field(k, u_inc, e0_inc, pos)
    L, N, _ = E.shape
    return E.reshape(L, 3 * N).T


def observables(X, geom, pos, eper_r, lf) -> dict:
    """C_abs, C_ext, S_fw (theta/phi) and S_bk from the solution block X (3N, L).

    P = X^T as (L, N, 3); E = 4 pi P / ((eper_r - 1) v) (scatterer.py:182-184);
    reductions per orientation follow scatterer.py:187-227.
    """
    k = geom["k"]
    L = X.shape[1]
    N = pos.shape[0]
    vol = lf ** 3
    P = X.T.reshape(L, N, 3)
    E = P * (4 * np.pi) / ((eper_r[None] - 1) * vol)
    out = {}
    if np.mean(eper_r.imag) >= 1e-12:
        out["C_abs"] = 4 * np.pi * k * np.sum(np.imag(P * np.conj(E)), axis=(1, 2))
    else:
        out["C_abs"] = np.zeros(L)
    Einc = incident_field(k, geom["u_inc"], geom["e0_inc"], pos)
    out["C_ext"] = 4 * np.pi * k * np.sum(np.imag(P * np.conj(Einc)), axis=(1, 2))
    r2 = np.sqrt(2)
    for tag in ("fw", "bk"):
        ph = np.exp(1j * k * (geom["u_" + tag] @ pos.T))
        pt = np.einsum("lnc,lc->ln", P, geom["theta_" + tag])
        pp = np.einsum("lnc,lc->ln", P, geom["phi_" + tag])
        st = k ** 2 * np.sum(pt * np.conj(r2 * ph), axis=1)
        sp = k ** 2 * np.sum(pp * np.conj(r2 * 1j * ph), axis=1)
        out["S_%s_theta" % tag] = st
        out["S_%s_phi" % tag] = sp
    out["S_bk"] = (-out["S_bk_theta"] + out["S_bk_phi"]) / r2
    return out


# ----------------------------------------------------------------------------
# Size-independent checks for full-size runs
# ----------------------------------------------------------------------------
def direct_offdiag_rows(rows, pos_idx, lf, k, S, f=3) -> np.ndarray:
    """Direct O(N) evaluation of selected output dipoles of A_off @ S.

    ``pos_idx`` (N_occ, 3) holds integer lattice coordinates of the occupied
    dipoles; ``S`` is (3 N_occ, L).  For each requested output dipole i the
    sum over all sources j != i of A'(r_i - r_j) S_j is formed in float64
    without any FFT.  This is the mathematical definition that the doubled
    grid FFT evaluates (mvp_fft.py:23-28), so it checks a full-size product
    at a handful of rows.
    """
    pos_idx = np.asarray(pos_idx, dtype=np.int64)
    L = S.shape[1]
    Sv = S.reshape(-1, f, L)
    out = np.zeros((len(rows), f, L), dtype=np.complex128)
    for o, i in enumerate(rows):
        d = (pos_idx[i][None, :] - pos_idx).astype(np.float64) * lf
        r = np.sqrt(np.sum(d * d, axis=1))
        mask = r > 0
        d, r, Sj = d[mask], r[mask], Sv[mask]
        u = d / r[:, None]
        ph = np.exp(1j * k * r) / r
        near = (1.0 - 1j * k * r) / (r * r)
        for a in range(3):
            acc = np.zeros(L, dtype=np.complex128)
            for b in range(3):
                delta = 1.0 if a == b else 0.0
                coef = ph * (k * k * (u[:, a] * u[:, b] - delta) + near * (delta - 3 * u[:, a] * u[:, b]))
                acc += coef @ Sj[:, b, :]
            out[o, a] = acc
    return out
