"""GPU drop-in for the reference module ``bl_krylov.bl_krylov``.

Same names and signatures as bl_krylov/bl_krylov.py (block-DDA_Py v0.3.0):
``_build_scatter_index``, ``_block_mvp``, ``bl_cocg_rq_jacobi_mvp_fft`` and
``bl_bicgstab_jacobi_mvp_fft``.  The products, the block Gram reductions, the
small L x L solves and the block updates all run in libbdda.so.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from bdda_b200 import _lib
from bdda_b200.runtime import TORCH_DTYPE, Occupancy, precision_code, ptr, stream_ptr, to_device
from mvp_fft.mvp_fft import as_green


def _build_scatter_index(address, f):
    """full_idx[f*m + c] = f*address[m] + c (bl_krylov.py:5-24); host-side, as in the reference."""
    address = np.asarray(address, dtype=np.int64)
    return (address[:, None] * f + np.arange(f)[None, :]).ravel()


def _address_from_index(full_idx, f):
    full_idx = np.asarray(full_idx.cpu() if isinstance(full_idx, torch.Tensor) else full_idx)
    full_idx = full_idx.astype(np.int64).ravel()
    if full_idx.size % f:
        raise ValueError("full_idx length is not a multiple of f")
    address = full_idx[0::f] // f
    if not np.array_equal(_build_scatter_index(address, f), full_idx):
        raise ValueError("full_idx is not a scatter index built by _build_scatter_index")
    return address


def _block_mvp(n, f, Au_til, full_idx, DIAG_A, S, jpre, precision=None):
    """AS = jpre * (DIAG_A * S + A_off S) for all L columns (bl_krylov.py:27-55)."""
    if f != 3:
        raise ValueError("_block_mvp: only f=3 (electric dipoles) is supported.")
    g = as_green(n, Au_til)
    plan = g.plan
    prec = precision_code(precision)
    dt = TORCH_DTYPE[prec]
    occ = Occupancy(plan, _address_from_index(full_idx, f))
    to_numpy = not isinstance(S, torch.Tensor)
    Sd = to_device(S, dt, plan.device)
    if Sd.dim() != 2 or Sd.shape[0] != 3 * occ.n_occ:
        raise ValueError("S must be (%d, L), got %r" % (3 * occ.n_occ, tuple(Sd.shape)))
    L = int(Sd.shape[1])
    d = to_device(DIAG_A, dt, plan.device)
    j = to_device(jpre, dt, plan.device)
    out = torch.empty_like(Sd)
    work = g.workspace(prec, L)
    _lib.check(_lib.load().bdda_block_mvp(plan.handle, prec, L, ptr(g.ghat(prec)), ptr(occ.cell_map),
                                          ptr(d), ptr(j), ptr(Sd), ptr(out), ptr(work),
                                          stream_ptr(plan.device)), "bdda_block_mvp")
    return out.cpu().numpy() if to_numpy else out


MIXED = ("mixed", "c64-refine", "fp32-refine", "mixed-reliable")


def _solve(kind, n, f, address, Au_til, DIAG_A, B, tol, itermax, X0=None, precision=None,
           history=None, verbose=False, inner_tol=1e-4, max_outer=20):
    """Shared body of the block solvers (C entry points ``bdda_solve`` / ``bdda_refine_solve``)."""
    if f != 3:
        raise ValueError("only f=3 (electric dipoles) is supported.")
    g = as_green(n, Au_til)
    plan = g.plan
    mixed = isinstance(precision, str) and precision.lower() in MIXED
    reliable = mixed and precision.lower() == "mixed-reliable" and kind == _lib.BICGSTAB
    prec = _lib.C128 if mixed else precision_code(precision)
    occ = address if isinstance(address, Occupancy) else Occupancy(plan, address)
    to_numpy = not isinstance(B, torch.Tensor)
    Bd = to_device(B, torch.complex128, plan.device)
    if Bd.dim() != 2 or Bd.shape[0] != 3 * occ.n_occ:
        raise ValueError("B must be (%d, L), got %r" % (3 * occ.n_occ, tuple(Bd.shape)))
    L = int(Bd.shape[1])
    if L > 64:
        raise ValueError("at most 64 right-hand sides per block solve (got L=%d); split the block" % L)
    diag = to_device(DIAG_A, torch.complex128, plan.device).reshape(-1)
    if diag.numel() != 3 * occ.n_occ:
        raise ValueError("DIAG_A must have %d entries" % (3 * occ.n_occ))
    X0d = None if X0 is None else to_device(X0, torch.complex128, plan.device).reshape(Bd.shape).contiguous()
    lib = _lib.load()
    X = torch.empty_like(Bd)
    itermax = int(itermax)
    hist = (C.c_double * max(itermax, 1))()
    it = C.c_int(0)
    err = C.c_double(float("inf"))
    if mixed:
        nbytes = int(lib.bdda_refine_workspace_bytes(plan.handle, L, occ.n_occ))
        work = torch.empty(max(nbytes, 16), dtype=torch.uint8, device=plan.device)
        status = lib.bdda_refine_solve(plan.handle, kind, L, occ.n_occ, ptr(g.ghat(_lib.C128)),
                                       ptr(g.ghat(_lib.C64)), ptr(occ.cell_map), ptr(diag), ptr(Bd), ptr(X0d),
                                       float(tol), itermax,
                                       float(1e-2 if reliable else inner_tol),
                                       -abs(int(max_outer)) if reliable else abs(int(max_outer)), ptr(X),
                                       C.byref(it), C.byref(err), hist, ptr(work), nbytes,
                                       stream_ptr(plan.device))
        _lib.check(status, "bdda_refine_solve")
    else:
        nbytes = int(lib.bdda_solver_workspace_bytes(plan.handle, kind, prec, L, occ.n_occ))
        work = torch.empty(max(nbytes, 16), dtype=torch.uint8, device=plan.device)
        status = lib.bdda_solve(plan.handle, kind, prec, L, occ.n_occ, ptr(g.ghat(prec)), ptr(occ.cell_map),
                                ptr(diag), ptr(Bd), ptr(X0d), float(tol), itermax, ptr(X), C.byref(it),
                                C.byref(err), hist, ptr(work), nbytes, stream_ptr(plan.device))
        _lib.check(status, "bdda_solve")
    ran = 0 if itermax == 0 else it.value + 1
    if history is not None:
        history.extend(hist[i] for i in range(ran))
    if verbose:
        for i in range(ran):
            print("iter= {:}, err= {:.4f}".format(i, hist[i]))
    del work
    return (X.cpu().numpy() if to_numpy else X), it.value, err.value


def bl_cocg_rq_jacobi_mvp_fft(n, f, address, Au_til, DIAG_A, B, tol, itermax, X0=None,
                              precision=None, history=None, verbose=False, inner_tol=1e-4, max_outer=20):
    """Block-COCG-rq with Jacobi preconditioning (bl_krylov.py:58-118).

    Returns ``(X, iter_fin, err_fin)`` with the reference's meaning: X the
    (f*N_occ, L) solution, iter_fin the 0-based index of the last iteration,
    err_fin = ||xi||_F / ||M^-1 B||_F at that iteration.  Not converging is
    not an error.  Extra keywords (all optional): ``X0`` initial guess,
    ``precision`` "c128" (default), "c64" (FP32 throughout), "mixed" (FP32
    block solves restarted inside an FP64 iterative refinement; err_fin is
    then the true residual ||M^-1 (B - A X)|| / ||M^-1 B||; ``inner_tol``
    and ``max_outer`` tune it) or, for BiCGSTAB, "mixed-reliable" (one FP32
    recursion with FP64 residual replacement, for small L), ``history``
    list receiving the per-iteration residuals, ``verbose`` prints them like
    the reference.
    The QR factorisations are CholeskyQR (R with real positive diagonal
    instead of LAPACK's Householder signs); X and err are independent of
    that choice.
    """
    return _solve(_lib.COCG_RQ, n, f, address, Au_til, DIAG_A, B, tol, itermax, X0, precision,
                  history, verbose, inner_tol, max_outer)


def bl_bicgstab_jacobi_mvp_fft(n, f, address, Au_til, DIAG_A, B, tol, itermax, X0=None,
                               precision=None, history=None, verbose=False, inner_tol=1e-4, max_outer=20):
    """Block-BiCGSTAB with Jacobi preconditioning (bl_krylov.py:121-187).

    Returns ``(X, iter_fin, err_fin)`` as the reference; err_fin is the
    recursively updated ||R||_F / ||M^-1 B||_F.  A singular R0^H V raises
    numpy.linalg.LinAlgError like numpy.linalg.solve.  Extra keywords as for
    :func:`bl_cocg_rq_jacobi_mvp_fft`.
    """
    return _solve(_lib.BICGSTAB, n, f, address, Au_til, DIAG_A, B, tol, itermax, X0, precision,
                  history, verbose, inner_tol, max_outer)
