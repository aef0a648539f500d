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


# "mixed": complex128 Krylov vectors, complex64 products, complex128 true residual
# (bdda_mixed_solve); "mixed-fp32": complex64 vectors and products restarted
# inside FP64 refinement (bdda_refine_solve); "mixed-reliable": one complex64
# recursion with FP64 residual replacement (BiCGSTAB)
MIXED = ("mixed", "mixed-fp32", "c64-refine", "fp32-refine", "mixed-reliable")


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
        return _solve_in_blocks(kind, n, f, occ, g, DIAG_A, Bd, tol, itermax, X0, precision, history, verbose,
                                inner_tol, max_outer, to_numpy)
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
    if mixed and precision.lower() == "mixed":
        nbytes = int(lib.bdda_mixed_workspace_bytes(plan.handle, L, occ.n_occ))
        work = torch.empty(max(nbytes, 16), dtype=torch.uint8, device=plan.device)
        status = lib.bdda_mixed_solve(plan.handle, kind, L, occ.n_occ, ptr(g.ghat(_lib.C128)),
                                      ptr(g.ghat(_lib.C64)), ptr(occ.cell_map), ptr(diag), ptr(Bd), ptr(X0d),
                                      float(tol), itermax, abs(int(max_outer)), ptr(X), C.byref(it),
                                      C.byref(err), hist, ptr(work), nbytes, stream_ptr(plan.device))
        _lib.check(status, "bdda_mixed_solve")
    elif mixed:
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


def _solve_in_blocks(kind, n, f, occ, g, DIAG_A, Bd, tol, itermax, X0, precision, history, verbose, inner_tol,
                     max_outer, to_numpy):
    """More than 64 right-hand sides: ceil(L / 64) column blocks of near-equal
    width solved one after another (the reference iterates on all L columns as
    one block).  iter_fin and err_fin are the largest of the blocks' (the
    largest relative residual bounds that of the whole block); ``history``
    receives, per iteration, the largest residual among the blocks still
    iterating."""
    L = int(Bd.shape[1])
    nblk = (L + 63) // 64
    X = torch.empty_like(Bd)
    X0d = None if X0 is None else to_device(X0, torch.complex128, Bd.device).reshape(Bd.shape)
    its, errs, hists = [], [], []
    for b in range(nblk):
        l0, l1 = b * L // nblk, (b + 1) * L // nblk
        h = []
        Xb, it, err = _solve(kind, n, f, occ, g, DIAG_A, Bd[:, l0:l1].contiguous(), tol, itermax,
                             None if X0d is None else X0d[:, l0:l1].contiguous(), precision, h, verbose,
                             inner_tol, max_outer)
        X[:, l0:l1] = Xb
        its.append(it)
        errs.append(err)
        hists.append(h)
    if history is not None:
        for k in range(max(len(h) for h in hists)):
            history.append(max(h[k] for h in hists if k < len(h)))
    return (X.cpu().numpy() if to_numpy else X), max(its), max(errs)


def bl_cocg_rq_jacobi_mvp_fft(n, f, address, Au_til, DIAG_A, B, tol, itermax, X0=None,
                              precision=None, history=None, verbose=False, inner_tol=1e-4, max_outer=20):
    """Block-COCG-rq with Jacobi preconditioning (bl_krylov.py:58-118).

    Returns ``(X, iter_fin, err_fin)`` with the reference's meaning: X the
    (f*N_occ, L) solution, iter_fin the 0-based index of the last iteration,
    err_fin = ||xi||_F / ||M^-1 B||_F at that iteration.  Not converging is
    not an error.  Extra keywords (all optional): ``X0`` initial guess,
    ``precision`` "c128" (default), "c64" (FP32 throughout), "mixed"
    (complex128 Krylov vectors and small solves, complex64 products, the
    complex128 true residual judged at the end with warm restarts; err_fin
    is then the true residual ||M^-1 (B - A X)|| / ||M^-1 B||), "mixed-fp32"
    (complex64 block solves restarted inside an FP64 iterative refinement;
    ``inner_tol`` and ``max_outer`` tune it) or, for BiCGSTAB,
    "mixed-reliable" (one FP32 recursion with FP64 residual replacement, for
    small L), ``history``
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


# ---- batched solves (no reference counterpart: the reference solves one problem per call) ----
class _BatchProblem(C.Structure):
    """include/bdda.h: bdda_batch_problem."""
    _fields_ = [("plan", C.c_void_p), ("n_occ", C.c_int), ("ghat", C.c_void_p), ("ghat_c64", C.c_void_p),
                ("cell_map", C.c_void_p), ("diag", C.c_void_p), ("B", C.c_void_p), ("X0", C.c_void_p),
                ("X", C.c_void_p)]


_BATCH_MODES = {"c128": _lib.BATCH_C128, "fp64": _lib.BATCH_C128, "complex128": _lib.BATCH_C128,
                "c64": _lib.BATCH_C64, "fp32": _lib.BATCH_C64, "complex64": _lib.BATCH_C64,
                "mixed": _lib.BATCH_MIXED}


def _batch_entry(p):
    if isinstance(p, dict):
        n, address, Au_til, DIAG_A, B, X0 = (p["n"], p["address"], p["Au_til"], p["DIAG_A"], p["B"],
                                              p.get("X0"))
    else:
        n, address, Au_til, DIAG_A, B = p[:5]
        X0 = p[5] if len(p) > 5 else None
    g = as_green(n, Au_til)
    plan = g.plan
    occ = address if isinstance(address, Occupancy) else Occupancy(plan, address)
    to_numpy = not isinstance(B, torch.Tensor)
    Bd = to_device(B, torch.complex128, plan.device)
    if Bd.dim() != 2 or Bd.shape[0] != 3 * occ.n_occ:
        raise ValueError("B must be (%d, L), got %r" % (3 * occ.n_occ, tuple(Bd.shape)))
    diag = to_device(DIAG_A, torch.complex128, plan.device).reshape(-1)
    if diag.numel() != 3 * occ.n_occ:
        raise ValueError("DIAG_A must have %d entries" % (3 * occ.n_occ))
    X0d = None if X0 is None else to_device(X0, torch.complex128, plan.device).reshape(Bd.shape).contiguous()
    return dict(g=g, occ=occ, B=Bd, diag=diag, X0=X0d, X=torch.empty_like(Bd), numpy=to_numpy)


def _batch_struct(entries, mode):
    arr = (_BatchProblem * len(entries))()
    for i, e in enumerate(entries):
        g = e["g"]
        s = arr[i]
        s.plan = g.plan.handle.value
        s.n_occ = e["occ"].n_occ
        s.ghat = ptr(g.ghat(_lib.C128)) if mode != _lib.BATCH_C64 else None
        s.ghat_c64 = ptr(g.ghat(_lib.C64)) if mode != _lib.BATCH_C128 else None
        s.cell_map = ptr(e["occ"].cell_map)
        s.diag = ptr(e["diag"])
        s.B = ptr(e["B"])
        s.X0 = ptr(e["X0"])
        s.X = ptr(e["X"])
    return arr


# A batch shares one column-tile width and one shared-memory size per pencil
# pass, set by its longest axis; problems are grouped with others whose longest
# padded axis is within this ratio, so small lattices keep wide tiles.
_SIZE_RATIO = 1.6
# Lattices of at least this many padded grid points run the one-problem solver
# (specialised, autotuned kernels; their launch overhead is negligible there).
_BATCH_MAX_POINTS = 4 << 20


def _batch_groups(entries, mode, L, itermax, max_bytes):
    """Index groups of similar lattice size whose workspace fits max_bytes
    (at most 1024 problems each), largest lattices first."""
    lib = _lib.load()
    size = [max(e["g"].plan.m) for e in entries]
    order = sorted(range(len(entries)), key=lambda i: -size[i])
    groups, cur = [], []
    for i in order:
        trial = cur + [i]
        nbytes = int(lib.bdda_batch_workspace_bytes(_batch_struct([entries[j] for j in trial], mode), len(trial),
                                                    mode, L, itermax))
        if cur and (len(trial) > 1024 or nbytes > max_bytes or size[cur[0]] > _SIZE_RATIO * size[i]):
            groups.append(cur)
            cur = [i]
        else:
            cur = trial
    if cur:
        groups.append(cur)
    return groups


def bl_bicgstab_jacobi_mvp_fft_batch(problems, tol, itermax, precision=None, max_outer=20,
                                     graph=True, history=None, statuses=None, max_bytes=None):
    """Block-BiCGSTAB (bl_krylov.py:121-187) on many independent problems at once.

    ``problems``: a sequence of ``(n, address, Au_til, DIAG_A, B)`` or
    ``(n, address, Au_til, DIAG_A, B, X0)`` tuples (or dicts with those keys),
    each exactly the arguments of :func:`bl_bicgstab_jacobi_mvp_fft` for one
    particle / wavelength / orientation block; grids may differ, L (the
    columns of B) is shared and is 8, 16, 32 or 64.  Returns one
    ``(X, iter_fin, err_fin)`` per problem, with the meaning of the one-problem
    solver.  ``precision``: "c128" (default), "c64", or "mixed" (complex128
    Krylov vectors with complex64 products, judged on the complex128 true
    residual, at most ``max_outer`` warm-restarted rounds; problems it leaves
    above ``tol`` are solved again in complex128 from their start, with the
    iterations they have left, iter_fin counting both).
    ``graph``
    replays the batched iteration as a CUDA graph.  ``history`` (list)
    receives one residual list per problem, ``statuses`` (list) one status
    code per problem.  A problem whose small system is singular raises
    numpy.linalg.LinAlgError after the batch finished, unless ``statuses`` is
    given, in which case its X is None.  Problems are split into groups whose
    device workspace stays under ``max_bytes`` (default: 70 % of the free
    device memory); each group holds lattices of similar size (largest padded
    axis within 1.6x), so every group gets launch shapes that fit it.  Large
    lattices (>= 4 Mi padded grid points) and groups of one run the one-problem
    solver instead.
    """
    key = "c128" if precision is None else str(precision).lower()
    if key not in _BATCH_MODES:
        raise ValueError("precision must be one of %s" % sorted(_BATCH_MODES))
    mode = _BATCH_MODES[key]
    entries = [_batch_entry(p) for p in problems]
    if not entries:
        return []
    Ls = {int(e["B"].shape[1]) for e in entries}
    if len(Ls) != 1 or next(iter(Ls)) not in (8, 16, 32, 64):
        raise ValueError("all problems need the same L, one of 8, 16, 32, 64 (got %s)" % sorted(Ls))
    L = Ls.pop()
    itermax = int(itermax)
    dev = entries[0]["g"].plan.device
    fixed_bound = max_bytes is not None
    if not fixed_bound:
        torch.cuda.empty_cache()
        free, _ = torch.cuda.mem_get_info(dev)
        max_bytes = int(0.7 * free)
    lib = _lib.load()
    results = [None] * len(entries)
    hists = [None] * len(entries)
    big = [i for i, e in enumerate(entries) if int(np.prod(e["g"].plan.m)) >= _BATCH_MAX_POINTS]
    small = [i for i in range(len(entries)) if i not in set(big)]
    groups = [[small[j] for j in g] for g in _batch_groups([entries[i] for i in small], mode, L, itermax, max_bytes)]
    for g in [g for g in groups if len(g) == 1]:
        big.append(g[0])
    groups = [g for g in groups if len(g) > 1]
    one_prec = {_lib.BATCH_C128: None, _lib.BATCH_C64: "c64", _lib.BATCH_MIXED: "mixed"}[mode]
    for i in big:   # one problem at a time
        e = entries[i]
        h = [] if history is not None else None
        try:
            X, it_, er_ = _solve(_lib.BICGSTAB, e["g"].plan.n, 3, e["occ"], e["g"], e["diag"], e["B"], tol, itermax,
                                 X0=e["X0"], precision=one_prec, history=h, max_outer=max_outer)
            s_ = 0 if er_ < tol else 1
        except np.linalg.LinAlgError:
            X, it_, er_, s_ = None, 0, float("inf"), 2
        if X is not None and e["numpy"]:
            X = X.cpu().numpy()
        results[i] = (X, int(it_), float(er_), s_)
        hists[i] = h
    for idx in groups:
        grp = [entries[i] for i in idx]
        arr = _batch_struct(grp, mode)
        nb = int(lib.bdda_batch_workspace_bytes(arr, len(grp), mode, L, itermax))
        if nb == 0:
            raise ValueError("bdda_batch_workspace_bytes rejected the batch")
        work = torch.empty(nb, dtype=torch.uint8, device=dev)
        st = (C.c_int * len(grp))()
        it = (C.c_int * len(grp))()
        er = (C.c_double * len(grp))()
        hist = (C.c_double * (len(grp) * max(itermax, 1)))() if history is not None else None
        rc = lib.bdda_batch_bicgstab(arr, len(grp), mode, L, float(tol), itermax, int(max_outer),
                                     1 if graph else 0, st, it, er, hist, ptr(work), nb, stream_ptr(dev))
        if rc not in (0, 1, 2):
            _lib.check(rc, "bdda_batch_bicgstab")
        del work
        torch.cuda.empty_cache()
        for i, e in enumerate(grp):
            s = int(st[i])
            X = None if s == 2 else (e["X"].cpu().numpy() if e["numpy"] else e["X"])
            results[idx[i]] = (X, int(it[i]), float(er[i]), s)
            if history is not None:
                ran = 0 if itermax == 0 or s == 2 else int(it[i]) + 1
                hists[idx[i]] = [hist[i * itermax + k] for k in range(min(ran, itermax))]
    hbase = 0
    if history is not None:
        hbase = len(history)
        history.extend(hists)
    if mode == _lib.BATCH_MIXED:
        # problems the mixed form leaves above tol (its recursion diverged under the
        # complex64 products) are solved again with complex128 products
        # with the iterations the batch left them (iter_fin counts both), so no
        # problem takes more than itermax iterations in all
        redo = [i for i, r in enumerate(results) if r[3] == 1 and not r[2] < tol and itermax - 1 - r[1] > 0]
        for left in sorted({itermax - 1 - results[i][1] for i in redo}):
            sub = [i for i in redo if itermax - 1 - results[i][1] == left]
            sub_hist = [] if history is not None else None
            sub_st = []
            again = bl_bicgstab_jacobi_mvp_fft_batch([problems[i] for i in sub], tol, left, "c128",
                                                     max_outer, graph, sub_hist, sub_st,
                                                     max_bytes if fixed_bound else None)
            for j, i in enumerate(sub):
                X, it, er = again[j]
                results[i] = (X, results[i][1] + 1 + it, er, sub_st[j])
                if history is not None:
                    history[hbase + i] = history[hbase + i] + sub_hist[j]
    if statuses is not None:
        statuses.extend(r[3] for r in results)
    elif any(r[3] == 2 for r in results):
        bad = [i for i, r in enumerate(results) if r[3] == 2]
        raise np.linalg.LinAlgError("Singular matrix in batched problems %s" % bad)
    return [r[:3] for r in results]
