"""GPU drop-in for the reference module ``bl_krylov.bl_krylov``.

Same names and signatures as bl_krylov/bl_krylov.py (block-DDA_Py v0.3.0):
``_build_scatter_index``, ``_block_mvp``, ``bl_cocg_rq_jacobi_mvp_fft`` and
``bl_bicgstab_jacobi_mvp_fft``.  The products, the block Gram reductions, the
small L x L solves and the block updates all run in libbdda.so.
"""
from __future__ import annotations

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
