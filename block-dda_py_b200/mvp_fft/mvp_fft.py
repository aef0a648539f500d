"""GPU drop-in for the reference module ``mvp_fft.mvp_fft``.

Same names and signatures as mvp_fft/mvp_fft.py (block-DDA_Py v0.3.0):
``build_interaction_tensor(n, lf, k)``, ``fft_init(n, f, lf, k)``,
``fft_mvp(n, f, A_tensor_tilde, P_block)`` and ``_FFT_WORKERS``.  The work
runs in libbdda.so on the current CUDA device; NumPy inputs give NumPy
outputs, torch tensors give device tensors.
"""
from __future__ import annotations

import os

import numpy as np
import torch

from bdda_b200 import _lib
from bdda_b200.runtime import (TORCH_DTYPE, GreenTensor, Plan, precision_code, ptr,
                               stream_ptr, to_device)

# Kept for interface parity with mvp_fft.py:9-10; the GPU path does not use it.
_FFT_WORKERS = int(os.environ.get("DDA_FFT_WORKERS", max(1, (os.cpu_count() or 1) - 2)))


def build_interaction_tensor(n, lf, k):
    """A'(r) on the doubled grid, (2Nx, 2Ny, 2Nz, 3, 3) complex128 (mvp_fft.py:13-94).

    Evaluated on the device; returned as a NumPy array like the reference.
    """
    plan = Plan(n, m=[2 * int(v) for v in np.asarray(n).ravel()])
    out = torch.empty(plan.m + (3, 3), dtype=torch.complex128, device=plan.device)
    _lib.check(_lib.load().bdda_green_real(plan.handle, float(lf), float(k), ptr(out),
                                           stream_ptr(plan.device)), "bdda_green_real")
    return out.cpu().numpy()


def fft_init(n, f, lf, k, m=None):
    """Spectrum of the interaction tensor, resident on the GPU (mvp_fft.py:97-119).

    Returns a :class:`bdda_b200.runtime.GreenTensor`; ``np.asarray`` of it is
    the reference's (2Nx, 2Ny, 2Nz, 3, 3) array.  ``m`` optionally fixes the
    cyclic grid (any m >= 2n-1 gives the same product).
    Raises ValueError for f != 3, like the reference (mvp_fft.py:116-117).
    """
    if f != 3:
        raise ValueError("fft_init: only f=3 (electric dipoles) is supported.")
    return GreenTensor(Plan(n, m=m), lf, k)


def as_green(n, A_tensor_tilde) -> GreenTensor:
    if isinstance(A_tensor_tilde, GreenTensor):
        g = A_tensor_tilde
        if tuple(int(v) for v in np.asarray(n).ravel()) != g.plan.n:
            raise ValueError("lattice n %r does not match the Green's tensor grid %r"
                             % (tuple(np.asarray(n).ravel()), g.plan.n))
        return g
    return GreenTensor.from_full(n, A_tensor_tilde)


def fft_mvp(n, f, A_tensor_tilde, P_block, precision=None):
    """Off-diagonal product A_off @ P_block via the doubled-grid FFT (mvp_fft.py:122-173).

    ``P_block`` is (f*Nx*Ny*Nz,) or (f*Nx*Ny*Nz, L) on the full cuboid; the
    result has the same shape.  ``precision`` (default complex128, the
    reference's arithmetic) may be "c64" for the FP32 product.
    """
    if f != 3:
        raise ValueError("fft_mvp: only f=3 (electric dipoles) is supported.")
    g = as_green(n, A_tensor_tilde)
    plan = g.plan
    prec = precision_code(precision)
    to_numpy = not isinstance(P_block, torch.Tensor)
    P = to_device(P_block, TORCH_DTYPE[prec], plan.device)
    squeeze = P.dim() == 1
    if squeeze:
        P = P[:, None]
    if P.dim() != 2 or P.shape[0] != 3 * plan.n_cells:
        raise ValueError("P_block must have %d rows, got shape %r" % (3 * plan.n_cells, tuple(P.shape)))
    P = P.contiguous()
    L = int(P.shape[1])
    out = torch.empty_like(P)
    work = g.workspace(prec, L)
    _lib.check(_lib.load().bdda_fft_mvp(plan.handle, prec, L, ptr(g.ghat(prec)), ptr(P), ptr(out),
                                        ptr(work), stream_ptr(plan.device)), "bdda_fft_mvp")
    res = out[:, 0] if squeeze else out
    return res.cpu().numpy() if to_numpy else res
