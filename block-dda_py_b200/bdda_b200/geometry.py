"""GRE lattice occupancy on the GPU (bdda_gre_occupancy).

The reference decides which lattice cells a Gaussian random ellipsoid
occupies with a k-d tree query of every cell against the surface points and
three cumulative sums along the axes (shape_model/gaussian_ellipsoid.py:
182-237).  Here the host sorts the surface points into uniform bins (a few
thousand to a few hundred thousand points: an argsort) and one sm_100a kernel
tests every cell against the points of its 27 neighbouring bins, then the
first / last near cell of every axis line gives the inside test.  The mask is
the reference's bit for bit (tests/test_geometry_gpu.py).
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib
from .runtime import ptr, require_cuda, stream_ptr


def _bins(surf: np.ndarray, thr: float):
    h = max(float(thr) * 1.01, 1e-300)   # bin edge >= threshold, with slack for rounding
    origin = surf.min(axis=0) - h
    nb = (np.floor((surf.max(axis=0) - origin) / h).astype(np.int64) + 2)
    b = np.floor((surf - origin) / h).astype(np.int64)
    b = np.clip(b, 0, nb - 1)
    flat = (b[:, 0] * nb[1] + b[:, 1]) * nb[2] + b[:, 2]
    order = np.argsort(flat, kind="stable")
    start = np.searchsorted(flat[order], np.arange(int(np.prod(nb)) + 1)).astype(np.int32)
    return np.ascontiguousarray(surf[order]), start, nb, origin, h


def occupancy(axes, surf: np.ndarray, thr: float, device=None):
    """(near, inside) boolean (Nx, Ny, Nz) masks of the lattice with the given axis arrays."""
    dev = device or require_cuda()
    lib = _lib.load()
    n = [len(a) for a in axes]
    surf = np.asarray(surf, dtype=np.float64).reshape(-1, 3)
    pts, start, nb, origin, h = _bins(surf, thr)
    if int(np.prod(nb)) >= 2 ** 31 - 1 or pts.shape[0] >= 2 ** 31 - 1:
        raise ValueError("surface bin grid too large")
    t = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a)).to(device=dev, dtype=dt)   # noqa: E731
    xs, ys, zs = (t(a, torch.float64) for a in axes)
    dpts = t(pts, torch.float64)
    dstart = t(start, torch.int32)
    nc = int(np.prod(n))
    near = torch.empty(nc, dtype=torch.uint8, device=dev)
    inside = torch.empty(nc, dtype=torch.uint8, device=dev)
    wb = int(lib.bdda_gre_occupancy_workspace_bytes(*n))
    work = torch.empty(max(wb, 16), dtype=torch.uint8, device=dev)
    _lib.check(lib.bdda_gre_occupancy(n[0], n[1], n[2], ptr(xs), ptr(ys), ptr(zs), pts.shape[0], ptr(dpts),
                                      ptr(dstart), int(nb[0]), int(nb[1]), int(nb[2]), float(origin[0]),
                                      float(origin[1]), float(origin[2]), float(h), float(thr), ptr(near),
                                      ptr(inside), ptr(work), wb, stream_ptr(dev)), "bdda_gre_occupancy")
    shape = tuple(n)
    return (near.cpu().numpy().astype(bool).reshape(shape), inside.cpu().numpy().astype(bool).reshape(shape))


def near_surface(axes, surf: np.ndarray, thr: float) -> np.ndarray:
    """Near-surface mask on the GPU: cells closer than ``thr`` to a surface point."""
    return occupancy(axes, surf, thr)[0]


def inside_from_gpu(axes, surf: np.ndarray, thr: float) -> np.ndarray:
    """Inside mask on the GPU (the ``mask_fn`` hook of :func:`bdda_b200.shapes.gre_geometry`)."""
    return occupancy(axes, surf, thr)[1]
