"""Device-side objects behind the drop-in API: plans, Green's spectra, buffers.

PyTorch is used only for device memory and streams: every buffer here is a
torch tensor from the caching allocator, passed to libbdda.so as a raw
pointer together with the current CUDA stream.  All arithmetic runs in the
library's sm_100a kernels.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib

PREC = {"c128": _lib.C128, "fp64": _lib.C128, "complex128": _lib.C128,
        "c64": _lib.C64, "fp32": _lib.C64, "complex64": _lib.C64}
TORCH_DTYPE = {_lib.C128: torch.complex128, _lib.C64: torch.complex64}


def require_cuda() -> torch.device:
    """The product path runs on the GPU only; there is no CPU fallback."""
    if not torch.cuda.is_available():
        raise RuntimeError("bdda_b200 needs a CUDA device (sm_100a); none is visible")
    return torch.device("cuda", torch.cuda.current_device())


def precision_code(precision) -> int:
    if precision is None:
        return _lib.C128
    if isinstance(precision, int) and precision in (_lib.C128, _lib.C64):
        return precision
    try:
        return PREC[str(precision).lower()]
    except KeyError:
        raise ValueError("precision must be one of %s" % sorted(PREC)) from None


def stream_ptr(device=None) -> int:
    return torch.cuda.current_stream(device).cuda_stream


def ptr(t: torch.Tensor | None) -> int | None:
    return None if t is None else t.data_ptr()


def to_device(x, dtype: torch.dtype, device: torch.device) -> torch.Tensor:
    """numpy / torch / sequence -> contiguous tensor of ``dtype`` on ``device``."""
    if isinstance(x, torch.Tensor):
        t = x.to(device=device, dtype=dtype)
    else:
        t = torch.from_numpy(np.ascontiguousarray(np.asarray(x))).to(device=device, dtype=dtype)
    return t.contiguous()


def empty_bytes(nbytes: int, device: torch.device) -> torch.Tensor:
    return torch.empty(max(int(nbytes), 16), dtype=torch.uint8, device=device)


class Plan:
    """Cuboid geometry, padded FFT grid and the device twiddle tables.

    ``m`` (optional) fixes the cyclic FFT grid; by default each axis uses the
    smallest even 7-smooth length >= 2N, which is the reference's doubled grid
    2N whenever 2N is 7-smooth.
    """

    def __init__(self, n, m=None):
        self.device = require_cuda()
        lib = _lib.load()
        n = [int(v) for v in np.asarray(n).ravel()]
        if len(n) != 3 or min(n) < 1:
            raise ValueError("lattice_n must hold three positive sizes, got %r" % (n,))
        h = C.c_void_p()
        _lib.check(lib.bdda_plan_create(_lib.int3(n), None if m is None else _lib.int3(m),
                                        C.byref(h)), "bdda_plan_create")
        self._h = h
        self.n = tuple(n)
        mm = (C.c_int * 3)()
        lib.bdda_plan_grid(h, mm)
        self.m = tuple(int(v) for v in mm)
        self.tables = empty_bytes(lib.bdda_plan_table_bytes(h), self.device)
        _lib.check(lib.bdda_plan_attach_tables(h, ptr(self.tables), stream_ptr(self.device)),
                   "bdda_plan_attach_tables")

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    @property
    def n_cells(self) -> int:
        return self.n[0] * self.n[1] * self.n[2]

    def radices(self, axis: int) -> list[int]:
        r = (C.c_int * 12)()
        ns = C.c_int()
        _lib.check(_lib.load().bdda_plan_radices(self._h, axis, r, C.byref(ns)), "bdda_plan_radices")
        return [int(r[i]) for i in range(ns.value)]

    def mvp_workspace_bytes(self, prec: int, L: int) -> int:
        return int(_lib.load().bdda_mvp_workspace_bytes(self._h, prec, int(L)))

    def wait_timeouts(self) -> int:
        """Bounded waits of this plan's pass kernels that ran out (0 in a correct run)."""
        c = C.c_uint()
        _lib.check(_lib.load().bdda_plan_wait_timeouts(self._h, C.byref(c), stream_ptr(self.device)),
                   "bdda_plan_wait_timeouts")
        return int(c.value)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and _lib._lib is not None:
            _lib._lib.bdda_plan_destroy(h)
            self._h = None


class GreenTensor:
    """Spectrum of the interaction tensor A'(r), resident in HBM.

    This is what ``fft_init`` returns.  The six unique components are stored
    in the library's order (x-pencil major, digit-reversed spectra);
    ``np.asarray(g)`` / :meth:`full` give the reference's
    (2Nx, 2Ny, 2Nz, 3, 3) complex128 layout (mvp_fft/mvp_fft.py:111-112)
    when the plan's grid is the doubled grid.
    """

    def __init__(self, plan: Plan, lf: float, k: float, ghat: torch.Tensor | None = None):
        self.plan = plan
        self.lf = float(lf)
        self.k = float(k)
        lib = _lib.load()
        npts = plan.m[0] * plan.m[1] * plan.m[2]
        if ghat is None:
            ghat = torch.empty(npts * 6, dtype=torch.complex128, device=plan.device)
            work = empty_bytes(lib.bdda_green_build_workspace_bytes(plan.handle), plan.device)
            _lib.check(lib.bdda_green_build(plan.handle, self.lf, self.k, ptr(ghat), ptr(work),
                                            stream_ptr(plan.device)), "bdda_green_build")
            del work
        self._g = {_lib.C128: ghat}
        self._work = {}

    @classmethod
    def from_full(cls, n, full) -> "GreenTensor":
        """Adopt a spectrum given in the reference layout (2Nx, 2Ny, 2Nz, 3, 3)."""
        n = [int(v) for v in np.asarray(n).ravel()]
        arr = full if isinstance(full, torch.Tensor) else np.asarray(full)
        shape = tuple(arr.shape)
        if shape[3:] != (3, 3) or len(shape) != 5:
            raise ValueError("A_tensor_tilde must have shape (Mx, My, Mz, 3, 3), got %r" % (shape,))
        plan = Plan(n, m=shape[:3])
        src = to_device(arr, torch.complex128, plan.device)
        ghat = torch.empty(shape[0] * shape[1] * shape[2] * 6, dtype=torch.complex128,
                           device=plan.device)
        _lib.check(_lib.load().bdda_green_import(plan.handle, ptr(src), ptr(ghat),
                                                 stream_ptr(plan.device)), "bdda_green_import")
        return cls(plan, float("nan"), float("nan"), ghat=ghat)

    def ghat(self, prec: int) -> torch.Tensor:
        if prec not in self._g:
            g64 = torch.empty(self._g[_lib.C128].numel(), dtype=torch.complex64, device=self.plan.device)
            _lib.check(_lib.load().bdda_green_convert(self.plan.handle, ptr(self._g[_lib.C128]),
                                                      ptr(g64), stream_ptr(self.plan.device)),
                       "bdda_green_convert")
            self._g[prec] = g64
        return self._g[prec]

    def workspace(self, prec: int, L: int) -> torch.Tensor:
        """Field buffer for one product at L right-hand sides (grown, then reused)."""
        need = self.plan.mvp_workspace_bytes(prec, L)
        buf = self._work.get(prec)
        if buf is None or buf.numel() < need:
            buf = empty_bytes(need, self.plan.device)
            self._work[prec] = buf
        return buf

    def release_workspace(self) -> None:
        self._work.clear()

    def full(self) -> torch.Tensor:
        """(Mx, My, Mz, 3, 3) complex128 on the device, natural frequency order."""
        mx, my, mz = self.plan.m
        out = torch.empty((mx, my, mz, 3, 3), dtype=torch.complex128, device=self.plan.device)
        _lib.check(_lib.load().bdda_green_export(self.plan.handle, ptr(self._g[_lib.C128]), ptr(out),
                                                 stream_ptr(self.plan.device)), "bdda_green_export")
        return out

    @property
    def shape(self):
        return tuple(self.plan.m) + (3, 3)

    def __array__(self, dtype=None, copy=None):
        a = self.full().cpu().numpy()
        return a if dtype is None else a.astype(dtype)


class Occupancy:
    """Occupied-cell list of a cuboid and its device cell -> dipole map."""

    def __init__(self, plan: Plan, address):
        address = np.asarray(address.cpu() if isinstance(address, torch.Tensor) else address)
        address = address.astype(np.int64).ravel()
        if address.size and (address.min() < 0 or address.max() >= plan.n_cells):
            raise ValueError("address out of range for lattice %r" % (plan.n,))
        if address.size > 1 and np.any(np.diff(np.sort(address)) == 0):
            raise ValueError("address holds duplicate cells")
        self.plan = plan
        self.n_occ = int(address.size)
        self.address = address
        self.address_dev = to_device(address, torch.int64, plan.device)
        self.cell_map = torch.empty(plan.n_cells, dtype=torch.int32, device=plan.device)
        _lib.check(_lib.load().bdda_occupancy_map(plan.handle, ptr(self.address_dev), self.n_occ,
                                                  ptr(self.cell_map), stream_ptr(plan.device)),
                   "bdda_occupancy_map")


def autotune(green: GreenTensor, occupancy: Occupancy, L: int, precision="c128", reps: int = 3,
             seed: int = 0) -> tuple[float, float]:
    """Pick each pencil pass's tile width and kernel variant for this grid and L.

    Runs block MVPs on random input (libbdda's ``bdda_autotune``), keeps the
    fastest launch choice per pass, and returns the product's time in ms
    before and after.  The choice is process-wide and applies to every later
    product with the same axis lengths, precision and L.
    """
    prec = precision_code(precision)
    plan = green.plan
    dev = plan.device
    dt = TORCH_DTYPE[prec]
    n3 = 3 * occupancy.n_occ
    g = torch.Generator(device=dev).manual_seed(int(seed))
    S = torch.randn((n3, int(L)), dtype=dt, device=dev, generator=g)
    diag = torch.ones(n3, dtype=dt, device=dev)
    out = torch.empty_like(S)
    before, after = C.c_double(), C.c_double()
    _lib.check(_lib.load().bdda_autotune(plan.handle, prec, int(L), ptr(green.ghat(prec)), ptr(occupancy.cell_map),
                                         ptr(diag), ptr(diag), ptr(S), ptr(out), ptr(green.workspace(prec, L)),
                                         int(reps), C.byref(before), C.byref(after), stream_ptr(dev)),
               "bdda_autotune")
    return before.value, after.value
