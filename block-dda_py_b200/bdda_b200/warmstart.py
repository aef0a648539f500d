"""Learned warm start for the block solvers (Fourier neural operator).

The network and its training run in libbdda's hand-written kernels
(bdda_fno_*): features from the occupancy map, the per-axis relative
permittivity and the Jacobi guess J = B / DIAG_A; forward, backward and Adam
on the GPU; the warm start X0 = J + scale * FNO(...).  The solve still runs to
the same residual and judges it; a column whose predicted initial residual
||M^-1 (B - A X0)|| exceeds ||M^-1 B|| starts from zero instead.

    model = WarmStartFNO(layers=4, modes=12, seed=4)
    data = make_dataset(...)              # solutions the solver itself generates
    model.fit(data, epochs=...)
    X0, n_fallback = model.warm_start(n, occupancy, green, diag, B, eps_r)
"""
from __future__ import annotations

import ctypes as C
import time

import numpy as np
import torch

from . import _lib
from .runtime import Occupancy, ptr, require_cuda, stream_ptr, to_device


class FnoConfig(C.Structure):
    """include/bdda.h: bdda_fno_config."""
    _fields_ = [("cin", C.c_int), ("width", C.c_int), ("cout", C.c_int), ("proj", C.c_int), ("layers", C.c_int),
                ("modes", C.c_int)]


def _n3(n):
    return (C.c_int * 3)(*[int(v) for v in n])


def chi_of(eps_r) -> np.ndarray:
    """(Re, Im) of (eps - 1) / (eps + 2) per axis, 6 doubles."""
    e = np.asarray(eps_r, dtype=np.complex128).ravel()
    if e.size == 1:
        e = np.repeat(e, 3)
    c = (e - 1.0) / (e + 2.0)
    return np.column_stack([c.real, c.imag]).ravel()


class WarmStartFNO:
    """FNO parameters (one FP32 device array), Adam state and per-shape workspaces."""

    def __init__(self, layers: int = 4, modes: int = 12, seed: int = 0, device=None):
        self.device = device or require_cuda()
        self.cfg = FnoConfig(13, 32, 6, 64, int(layers), int(modes))
        lib = _lib.load()
        self.n_params = int(lib.bdda_fno_param_count(C.byref(self.cfg)))
        if self.n_params == 0:
            raise ValueError("bad FNO configuration")
        self.params = torch.zeros(self.n_params, dtype=torch.float32, device=self.device)
        self._init(seed)
        self.grads = torch.zeros_like(self.params)
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.step = 0
        self._work = {}

    # ---- parameters ----
    def _slice(self, what, layer, size):
        off = int(_lib.load().bdda_fno_offset(C.byref(self.cfg), what, layer))
        return self.params[off:off + size]

    def _init(self, seed):
        g = torch.Generator(device="cpu").manual_seed(int(seed))
        c = self.cfg
        K = c.modes ** 3

        def put(what, layer, shape, std):
            n = int(np.prod(shape))
            self._slice(what, layer, n).copy_((torch.randn(n, generator=g) * std).to(self.device))
        put(0, 0, (c.cin, c.width), 1.0 / np.sqrt(c.cin))
        for l in range(c.layers):
            put(2, l, (K, c.width, c.width, 2), 1.0 / (c.width * np.sqrt(2.0)))
            put(3, l, (c.width, c.width), 1.0 / np.sqrt(c.width))
        put(5, 0, (c.width, c.proj), 1.0 / np.sqrt(c.width))
        put(7, 0, (c.proj, c.cout), 0.1 / np.sqrt(c.proj))   # starts near X0 = J

    def save(self, path):
        c = self.cfg
        np.savez_compressed(path, params=self.params.cpu().numpy(), layers=c.layers, modes=c.modes)

    @classmethod
    def load(cls, path, device=None):
        with np.load(path) as z:
            m = cls(int(z["layers"]), int(z["modes"]), device=device)
            m.params.copy_(torch.from_numpy(z["params"]).to(m.device))
        return m

    # ---- workspaces ----
    def _workspace(self, L, n):
        key = (int(L),) + tuple(int(v) for v in n)
        w = self._work.get(key)
        if w is None:
            nb = int(_lib.load().bdda_fno_workspace_bytes(C.byref(self.cfg), int(L), _n3(n)))
            if nb == 0:
                raise ValueError("bad FNO shape %r" % (key,))
            if len(self._work) > 1:
                self._work.clear()
                torch.cuda.empty_cache()
            w = torch.empty(nb, dtype=torch.uint8, device=self.device)
            self._work[key] = w
        return w

    def supports(self, n) -> bool:
        return all(self.cfg.modes <= int(v) <= 512 for v in n)

    def buffer(self, work, L, n, which, count, dtype=torch.float32):
        off = int(_lib.load().bdda_fno_buffer_offset(C.byref(self.cfg), int(L), _n3(n), which))
        es = torch.tensor([], dtype=dtype).element_size()
        return work[off:off + count * es].view(dtype)

    # ---- the network on one particle ----
    def features(self, n, occ: Occupancy, diag, B, eps_r):
        L = int(B.shape[1])
        work = self._workspace(L, n)
        scale = torch.empty(L, dtype=torch.float64, device=self.device)
        chi = (C.c_double * 6)(*chi_of(eps_r))
        _lib.check(_lib.load().bdda_fno_features(C.byref(self.cfg), _n3(n), occ.n_occ, L, ptr(occ.cell_map),
                                                 ptr(diag), ptr(B), chi, ptr(scale), ptr(work), work.numel(),
                                                 stream_ptr(self.device)), "bdda_fno_features")
        return work, scale

    def forward(self, work, L, n, train=False):
        _lib.check(_lib.load().bdda_fno_forward(C.byref(self.cfg), int(L), _n3(n), ptr(self.params),
                                                1 if train else 0, ptr(work), work.numel(),
                                                stream_ptr(self.device)), "bdda_fno_forward")

    # samples (orientations) per call: activations of at most max_rows lattice
    # rows (~3 KB of workspace per row); inference takes larger calls, since
    # its launches are few per call and the solve has not allocated yet
    max_rows = 4_000_000
    max_rows_infer = 16_000_000

    def _chunks(self, n, L, rows=None):
        rows = self.max_rows if rows is None else rows
        per = max(1, min(L, rows // int(np.prod([int(v) for v in n]))))
        return [(c, min(L, c + per)) for c in range(0, L, per)]

    def predict(self, n, occ, diag, B, eps_r) -> torch.Tensor:
        """X0 = J + scale * FNO, complex128 (3 n_occ, L)."""
        L = int(B.shape[1])
        X0 = torch.empty_like(B)
        for c0, c1 in self._chunks(n, L, self.max_rows_infer):
            Bc = B[:, c0:c1].contiguous()
            work, scale = self.features(n, occ, diag, Bc, eps_r)
            self.forward(work, c1 - c0, n)
            Xc = torch.empty_like(Bc)
            _lib.check(_lib.load().bdda_fno_warm_start(C.byref(self.cfg), _n3(n), occ.n_occ, c1 - c0,
                                                       ptr(occ.cell_map), ptr(diag), ptr(Bc), ptr(scale), ptr(Xc),
                                                       ptr(work), work.numel(), stream_ptr(self.device)),
                       "bdda_fno_warm_start")
            X0[:, c0:c1] = Xc
        return X0

    def loss_and_grad(self, n, occ, diag, B, eps_r, X) -> float:
        """Forward, loss against the solution X and backward over the orientations of
        one particle, in chunks of orientations whose losses (each a mean over the
        chunk) add; the summed gradient is in self.grads."""
        lib = _lib.load()
        L = int(B.shape[1])
        self.grads.zero_()
        total = 0.0
        for c0, c1 in self._chunks(n, L):
            Bc = B[:, c0:c1].contiguous() if (c0, c1) != (0, L) else B
            Xc = X[:, c0:c1].contiguous() if (c0, c1) != (0, L) else X
            b = c1 - c0
            work, scale = self.features(n, occ, diag, Bc, eps_r)
            self.forward(work, b, n, train=True)
            loss = C.c_double(0.0)
            _lib.check(lib.bdda_fno_loss(C.byref(self.cfg), b, _n3(n), occ.n_occ, ptr(occ.cell_map), ptr(diag),
                                         ptr(Bc), ptr(Xc), ptr(scale), C.byref(loss), ptr(work), work.numel(),
                                         stream_ptr(self.device)), "bdda_fno_loss")
            _lib.check(lib.bdda_fno_backward(C.byref(self.cfg), b, _n3(n), ptr(self.params), None, ptr(self.grads),
                                             ptr(work), work.numel(), stream_ptr(self.device)), "bdda_fno_backward")
            torch.cuda.current_stream(self.device).synchronize()
            total += float(loss.value) * b / L
        return total

    def adam(self, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8, weight_decay=0.0):
        self.step += 1
        _lib.check(_lib.load().bdda_fno_adam(ptr(self.params), ptr(self.grads), ptr(self.m), ptr(self.v),
                                             self.n_params, lr, beta1, beta2, eps, weight_decay, self.step,
                                             stream_ptr(self.device)), "bdda_fno_adam")

    def fit(self, data, epochs=10, lr=1e-3, lr_final=1e-4, seed=0, log=None) -> list:
        """Adam over the samples (one particle, all its orientations, per step); cosine-decayed rate."""
        rng = np.random.default_rng(seed)
        steps = max(1, epochs * len(data))
        losses = []
        k = 0
        for ep in range(epochs):
            order = rng.permutation(len(data))
            tot = 0.0
            for i in order:
                d = data[i]
                rate = lr_final + 0.5 * (lr - lr_final) * (1 + np.cos(np.pi * k / steps))
                tot += self.loss_and_grad(d["n"], d["occ"], d["diag"], d["B"], d["eps_r"], d["X"])
                self.adam(lr=float(rate))
                k += 1
            losses.append(tot / len(data))
            if log:
                log("epoch %d loss %.4f" % (ep, losses[-1]))
        return losses

    # ---- warm start with the fallback rule ----
    def warm_start(self, n, occ, green, diag, B, eps_r, mode="fallback"):
        """(X0 or None, columns that fell back).

        mode "fallback": a column whose predicted initial residual
        ||M^-1 (B - A X0)|| exceeds ||M^-1 B|| starts from zero.  mode
        "project": X0 = P G with P the L predicted columns and G (L x L) the
        least-squares fit min ||M^-1 B - (M^-1 A P) G||_F, from the same one
        product; its residual is at most the zero start's (G = 0 is a
        candidate), so no column falls back.  Either way the solver still
        runs to its tolerance and judges the result.
        """
        L = int(B.shape[1])
        if not self.supports(n):
            return None, L
        X0 = self.predict(n, occ, diag, B, eps_r)
        lib = _lib.load()
        jpre = 1.0 / diag
        AX = torch.empty_like(X0)
        work = green.workspace(_lib.C128, L)
        _lib.check(lib.bdda_block_mvp(green.plan.handle, _lib.C128, L, ptr(green.ghat(_lib.C128)), ptr(occ.cell_map),
                                      ptr(diag), ptr(jpre), ptr(X0), ptr(AX), ptr(work),
                                      stream_ptr(self.device)), "bdda_block_mvp")
        Bj = B * jpre[:, None]
        if mode == "project":
            G = AX.conj().T @ AX                      # L x L normal equations (complex128)
            rhs = AX.conj().T @ Bj
            ridge = 1e-12 * torch.diagonal(G).real.mean().clamp_min(1e-300)
            coef = torch.linalg.solve(G + ridge * torch.eye(L, dtype=G.dtype, device=G.device), rhs)
            return X0 @ coef, 0
        r = torch.linalg.vector_norm(Bj - AX, dim=0)
        b = torch.linalg.vector_norm(Bj, dim=0)
        bad = ~(r <= b)
        nb = int(bad.sum().item())
        if nb == L:
            return None, L
        if nb:
            X0[:, bad] = 0
        return X0, nb


# ---------------------------------------------------------------------------
# training data: GRE particles solved by the batched solver
# ---------------------------------------------------------------------------
def sample_particles(count, seed, x_range=(4.0, 12.0), ratio_range=(0.5, 1.0), beta_range=(0.0, 0.2),
                     re_range=(1.3, 1.7), im_range=(0.0, 0.1), biref=0.05):
    """Shape and material parameters (config of the learned warm start)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        re = rng.uniform(*re_range)
        im = rng.uniform(*im_range)
        d = rng.uniform(-biref, biref, 3)
        out.append(dict(x=float(rng.uniform(*x_range)), ab=float(rng.uniform(*ratio_range)),
                        bc=float(rng.uniform(*ratio_range)), beta=float(rng.uniform(*beta_range)),
                        seed=int(seed * 100000 + i), m_p=[complex(re + d[a], im) for a in range(3)],
                        euler_seed=int(seed * 100000 + 50000 + i)))
    return out


def _shape(spec):
    from .shapes import gre_particle
    g = gre_particle(spec["x"], spec["ab"], spec["bc"], spec["beta"], spec["seed"], coarse=(13, 50), workers=1)
    return {k: g[k] for k in ("lattice_n", "lattice_lf", "is_in", "grid")}


def make_dataset(specs, L=16, tol=1e-5, itermax=600, shapes=None, max_cells=128, log=None):
    """Solve every particle (complex128 batched block-BiCGSTAB, tol) and keep
    what training needs.  ``shapes``: precomputed lattices (from ``_shape``)."""
    from bl_dda import scatterer as sc
    from .inputs import so3_euler
    sc.DiscreteDipoles.verbose = False
    t0 = time.time()
    if shapes is None:
        shapes = [_shape(s) for s in specs]
    dds, keep = [], []
    for spec, g in zip(specs, shapes):
        if max(g["lattice_n"]) > max_cells or min(g["lattice_n"]) < 12 or not g["is_in"].any():
            continue
        t = sc.Target("gre", g["lattice_n"], g["lattice_lf"], g["grid"], g["is_in"], spec["m_p"])
        d = sc.DiscreteDipoles(t, sc.IncidentField(1.0, 1.0, so3_euler(L, spec["euler_seed"])))
        d.tol, d.itermax = tol, itermax
        d.set_interaction_matrix()
        dds.append(d)
        keep.append(spec)
    sc.solve_matrix_equations(dds, precision="c128")
    torch.cuda.empty_cache()
    data = []
    for spec, d in zip(keep, dds):
        eps = (np.asarray(spec["m_p"]) / 1.0) ** 2
        data.append(dict(n=tuple(int(v) for v in d.lattice_n), occ=d._dev["occ"], diag=d._dev["diag"],
                         B=d._dev["B"], X=d._dev["X"], eps_r=eps, green=d.Au_til, iters=d.iter_fin + 1,
                         converged=d.converge, spec=spec))
    if log:
        log("dataset: %d particles in %.1f s" % (len(data), time.time() - t0))
    return data
