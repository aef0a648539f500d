"""CPU oracle of the learned warm start -- TEST INFRASTRUCTURE ONLY.

A float64 restatement, on torch's CPU autograd, of the Fourier neural operator
that libbdda's hand-written kernels run (bdda_fno.cu): the same features,
layers, truncated DFTs (explicit DFT matrices over the kept frequencies
0..modes/2-1 and N-modes/2..N-1 per axis), GELU (erf form), loss and
parameter layout.  The warm start has no counterpart in the reference, so
the oracle pins the GPU network's outputs and gradients, not a reference
result ("parity unpinned" against the reference: it is checked against its
own mathematics and against finite differences).

Only ``tests/`` import it; the CUDA product path never routes through here.
"""
from __future__ import annotations

import numpy as np
import torch

CIN, WIDTH, COUT, PROJ = 13, 32, 6, 64


def param_layout(layers: int, modes: int, cin=CIN, width=WIDTH, cout=COUT, proj=PROJ):
    """(name, shape) of the flat FP32 parameter array, in order (bdda_fno.cu param_layout)."""
    K = modes ** 3
    out = [("P", (cin, width)), ("p", (width,))]
    for l in range(layers):
        out += [("R%d" % l, (K, width, width, 2)), ("W%d" % l, (width, width)), ("b%d" % l, (width,))]
    out += [("Q1", (width, proj)), ("q1", (proj,)), ("Q2", (proj, cout)), ("q2", (cout,))]
    return out


def unflatten(flat: np.ndarray, layers: int, modes: int) -> dict:
    params, off = {}, 0
    for name, shape in param_layout(layers, modes):
        n = int(np.prod(shape))
        params[name] = torch.tensor(np.asarray(flat[off:off + n], dtype=np.float64).reshape(shape),
                                    requires_grad=True)
        off += n
    return params


def flatten_grads(params: dict, layers: int, modes: int) -> np.ndarray:
    return np.concatenate([params[name].grad.detach().numpy().ravel() for name, _ in param_layout(layers, modes)])


def dft_matrix(N: int, modes: int) -> torch.Tensor:
    """F[n, j] = exp(-2 pi i f_j n / N), f_j = j for j < modes/2 else N - (modes - j)."""
    h = modes // 2
    f = np.array([j if j < h else N - (modes - j) for j in range(modes)])
    n = np.arange(N)
    return torch.tensor(np.exp(-2j * np.pi * np.outer(n, f) / N), dtype=torch.complex128)


def gelu(z):
    return 0.5 * z * (1.0 + torch.erf(z / np.sqrt(2.0)))


def features(cell_map: np.ndarray, n_occ: int, diag: np.ndarray, B: np.ndarray, chi: np.ndarray):
    """(x [L, cells, 13], scale [L], J [3 n_occ, L]) as bdda_fno_features builds them."""
    L = B.shape[1]
    J = B / diag[:, None]
    scale = np.sqrt(np.mean(np.abs(J) ** 2, axis=0))
    ncell = cell_map.size
    x = np.zeros((L, ncell, CIN))
    occ = cell_map >= 0
    m = cell_map[occ]
    x[:, occ, 0] = 1.0
    x[:, occ, 1:7] = chi[None, None, :]
    Jc = J.reshape(n_occ, 3, L)[m]                     # (cells_in, 3, L)
    for a in range(3):
        x[:, occ, 7 + 2 * a] = (Jc[:, a, :].real / scale).T
        x[:, occ, 8 + 2 * a] = (Jc[:, a, :].imag / scale).T
    return x, scale, J


def forward(params: dict, x: torch.Tensor, n, layers: int, modes: int) -> torch.Tensor:
    """x [B, Nx, Ny, Nz, cin] float64 -> y [B, Nx, Ny, Nz, cout]."""
    Nx, Ny, Nz = (int(v) for v in n)
    Fx, Fy, Fz = dft_matrix(Nx, modes), dft_matrix(Ny, modes), dft_matrix(Nz, modes)
    v = x @ params["P"] + params["p"]
    ncell = Nx * Ny * Nz
    for l in range(layers):
        vc = v.to(torch.complex128)
        A = torch.einsum("bxyzc,zk,yj,xi->bijkc", vc, Fz, Fy, Fx)
        R = torch.complex(params["R%d" % l][..., 0], params["R%d" % l][..., 1])      # (K, W, W)
        K = modes ** 3
        S = torch.einsum("bki,kio->bko", A.reshape(A.shape[0], K, -1), R).reshape(A.shape)
        s = torch.einsum("bijkc,xi,yj,zk->bxyzc", S, Fx.conj(), Fy.conj(), Fz.conj()).real / ncell
        z = v @ params["W%d" % l] + params["b%d" % l] + s
        v = gelu(z) if l + 1 < layers else z
    h = gelu(v @ params["Q1"] + params["q1"])
    return h @ params["Q2"] + params["q2"]


def loss(y: torch.Tensor, target: torch.Tensor, mask: torch.Tensor) -> torch.Tensor:
    """Mean over samples of sum mask |y - t|^2 / sum mask |t|^2 (bdda_fno_loss)."""
    m = mask[None, ..., None]
    num = ((y - target) ** 2 * m).flatten(1).sum(1)
    den = (target ** 2 * m).flatten(1).sum(1)
    return (num / den).mean()


def target(cell_map: np.ndarray, n_occ: int, J: np.ndarray, X: np.ndarray, scale: np.ndarray) -> np.ndarray:
    """(X - J) / scale at the occupied cells, [L, cells, 6]."""
    L = X.shape[1]
    t = np.zeros((L, cell_map.size, 6))
    occ = cell_map >= 0
    D = ((X - J) / scale[None, :]).reshape(n_occ, 3, L)[cell_map[occ]]
    for a in range(3):
        t[:, occ, 2 * a] = D[:, a, :].real.T
        t[:, occ, 2 * a + 1] = D[:, a, :].imag.T
    return t
