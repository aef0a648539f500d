"""The learned warm start's CPU oracle (float64 autograd) against central
finite differences, and its feature / target construction (CPU)."""
import numpy as np
import torch

from oracle import fno_oracle as F


def _case(seed=2):
    rng = np.random.default_rng(seed)
    n = (6, 7, 8)
    ncell = int(np.prod(n))
    address = np.sort(rng.choice(ncell, 200, replace=False))
    cell_map = np.full(ncell, -1, np.int64)
    cell_map[address] = np.arange(address.size)
    L = 2
    diag = rng.uniform(2, 5, 3 * address.size) + 1j * rng.uniform(-1, 1, 3 * address.size)
    B = rng.standard_normal((3 * address.size, L)) + 1j * rng.standard_normal((3 * address.size, L))
    X = B / diag[:, None] * (1 + 0.2 * rng.standard_normal((3 * address.size, L)))
    return n, cell_map, address.size, L, diag, B, X, rng


def test_oracle_gradients_match_finite_differences():
    n, cell_map, n_occ, L, diag, B, X, rng = _case()
    layers, modes = 2, 4
    flat = rng.standard_normal(sum(int(np.prod(sh)) for _, sh in F.param_layout(layers, modes))) * 0.1
    x, scale, J = F.features(cell_map, n_occ, diag, B, np.array([0.3, 0.01] * 3))
    xt = torch.tensor(x.reshape((L,) + n + (13,)))
    t = torch.tensor(F.target(cell_map, n_occ, J, X, scale).reshape((L,) + n + (6,)))
    mask = torch.tensor((cell_map >= 0).reshape(n).astype(np.float64))

    def f(v):
        p = F.unflatten(v, layers, modes)
        return F.loss(F.forward(p, xt, n, layers, modes), t, mask)
    p = F.unflatten(flat, layers, modes)
    F.loss(F.forward(p, xt, n, layers, modes), t, mask).backward()
    g = F.flatten_grads(p, layers, modes)
    for idx in rng.choice(flat.size, 8, replace=False):
        e = np.zeros_like(flat)
        e[idx] = 1e-5
        fd = (f(flat + e).item() - f(flat - e).item()) / 2e-5
        assert abs(fd - g[idx]) < 1e-7 + 1e-5 * abs(g[idx])


def test_features_and_target_layout():
    n, cell_map, n_occ, L, diag, B, X, rng = _case(3)
    x, scale, J = F.features(cell_map, n_occ, diag, B, np.arange(6.0))
    occ = cell_map >= 0
    assert np.all(x[:, ~occ, :] == 0) and np.all(x[:, occ, 0] == 1) and np.all(x[:, occ, 1:7] == np.arange(6.0))
    m = 5
    cell = np.flatnonzero(cell_map == m)[0]
    for a in range(3):
        assert np.isclose(x[1, cell, 7 + 2 * a] * scale[1], J[3 * m + a, 1].real)
    t = F.target(cell_map, n_occ, J, X, scale)
    assert np.isclose(t[0, cell, 3] * scale[0], (X - J)[3 * m + 1, 0].imag)
    # the DFT matrix keeps frequencies 0, 1 and N-2, N-1 for 4 modes
    Fm = F.dft_matrix(9, 4).numpy()
    assert np.allclose(Fm[1, :], np.exp(-2j * np.pi * np.array([0, 1, 7, 8]) / 9))
