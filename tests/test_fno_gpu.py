"""Learned warm start: the hand-written FNO kernels against the float64 CPU
oracle (features, forward output, loss, and the gradient of every parameter
block), and the warm start with its fallback rule."""
import ctypes as C

import numpy as np
import pytest
import torch

from oracle import fno_oracle as F

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-30))


@pytest.fixture(scope="module")
def small():
    """A 12 x 13 x 14 lattice, 60 % occupied, L = 3 orientations, random data."""
    from bdda_b200.runtime import Occupancy, Plan
    rng = np.random.default_rng(11)
    n = (12, 13, 14)
    ncell = int(np.prod(n))
    address = np.sort(rng.choice(ncell, int(0.6 * ncell), replace=False))
    n_occ = address.size
    L = 3
    diag = (rng.uniform(2, 5, 3 * n_occ) + 1j * rng.uniform(-1, 1, 3 * n_occ))
    B = rng.standard_normal((3 * n_occ, L)) + 1j * rng.standard_normal((3 * n_occ, L))
    X = B / diag[:, None] * (1 + 0.3 * rng.standard_normal((3 * n_occ, L)))
    eps = np.array([2.3 + 0.1j, 2.5 + 0.05j, 2.1 + 0.2j])
    plan = Plan(n)
    occ = Occupancy(plan, address)
    cell_map = np.full(ncell, -1, np.int64)
    cell_map[address] = np.arange(n_occ)
    return dict(n=n, L=L, n_occ=n_occ, diag=diag, B=B, X=X, eps=eps, occ=occ, cell_map=cell_map, rng=rng)


def test_fno_kernels_match_cpu_oracle(small):
    from bdda_b200.warmstart import WarmStartFNO, chi_of
    s = small
    layers, modes = 2, 4
    model = WarmStartFNO(layers=layers, modes=modes, seed=3)
    # random (not just initial) parameters so every path carries signal
    g = torch.Generator(device="cpu").manual_seed(5)
    model.params.copy_((torch.randn(model.n_params, generator=g) * 0.15).to(model.device))
    dev = model.device
    diag = torch.as_tensor(s["diag"], device=dev)
    B = torch.as_tensor(s["B"], device=dev)
    X = torch.as_tensor(s["X"], device=dev)
    n, L, ncell = s["n"], s["L"], int(np.prod(s["n"]))
    loss_gpu = model.loss_and_grad(n, s["occ"], diag, B, s["eps"], X)
    work = model._workspace(L, n)
    x_gpu = model.buffer(work, L, n, 0, L * ncell * 13).cpu().numpy().reshape(L, ncell, 13)
    y_gpu = model.buffer(work, L, n, 1, L * ncell * 6).cpu().numpy().reshape(L, ncell, 6)
    # features
    x_ref, scale, J = F.features(s["cell_map"], s["n_occ"], s["diag"], s["B"], chi_of(s["eps"]))
    assert _rel(x_gpu, x_ref) < 1e-6
    # forward on the same (FP32) features, loss, gradients
    params = F.unflatten(model.params.cpu().numpy(), layers, modes)
    xt = torch.tensor(x_gpu.astype(np.float64).reshape((L,) + tuple(n) + (13,)))
    y = F.forward(params, xt, n, layers, modes)
    assert _rel(y_gpu.reshape(y.shape), y.detach().numpy()) < 1e-4
    t = F.target(s["cell_map"], s["n_occ"], J, s["X"], scale).reshape((L,) + tuple(n) + (6,))
    mask = torch.tensor((s["cell_map"] >= 0).reshape(n).astype(np.float64))
    loss = F.loss(y, torch.tensor(t), mask)
    assert abs(loss_gpu - loss.item()) < 1e-4 * loss.item()
    loss.backward()
    g_gpu = model.grads.cpu().numpy()
    off = 0
    for name, shape in F.param_layout(layers, modes):
        k = int(np.prod(shape))
        gr = params[name].grad.numpy().ravel()
        assert _rel(g_gpu[off:off + k], gr) < 2e-3, name
        off += k


def test_warm_start_is_jacobi_plus_scaled_output_and_falls_back(small):
    from bdda_b200.warmstart import WarmStartFNO
    from mvp_fft import mvp_fft
    s = small
    model = WarmStartFNO(layers=2, modes=4, seed=1)
    dev = model.device
    diag = torch.as_tensor(s["diag"], device=dev)
    B = torch.as_tensor(s["B"], device=dev)
    X0 = model.predict(s["n"], s["occ"], diag, B, s["eps"]).cpu().numpy()
    L, ncell = s["L"], int(np.prod(s["n"]))
    work = model._workspace(L, s["n"])
    y = model.buffer(work, L, s["n"], 1, L * ncell * 6).cpu().numpy().reshape(L, ncell, 6)
    _, scale, J = F.features(s["cell_map"], s["n_occ"], s["diag"], s["B"], np.zeros(6))
    occ = s["cell_map"] >= 0
    yo = y[:, occ, :]                                   # (L, n_occ, 6) in dipole order
    corr = (yo[..., 0::2] + 1j * yo[..., 1::2]).transpose(1, 2, 0).reshape(3 * s["n_occ"], L)
    assert _rel(X0, J + corr * scale[None, :]) < 1e-6
    # a column whose predicted initial residual exceeds ||M^-1 B|| starts from zero
    green = mvp_fft.fft_init(s["n"], 3, 0.05, 2.0)
    X0w, nfb = model.warm_start(s["n"], s["occ"], green, diag, B, s["eps"])
    assert 0 <= nfb <= L
    if X0w is not None:
        zero_cols = (X0w.abs().sum(0) == 0).sum().item()
        assert zero_cols == nfb


def test_trained_warm_start_gains_over_zero_start():
    """Trained on the GPU on solver solutions (24 small GRE particles), the
    warm start the solver receives (after the fallback rule) lowers the
    initial residual of held-out particles below the zero start's (relative
    residual 1) and costs no iterations; every solve converges to the same
    tolerance."""
    from bdda_b200.warmstart import WarmStartFNO, make_dataset, sample_particles
    from bl_krylov import bl_krylov as bk
    kw = dict(x_range=(4.0, 6.0))
    train = make_dataset(sample_particles(24, seed=7, **kw), L=8)
    held = make_dataset(sample_particles(4, seed=77, **kw), L=8)
    model = WarmStartFNO(layers=4, modes=6, seed=7)
    losses = model.fit(train, epochs=12, lr=2e-3, lr_final=2e-4, seed=7)
    assert losses[-1] < 0.7 * losses[0]
    r0, it_zero, it_warm = [], 0, 0
    for d in held:
        X0, nfb = model.warm_start(d["n"], d["occ"], d["green"], d["diag"], d["B"], d["eps_r"])
        Bj = d["B"] / d["diag"][:, None]
        if X0 is None:
            r0.append(1.0)
        else:
            AX = bk._block_mvp(d["n"], 3, d["green"], bk._build_scatter_index(d["occ"].address, 3), d["diag"], X0,
                               1.0 / d["diag"])
            r0.append(float((torch.linalg.vector_norm(Bj - AX) / torch.linalg.vector_norm(Bj)).item()))
        args = (d["n"], 3, d["occ"], d["green"], d["diag"], d["B"], 1e-5, 400)
        _, i0, e0 = bk.bl_bicgstab_jacobi_mvp_fft(*args)
        _, i1, e1 = bk.bl_bicgstab_jacobi_mvp_fft(*args, X0=X0)
        assert e0 < 1e-5 and e1 < 1e-5
        it_zero += i0 + 1
        it_warm += i1 + 1
    assert max(r0) <= 1.0 + 1e-9 and np.mean(r0) < 0.95
    assert it_warm <= it_zero + 2
    # the projected start (least-squares fit over the predicted columns) starts
    # no higher than the per-column fallback, and converges to the same tolerance
    for d, r_fb in zip(held, r0):
        Xp, nfb = model.warm_start(d["n"], d["occ"], d["green"], d["diag"], d["B"], d["eps_r"], mode="project")
        assert nfb == 0
        Bj = d["B"] / d["diag"][:, None]
        AX = bk._block_mvp(d["n"], 3, d["green"], bk._build_scatter_index(d["occ"].address, 3), d["diag"], Xp,
                           1.0 / d["diag"])
        rp = float((torch.linalg.vector_norm(Bj - AX) / torch.linalg.vector_norm(Bj)).item())
        assert rp <= r_fb + 1e-9
        _, ip, ep = bk.bl_bicgstab_jacobi_mvp_fft(d["n"], 3, d["occ"], d["green"], d["diag"], d["B"], 1e-5, 400,
                                                  X0=Xp)
        assert ep < 1e-5
