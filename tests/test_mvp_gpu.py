"""GPU parity of the Green's tensor and the FFT products against the oracle
and the reference's golden vectors (sm_100a kernels through the C ABI)."""
import numpy as np
import pytest
import torch

from conftest import load_golden
from oracle import dda_oracle as O

pytestmark = pytest.mark.gpu

# complex128 products: FFT rounding only (a few 1e-15 of the largest entry);
# complex64 products: FP32 rounding of the same chain.
TOL_C128 = 1e-12
TOL_C64 = 2e-5


def rel(a, b):
    a = a.cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a)
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


@pytest.fixture(scope="module")
def mf():
    from mvp_fft import mvp_fft
    return mvp_fft


@pytest.fixture(scope="module")
def bk():
    from bl_krylov import bl_krylov
    return bl_krylov


def test_interaction_tensor_matches_reference(mf):
    g = load_golden("green_small")
    A = mf.build_interaction_tensor(g["n"], float(g["lf"]), float(g["k"]))
    assert A.shape == g["A"].shape and A.dtype == np.complex128
    assert rel(A, g["A"]) < 1e-14


def test_fft_init_matches_reference(mf):
    g = load_golden("green_small")
    til = mf.fft_init(g["n"], 3, float(g["lf"]), float(g["k"]))
    assert til.shape == g["A_til"].shape
    assert rel(np.asarray(til), g["A_til"]) < TOL_C128
    with pytest.raises(ValueError):
        mf.fft_init(g["n"], 2, float(g["lf"]), float(g["k"]))


def test_fft_mvp_matches_reference(mf):
    g = load_golden("fft_mvp_small")
    til = mf.fft_init(g["n"], 3, float(g["lf"]), float(g["k"]))
    assert rel(mf.fft_mvp(g["n"], 3, til, g["P"]), g["Y"]) < TOL_C128
    y1 = mf.fft_mvp(g["n"], 3, til, g["p1"])
    assert y1.shape == g["y1"].shape and rel(y1, g["y1"]) < TOL_C128
    # a spectrum handed over in the reference's own layout is adopted as-is
    ref_til = O.fft_init(g["n"], 3, float(g["lf"]), float(g["k"]))
    assert rel(mf.fft_mvp(g["n"], 3, ref_til, g["P"]), g["Y"]) < TOL_C128
    # FP32 product
    assert rel(mf.fft_mvp(g["n"], 3, til, g["P"], precision="c64"), g["Y"]) < TOL_C64


def test_block_mvp_matches_reference(bk, mf):
    g = load_golden("block_mvp_small")
    til = mf.fft_init(g["n"], 3, float(g["lf"]), float(g["k"]))
    AS = bk._block_mvp(g["n"], 3, til, g["full_idx"], g["diag_A"], g["S"], 1.0 / g["diag_A"])
    assert rel(AS, g["AS"]) < TOL_C128


# odd, prime, padded (non-2N) and unit sizes; L from 1 to 11
CASES = [((7, 9, 11), 3), ((13, 5, 6), 1), ((28, 28, 28), 8), ((4, 17, 3), 5), ((1, 6, 5), 2),
         ((19, 11, 37), 11), ((12, 12, 12), 64)]


@pytest.mark.parametrize("n,L", CASES)
@pytest.mark.parametrize("prec", ["c128", "c64"])
def test_block_mvp_random_against_oracle(bk, mf, n, L, prec):
    rng = np.random.default_rng(hash((n, L)) % 2 ** 32)
    nc = int(np.prod(n))
    address = np.sort(rng.choice(nc, max(1, int(0.6 * nc)), replace=False))
    N = address.size
    lf, k = 0.045, 2 * np.pi * 1.33 / 0.7
    diag = (rng.standard_normal(3 * N) + 4.0) + 1j * rng.standard_normal(3 * N)
    S = rng.standard_normal((3 * N, L)) + 1j * rng.standard_normal((3 * N, L))
    til_ref = O.fft_init(n, 3, lf, k)
    idx = O.scatter_index(address, 3)
    ref = O.block_mvp(n, 3, til_ref, idx, diag, S, 1.0 / diag)
    til = mf.fft_init(n, 3, lf, k)
    out = bk._block_mvp(n, 3, til, idx, diag, S, 1.0 / diag, precision=prec)
    assert rel(out, ref) < (TOL_C128 if prec == "c128" else TOL_C64)


def test_fft_mvp_is_linear_and_device_resident(mf):
    """Torch inputs stay on the device; A(aP + bQ) = a AP + b AQ."""
    n = (24, 20, 30)
    rng = np.random.default_rng(3)
    til = mf.fft_init(n, 3, 0.03, 9.0)
    dev = torch.device("cuda")
    P = torch.from_numpy(rng.standard_normal((3 * 14400, 4)) + 1j * rng.standard_normal((3 * 14400, 4))).to(dev)
    Q = torch.from_numpy(rng.standard_normal((3 * 14400, 4)) + 1j * rng.standard_normal((3 * 14400, 4))).to(dev)
    a, b = 0.3 - 1.1j, 2.0 + 0.5j
    lhs = mf.fft_mvp(n, 3, til, a * P + b * Q)
    rhs = a * mf.fft_mvp(n, 3, til, P) + b * mf.fft_mvp(n, 3, til, Q)
    assert lhs.is_cuda
    assert (lhs - rhs).abs().max().item() / rhs.abs().max().item() < 1e-13


def test_green_tensor_on_padded_grid(mf):
    """An explicit non-doubled grid gives the same product."""
    n = (5, 4, 6)
    rng = np.random.default_rng(4)
    P = rng.standard_normal((360, 2)) + 1j * rng.standard_normal((360, 2))
    ref = O.fft_mvp(n, 3, O.fft_init(n, 3, 0.05, 7.0), P)
    til = mf.fft_init(n, 3, 0.05, 7.0, m=(9, 10, 15))
    assert rel(mf.fft_mvp(n, 3, til, P), ref) < TOL_C128
