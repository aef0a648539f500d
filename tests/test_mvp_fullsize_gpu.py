"""Block MVP at the full size of the x=20 particle (93 x 112 x 174 lattice,
438,606 dipoles, L = 64): specialised vs generic kernels, FP32 vs FP64, and
selected output dipoles against a direct O(N) sum over every source."""
import os

import numpy as np
import pytest
import torch

from oracle import dda_oracle as O
from bdda_b200.inputs import lattice_index, load_geometry

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def case():
    from bdda_b200 import _lib
    from bdda_b200.runtime import GreenTensor, Occupancy, Plan
    geo = load_geometry(os.path.join(GOLDEN, "geometry_cfg2.npz"))
    k = 2 * np.pi * float(geo["m_m"]) / float(geo["wl_0"])
    plan = Plan(geo["lattice_n"])
    green = GreenTensor(plan, geo["lattice_lf"], k)
    occ = Occupancy(plan, geo["address"])
    gen = torch.Generator(device="cuda").manual_seed(7)
    S = torch.randn((3 * occ.n_occ, 64), dtype=torch.complex128, device="cuda", generator=gen)
    return dict(lib=_lib, geo=geo, k=k, plan=plan, green=green, occ=occ, S=S)


def _mvp(c, prec, S):
    from bdda_b200.runtime import TORCH_DTYPE, ptr, stream_ptr
    lib = c["lib"]
    dt = TORCH_DTYPE[prec]
    Sd = S.to(dt)
    one = torch.ones(Sd.shape[0], dtype=dt, device="cuda")   # diag = jpre = 1: out = S + A_off S
    out = torch.empty_like(Sd)
    work = c["green"].workspace(prec, Sd.shape[1])
    lib.check(lib.load().bdda_block_mvp(c["plan"].handle, prec, Sd.shape[1], ptr(c["green"].ghat(prec)),
                                        ptr(c["occ"].cell_map), ptr(one), ptr(one), ptr(Sd), ptr(out),
                                        ptr(work), stream_ptr()), "mvp")
    torch.cuda.synchronize()
    return out.to(torch.complex128) - S


def test_specialised_kernels_match_generic_and_direct_sum(case):
    lib = case["lib"].load()
    Y = _mvp(case, 0, case["S"])
    lib.bdda_tune_fixed(0)
    try:
        Yg = _mvp(case, 0, case["S"])
    finally:
        lib.bdda_tune_fixed(1)
    scale = Y.abs().max().item()
    assert (Y - Yg).abs().max().item() / scale < 1e-12
    # direct sum over all 438,606 sources for four output dipoles (first 8 columns)
    geo = case["geo"]
    pidx = lattice_index(geo["address"], geo["lattice_n"])
    rows = [0, 123457, 300001, case["occ"].n_occ - 1]
    S8 = case["S"][:, :8].cpu().numpy()
    d = O.direct_offdiag_rows(rows, pidx, geo["lattice_lf"], case["k"], S8)
    Yr = Y[:, :8].cpu().numpy().reshape(-1, 3, 8)[rows]
    assert np.max(np.abs(Yr - d)) / np.max(np.abs(d)) < 1e-11


def test_fp32_product_tracks_fp64(case):
    Y = _mvp(case, 0, case["S"])
    Y32 = _mvp(case, 1, case["S"])
    assert (Y32 - Y).abs().max().item() / Y.abs().max().item() < 2e-5


@pytest.mark.parametrize("prec", [0, 1])
def test_autotuned_launch_choices_keep_the_product(case, prec):
    """The autotuner only changes launch shapes: every candidate it leaves in
    place gives the same product, and it never ends slower than it started
    by more than timing noise."""
    from bdda_b200.runtime import autotune
    lib = case["lib"].load()
    Y0 = _mvp(case, prec, case["S"])
    before, after = autotune(case["green"], case["occ"], 64, prec, reps=2)
    assert after <= 1.05 * before
    import ctypes as C
    lt, var = C.c_int(), C.c_int()
    mx = case["plan"].m[0]
    assert lib.bdda_tune_pass_get(prec, 1, mx, 64, C.byref(lt), C.byref(var)) == 0
    assert lt.value in (2, 4, 8) and var.value >= -1
    Y1 = _mvp(case, prec, case["S"])
    tol = 1e-12 if prec == 0 else 2e-5
    assert (Y1 - Y0).abs().max().item() / Y0.abs().max().item() < tol


def test_every_compiled_complex64_variant_gives_the_product(case):
    """Each specialised complex64 kernel of each pass (one-column and
    column-pair jobs, every CTA size and register bound), forced in turn,
    gives the product of the pass's generic kernel: the pair kernels run the
    one-column arithmetic on 16-byte accesses, so the difference stays at
    the level of the generic kernel's own rounding (<= 1e-6 relative)."""
    import ctypes as C
    lib = case["lib"].load()
    plan = case["plan"]
    Y0 = _mvp(case, 1, case["S"])
    scale = Y0.abs().max().item()
    tested = 0
    try:
        for kind, axis in ((0, 2), (0, 1), (1, 0), (2, 1), (2, 2)):
            M = plan.m[axis]
            buf, n = (C.c_int * 64)(), C.c_int()
            assert lib.bdda_tune_pass_variants(plan.handle, 1, kind, axis, 8, buf, 64, C.byref(n)) == 0
            variants = list(buf[:n.value])
            assert any(v >= 512 for v in variants), (kind, axis, variants)
            for v in variants + [-1]:
                assert lib.bdda_tune_pass(1, kind, M, 64, 8, v) == 0
                Y = _mvp(case, 1, case["S"])
                err = (Y - Y0).abs().max().item() / scale
                assert err < 1e-6, (kind, axis, v, err)
                tested += 1
            assert lib.bdda_tune_pass(1, kind, M, 64, 0, 0) == 0
    finally:
        for kind, axis in ((0, 2), (0, 1), (1, 0), (2, 1), (2, 2)):
            lib.bdda_tune_pass(1, kind, plan.m[axis], 64, 0, 0)
    assert tested >= 20
    assert plan.wait_timeouts() == 0


@pytest.mark.parametrize("prec", [0, 1])
def test_tma_filled_tiles_give_the_plain_kernels_product(case, prec):
    """Each kernel whose tile is filled by a bulk tensor copy (id >= 1024)
    gives the product of the same kernel with the first stage's global loads
    (id - 1024) to rounding: the copy moves the same values, zero-filled past
    the source rows and columns as the loads are, and the arithmetic is the
    same source (complex128 1e-15; complex64 1e-6, where the compiler's
    contraction of the two instantiations may differ); no bounded wait of the
    copies ran out."""
    import ctypes as C
    lib = case["lib"].load()
    plan = case["plan"]
    tested = 0
    try:
        for kind, axis in ((0, 1), (1, 0), (2, 1), (2, 2)):
            M = plan.m[axis]
            n_tma = 0
            for lt in (4, 8):
                buf, n = (C.c_int * 64)(), C.c_int()
                assert lib.bdda_tune_pass_variants(plan.handle, prec, kind, axis, lt, buf, 64, C.byref(n)) == 0
                for v in [v for v in buf[:n.value] if v & 1024]:
                    assert lib.bdda_tune_pass(prec, kind, M, 64, lt, v - 1024) == 0
                    Yp = _mvp(case, prec, case["S"])
                    assert lib.bdda_tune_pass(prec, kind, M, 64, lt, v) == 0
                    Yt = _mvp(case, prec, case["S"])
                    err = (Yt - Yp).abs().max().item() / Yp.abs().max().item()
                    assert err <= (1e-15 if prec == 0 else 1e-6), (prec, kind, axis, lt, v, err)
                    n_tma += 1
            assert n_tma, (prec, kind, axis)
            tested += n_tma
            assert lib.bdda_tune_pass(prec, kind, M, 64, 0, 0) == 0
    finally:
        for kind, axis in ((0, 2), (0, 1), (1, 0), (2, 1), (2, 2)):
            lib.bdda_tune_pass(prec, kind, plan.m[axis], 64, 0, 0)
    assert tested >= 4
    assert plan.wait_timeouts() == 0


@pytest.mark.parametrize("prec", [0, 1])
def test_generic_kernels_with_tma_tiles_give_the_same_product(case, prec):
    """The run-time-radix kernels with the TMA-filled tile (variant -2, the
    default for radix sequences without specialised kernels) give the product
    of the same kernels with the first stage's global loads (variant -1):
    complex128 to 1e-15, complex64 to 1e-6."""
    lib = case["lib"].load()
    plan = case["plan"]
    passes = ((0, 2), (0, 1), (1, 0), (2, 1), (2, 2))
    out = {}
    try:
        for v in (-1, -2):
            for kind, axis in passes:
                assert lib.bdda_tune_pass(prec, kind, plan.m[axis], 64, 8 if prec else 4, v) == 0
            out[v] = _mvp(case, prec, case["S"])
    finally:
        for kind, axis in passes:
            lib.bdda_tune_pass(prec, kind, plan.m[axis], 64, 0, 0)
    err = (out[-2] - out[-1]).abs().max().item() / out[-1].abs().max().item()
    assert err <= (1e-15 if prec == 0 else 1e-6), err
    assert plan.wait_timeouts() == 0


@pytest.mark.parametrize("prec", [0, 1])
def test_two_stage_x_pass_gives_the_plan_stage_product(case, prec):
    """The X-pass kernels that transform the 192-point axis as 24 x 8 (ids
    from 2048; the plan's stages are [8,8,3]) give the product of the
    generic run-time-radix kernels: 1e-12 in complex128, 1e-6 in complex64
    (different rounding order); with and without the TMA-filled tile."""
    import ctypes as C
    lib = case["lib"].load()
    plan = case["plan"]
    M = plan.m[0]
    lib.bdda_tune_fixed(0)
    try:
        Yg = _mvp(case, prec, case["S"])
    finally:
        lib.bdda_tune_fixed(1)
    scale = Yg.abs().max().item()
    tested = 0
    try:
        for lt in (4, 8):
            buf, n = (C.c_int * 64)(), C.c_int()
            assert lib.bdda_tune_pass_variants(plan.handle, prec, 1, 0, lt, buf, 64, C.byref(n)) == 0
            for v in [v for v in buf[:n.value] if v >= 2048]:
                assert lib.bdda_tune_pass(prec, 1, M, 64, lt, v) == 0
                Y = _mvp(case, prec, case["S"])
                err = (Y - Yg).abs().max().item() / scale
                assert err < (1e-12 if prec == 0 else 1e-6), (prec, lt, v, err)
                tested += 1
    finally:
        lib.bdda_tune_pass(prec, 1, M, 64, 0, 0)
    assert tested >= 4
    assert plan.wait_timeouts() == 0
