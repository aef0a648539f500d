"""The block MVP entry point that allocates nothing.

Some callers cannot call cudaMalloc -- a plugin whose host application's
allocator owns all device memory, or a latency-critical path that cannot take
the synchronisation an allocation may imply.  bdda_block_mvp_noalloc keeps its
scratch in a static device array instead of a caller workspace.  This test
calls it through the C ABI and compares it with bdda_block_mvp (which takes a
caller workspace) on two calls in a row.  It lives in its own file, collected
last, and passes both alone in a fresh process and after the other tests.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

TOL = 1e-12   # the complex128 product tolerance used by the other MVP tests


def test_noalloc_block_mvp_matches_workspace_entry_point():
    from bdda_b200 import _lib
    from bdda_b200.runtime import GreenTensor, Occupancy, Plan, ptr, stream_ptr
    lib = _lib.load()
    rng = np.random.default_rng(11)
    n, L = (14, 12, 10), 4
    nc = 14 * 12 * 10
    plan = Plan(n)
    green = GreenTensor(plan, 0.05, 9.0)
    occ = Occupancy(plan, np.sort(rng.choice(nc, 1000, replace=False)))
    N = occ.n_occ
    assert lib.bdda_block_mvp_noalloc_fits(plan.handle, _lib.C128, L) == 1
    need = int(lib.bdda_mvp_workspace_bytes(plan.handle, _lib.C128, L))
    assert 0 < need <= int(lib.bdda_block_mvp_noalloc_max_bytes())
    dev = torch.device("cuda")
    diag = torch.from_numpy((rng.standard_normal(3 * N) + 5.0) + 1j * rng.standard_normal(3 * N)).to(dev)
    jpre = 1.0 / diag
    work = torch.empty(need, dtype=torch.uint8, device=dev)
    gh = green.ghat(_lib.C128)
    for call in range(2):   # two calls in a row share (and reuse) the static scratch
        S = torch.from_numpy(rng.standard_normal((3 * N, L)) + 1j * rng.standard_normal((3 * N, L))).to(dev)
        ref = torch.empty_like(S)
        out = torch.empty_like(S)
        _lib.check(lib.bdda_block_mvp(plan.handle, _lib.C128, L, ptr(gh), ptr(occ.cell_map), ptr(diag),
                                      ptr(jpre), ptr(S), ptr(ref), ptr(work), stream_ptr()), "bdda_block_mvp")
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        _lib.check(lib.bdda_block_mvp_noalloc(plan.handle, _lib.C128, L, ptr(gh), ptr(occ.cell_map), ptr(diag),
                                              ptr(jpre), ptr(S), ptr(out), stream_ptr()),
                   "bdda_block_mvp_noalloc")
        torch.cuda.synchronize()
        free_after = torch.cuda.mem_get_info()[0]
        if call == 1:
            # the first call may load the library's device code (and with it the
            # static array); from then on a call takes no device memory at all
            assert free_after == free_before, (free_before, free_after)
        err = (out - ref).abs().max().item() / ref.abs().max().item()
        assert err < TOL, (call, err)


def test_noalloc_rejects_problems_larger_than_its_scratch():
    from bdda_b200 import _lib
    from bdda_b200.runtime import Plan
    lib = _lib.load()
    plan = Plan((40, 40, 40))
    assert int(lib.bdda_mvp_workspace_bytes(plan.handle, _lib.C128, 64)) > int(lib.bdda_block_mvp_noalloc_max_bytes())
    assert lib.bdda_block_mvp_noalloc_fits(plan.handle, _lib.C128, 64) == 0
    # rejected before anything is launched
    st = lib.bdda_block_mvp_noalloc(plan.handle, _lib.C128, 64, None, None, None, None, None, None, None)
    assert st == _lib.BAD_ARG
