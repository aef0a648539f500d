"""libbdda.so loads, exports every entry point of include/bdda.h, and its
host-only plan logic behaves (no GPU needed)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from bdda_b200 import _lib

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "bdda.h")


def header_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(bdda_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    names = header_functions()
    assert len(names) >= 15
    for name in names:
        assert hasattr(lib, name), name


def test_bindings_cover_the_header_exactly():
    assert sorted(_lib.PROTOTYPES) == header_functions()


def test_status_strings():
    assert _lib.status_string(_lib.OK) == "ok"
    assert "singular" in _lib.status_string(_lib.BREAKDOWN)
    with pytest.raises(ValueError):
        _lib.check(_lib.BAD_ARG, "x")
    with pytest.raises(np.linalg.LinAlgError):
        _lib.check(_lib.BREAKDOWN, "x")
    assert _lib.check(_lib.NOT_CONVERGED, "x") == _lib.NOT_CONVERGED


def _plan(n, m=None):
    lib = _lib.load()
    h = C.c_void_p()
    st = lib.bdda_plan_create(_lib.int3(n), None if m is None else _lib.int3(m), C.byref(h))
    if st != _lib.OK:
        return st, None, None
    mm = (C.c_int * 3)()
    lib.bdda_plan_grid(h, mm)
    rad = []
    for a in range(3):
        r = (C.c_int * 12)()
        ns = C.c_int()
        lib.bdda_plan_radices(h, a, r, C.byref(ns))
        rad.append([r[i] for i in range(ns.value)])
    lib.bdda_plan_destroy(h)
    return st, list(mm), rad


def smooth7(m):
    for p in (2, 3, 5, 7):
        while m % p == 0:
            m //= p
    return m == 1


@pytest.mark.parametrize("n", [(28, 28, 28), (17, 17, 17), (93, 112, 174), (5, 6, 7), (1, 1, 1),
                               (11, 13, 37), (3, 2, 4), (64, 100, 215)])
def test_plan_grid_choice(n):
    """Each axis gets an even 7-smooth length >= 2N factored into radices <= 10;
    the x axis (fused Green multiply) ends with a radix <= 4; lengths stay
    within 2N + 2N/4."""
    st, m, rad = _plan(n)
    assert st == _lib.OK
    for a, (N, M, r) in enumerate(zip(n, m, rad)):
        assert 2 * N <= M <= 2 * N + (2 * N) // 4 + 2 and M % 2 == 0 and smooth7(M)
        assert int(np.prod(r)) == M and set(r) <= {2, 3, 4, 5, 6, 7, 8, 9, 10}
        assert r == sorted(r, reverse=True)
        if a == 0:
            assert r[-1] <= 4


def test_plan_factorization_minimises_stages():
    st, m, rad = _plan((93, 112, 174), (192, 224, 350))
    assert st == _lib.OK
    assert [len(r) for r in rad] == [3, 3, 3]
    st, m, rad = _plan((28, 28, 28), (56, 56, 56))
    assert rad[1] == [8, 7] and rad[0][-1] <= 4


def test_plan_accepts_explicit_grid_and_rejects_short_or_rough():
    assert _plan((5, 4, 6), (9, 10, 15))[0] == _lib.OK
    assert _plan((5, 4, 6), (8, 10, 15))[0] == _lib.BAD_ARG     # 8 < 2*5-1
    assert _plan((5, 4, 6), (11, 10, 15))[0] == _lib.BAD_ARG    # 11 is not 7-smooth
    assert _plan((0, 4, 6))[0] == _lib.BAD_ARG


def test_batch_workspace_query_checks_arguments():
    """Host-only: the batched solver's workspace query accepts valid work lists and rejects bad ones."""
    import ctypes as C
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "block-dda_py_b200"))
    from bl_krylov.bl_krylov import _BatchProblem
    lib = _lib.load()
    plans = []
    for n in ((8, 7, 6), (17, 17, 17)):
        h = C.c_void_p()
        assert lib.bdda_plan_create((C.c_int * 3)(*n), None, C.byref(h)) == 0
        plans.append(h)
    arr = (_BatchProblem * 2)()
    for i, h in enumerate(plans):
        s = arr[i]
        s.plan = h.value
        s.n_occ = 100 * (i + 1)
        s.ghat = s.ghat_c64 = s.cell_map = s.diag = s.B = s.X = 256   # never dereferenced by the query
    try:
        b8 = lib.bdda_batch_workspace_bytes(arr, 2, _lib.BATCH_MIXED, 8, 50)
        b64 = lib.bdda_batch_workspace_bytes(arr, 2, _lib.BATCH_MIXED, 64, 50)
        assert 0 < b8 < b64
        assert lib.bdda_batch_workspace_bytes(arr, 2, _lib.BATCH_C64, 8, 50) < b8
        assert lib.bdda_batch_workspace_bytes(arr, 2, _lib.BATCH_MIXED, 12, 50) == 0   # L not 8/16/32/64
        assert lib.bdda_batch_workspace_bytes(arr, 0, _lib.BATCH_MIXED, 8, 50) == 0
        assert lib.bdda_batch_workspace_bytes(arr, 2, 3, 8, 50) == 0
        arr[1].ghat_c64 = None
        assert lib.bdda_batch_workspace_bytes(arr, 2, _lib.BATCH_MIXED, 8, 50) == 0   # spectrum missing
        assert lib.bdda_batch_workspace_bytes(arr, 2, _lib.BATCH_C128, 8, 50) > 0
    finally:
        for h in plans:
            lib.bdda_plan_destroy(h)


def test_mixed_settings_round_trip_and_reject_bad_values():
    """Host-only: bdda_tune_mixed sets the mixed BiCGSTAB's replacement drop,
    complex128 switch and divergence factor, keeps them on bad values, and
    bdda_tune_mixed_get reads them."""
    lib = _lib.load()
    d, s, f = C.c_double(), C.c_double(), C.c_double()
    get = lambda: (lib.bdda_tune_mixed_get(C.byref(d), C.byref(s), C.byref(f)), d.value, s.value, f.value)
    rc, d0, s0, f0 = get()
    assert rc == 0 and (d0, s0, f0) == (0.1, 0.0, 10.0)
    try:
        assert lib.bdda_tune_mixed(0.05, 10.0, 50.0) == 0
        assert get() == (0, 0.05, 10.0, 50.0)
        for bad in ((0.0, 0.0, 10.0), (1.0, 0.0, 10.0), (0.1, -1.0, 10.0), (float("nan"), 0.0, 10.0),
                    (0.1, 0.0, 1.0), (0.1, 0.0, float("nan"))):
            assert lib.bdda_tune_mixed(*bad) == _lib.BAD_ARG
        assert get() == (0, 0.05, 10.0, 50.0)
        assert lib.bdda_tune_mixed_get(None, C.byref(s), C.byref(f)) == _lib.BAD_ARG
    finally:
        lib.bdda_tune_mixed(d0, s0, f0)


def test_pass_variant_lists_name_the_compiled_kernels():
    """Host-only: for the x=20 particle's grid (192 x 224 x 350) every complex64
    pass has one-column and column-pair (id bit 512) specialised kernels at
    tile width 8, complex128 only one-column ones; the passes with a dense
    source also have TMA-filled ones (id >= 1024); the count is reported even
    when cap is 0; bad arguments are rejected."""
    lib = _lib.load()
    h = C.c_void_p()
    assert lib.bdda_plan_create((C.c_int * 3)(93, 112, 174), None, C.byref(h)) == 0
    try:
        m = (C.c_int * 3)()
        assert lib.bdda_plan_grid(h, m) == 0 and list(m) == [192, 224, 350]
        buf, n = (C.c_int * 64)(), C.c_int()
        for kind, axis in ((0, 2), (0, 1), (1, 0), (2, 1), (2, 2)):
            assert lib.bdda_tune_pass_variants(h, 1, kind, axis, 8, buf, 64, C.byref(n)) == 0
            ids = list(buf[:n.value])
            assert any(v >= 512 for v in ids) and any(0 < v < 512 for v in ids), (kind, axis, ids)
            assert len(set(ids)) == len(ids)
            assert lib.bdda_tune_pass_variants(h, 1, kind, axis, 8, None, 0, C.byref(n)) == 0 and n.value == len(ids)
            # dense-source passes (all but the gathering Z pass) also have TMA-filled kernels (id >= 1024)
            assert any(v & 1024 for v in ids) == ((kind, axis) != (0, 2)), (kind, axis, ids)
            # the X pass also has two-stage (24 x 8) kernels, ids from 2048
            assert any(v >= 2048 for v in ids) == ((kind, axis) == (1, 0)), (kind, axis, ids)
            assert lib.bdda_tune_pass_variants(h, 0, kind, axis, 4, buf, 64, C.byref(n)) == 0
            ids = list(buf[:n.value])
            assert ids and all(not (v & 512) for v in ids) and len(set(ids)) == len(ids), (kind, axis, ids)
            assert any(v & 1024 for v in ids) == ((kind, axis) != (0, 2)), (kind, axis, ids)
        assert lib.bdda_tune_pass_variants(h, 1, 3, 0, 8, buf, 64, C.byref(n)) == _lib.BAD_ARG
        assert lib.bdda_tune_pass_variants(h, 1, 1, 3, 8, buf, 64, C.byref(n)) == _lib.BAD_ARG
        assert lib.bdda_tune_pass_variants(None, 1, 1, 0, 8, buf, 64, C.byref(n)) == _lib.BAD_ARG
        # the wait-timeout counter lives in the device tables: none attached yet
        cnt = C.c_uint()
        assert lib.bdda_plan_wait_timeouts(h, C.byref(cnt), None) == _lib.NO_WORKSPACE
        assert lib.bdda_plan_wait_timeouts(h, None, None) == _lib.BAD_ARG
        assert lib.bdda_plan_wait_timeouts(None, C.byref(cnt), None) == _lib.BAD_ARG
    finally:
        lib.bdda_plan_destroy(h)
