"""Batched block-BiCGSTAB (bdda_batch_bicgstab) against the one-problem
solver: problems with different grids, occupancies and right-hand sides in
one call give, each, the one-problem result (the same residual history over
the first iterations, the stopping iteration within a few, X within the
solve tolerance's reach), and one problem's breakdown or NaN does not touch
the others."""
import os

import numpy as np
import pytest
import torch

from oracle import dda_oracle as O
from bdda_b200.inputs import load_geometry

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def rel(a, b):
    a = a.cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a)
    b = b.cpu().numpy() if isinstance(b, torch.Tensor) else np.asarray(b)
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


def _problem(name, L, seed, keep=1.0):
    if name == "elongated":   # a GRE with a non-cubic lattice: passes of one kind differ in length
        from bdda_b200.inputs import so3_euler
        from bdda_b200.shapes import gre_particle
        rec = gre_particle(5.0, 0.6, 0.7, 0.1, seed=7, coarse=(13, 50))
        rec.update(euler=so3_euler(L, 5), m_p_xyz=np.array([1.5 + 0.01j, 1.55 + 0.01j, 1.45 + 0.02j]))
    else:
        rec = load_geometry(os.path.join(GOLDEN, name + ".npz"))
    rng = np.random.default_rng(seed)
    n, lf = rec["lattice_n"], float(rec["lattice_lf"])
    address = rec["address"]
    if keep < 1.0:
        address = np.sort(rng.choice(address, int(keep * address.size), replace=False))
    geom = O.incident_geometry(float(rec["wl_0"]), float(rec["m_m"]), rec["euler"])
    _, _, diag = O.polarizability(rec["m_p_xyz"], float(rec["m_m"]), lf, geom["k"], address.size)
    B = rng.standard_normal((3 * address.size, L)) + 1j * rng.standard_normal((3 * address.size, L))
    return dict(n=n, lf=lf, k=geom["k"], address=address, diag=diag, B=B)


@pytest.fixture(scope="module")
def bk():
    from bl_krylov import bl_krylov
    return bl_krylov


@pytest.fixture(scope="module")
def batch(bk):
    from mvp_fft import mvp_fft
    L = 8
    probs = [_problem("kat_test_dda", L, 1), _problem("geometry_cfg1", L, 2),
             _problem("geometry_cfg1", L, 3, keep=0.6), _problem("kat_test_dda", L, 4, keep=0.8),
             _problem("elongated", L, 6)]
    for p in probs:
        p["til"] = mf_til = mvp_fft.fft_init(p["n"], 3, p["lf"], p["k"])
        del mf_til
    return probs


def _args(p, B=None, X0=None):
    t = (p["n"], p["address"], p["til"], p["diag"], p["B"] if B is None else B)
    return t if X0 is None else t + (X0,)


def _single(t):
    """Batch problem tuple -> positional arguments of the one-problem solver (f = 3)."""
    return (t[0], 3) + tuple(t[1:5])


@pytest.mark.parametrize("precision", ["c128", "c64"])
def test_batch_matches_one_problem_solves(bk, batch, precision):
    tol = 1e-8 if precision == "c128" else 1e-4
    hist = []
    out = bk.bl_bicgstab_jacobi_mvp_fft_batch([_args(p) for p in batch], tol, 300, precision=precision,
                                              history=hist)
    for p, (X, it, err), h in zip(batch, out, hist):
        hs = []
        Xs, its, errs = bk.bl_bicgstab_jacobi_mvp_fft(*_single(_args(p)), tol, 300, precision=precision,
                                                      history=hs)
        assert err < tol and errs < tol
        # the batch splits its reductions differently, so rounding differs: the first
        # iterations follow the one-problem trajectory, the stopping iteration near a
        # tight tolerance may move by a few
        first = 8 if precision == "c128" else 3
        assert np.allclose(h[:first], hs[:first], rtol=1e-7 if precision == "c128" else 1e-3, atol=0)
        assert abs(it - its) <= 3
        assert len(h) == it + 1 and abs(h[-1] - err) <= 1e-12 * err
        assert rel(X, Xs) < (1e-6 if precision == "c128" else 5e-3)


def test_graph_replay_equals_direct_launches(bk, batch):
    args = [_args(p) for p in batch]
    a = bk.bl_bicgstab_jacobi_mvp_fft_batch(args, 1e-6, 200, graph=True)
    b = bk.bl_bicgstab_jacobi_mvp_fft_batch(args, 1e-6, 200, graph=False)
    for (Xa, ia, ea), (Xb, ib, eb) in zip(a, b):
        assert ia == ib and ea == eb and np.array_equal(Xa, Xb)


def test_mixed_batch_meets_true_residual(bk, batch):
    tol = 1e-5
    out = bk.bl_bicgstab_jacobi_mvp_fft_batch([_args(p) for p in batch], tol, 400, precision="mixed")
    for p, (X, it, err) in zip(batch, out):
        assert err < tol
        true = O.true_residual(p["n"], 3, p["address"], O.fft_init(p["n"], 3, p["lf"], p["k"]), p["diag"],
                               p["B"], X)
        assert abs(true - err) < 1e-3 * err + 1e-9     # err_fin is the FP64 true residual
        Xs, its, errs = bk.bl_bicgstab_jacobi_mvp_fft(*_single(_args(p)), tol, 400, precision="mixed")
        assert abs(it - its) <= 3
        assert rel(X, Xs) < 1e-3


def test_warm_start_and_itermax_zero(bk, batch):
    sols = [bk.bl_bicgstab_jacobi_mvp_fft(*_single(_args(p)), 1e-9, 300)[0] for p in batch]
    out = bk.bl_bicgstab_jacobi_mvp_fft_batch([_args(p, X0=x) for p, x in zip(batch, sols)], 1e-6, 50)
    for (X, it, err), x in zip(out, sols):
        assert it == 0 and err < 1e-6 and rel(X, x) < 1e-6
    out = bk.bl_bicgstab_jacobi_mvp_fft_batch([_args(p) for p in batch], 1e-6, 0)
    for X, it, err in out:
        assert it == 0 and err == float("inf") and not np.any(X)


def test_one_problem_failing_leaves_the_others(bk, batch):
    Bdup = batch[1]["B"].copy()
    Bdup[:, 2] = Bdup[:, 0]                       # R0^H V exactly singular
    Bnan = batch[2]["B"].copy()
    Bnan[7, 3] = np.nan
    args = [_args(batch[0]), _args(batch[1], B=Bdup), _args(batch[2], B=Bnan), _args(batch[3]), _args(batch[4])]
    st = []
    out = bk.bl_bicgstab_jacobi_mvp_fft_batch(args, 1e-6, 200, statuses=st)
    assert st[0] == 0 and st[3] == 0 and st[4] == 0 and st[1] == 2 and st[2] == 1
    assert out[1][0] is None and not np.isfinite(out[2][2])
    for i in (0, 3, 4):
        Xs, its, _ = bk.bl_bicgstab_jacobi_mvp_fft(*_single(args[i]), 1e-6, 200)
        assert abs(out[i][1] - its) <= 1 and rel(out[i][0], Xs) < 1e-4
    with pytest.raises(np.linalg.LinAlgError):
        bk.bl_bicgstab_jacobi_mvp_fft_batch(args[:2], 1e-6, 200)


def test_bad_arguments(bk, batch):
    p = batch[0]
    with pytest.raises(ValueError):   # L not shared
        bk.bl_bicgstab_jacobi_mvp_fft_batch([_args(p), _args(p, B=p["B"][:, :4])], 1e-6, 10)
    with pytest.raises(ValueError):   # L not one of 8, 16, 32, 64
        bk.bl_bicgstab_jacobi_mvp_fft_batch([_args(p, B=np.tile(p["B"], (1, 2))[:, :12])], 1e-6, 10)
    with pytest.raises(ValueError):
        bk.bl_bicgstab_jacobi_mvp_fft_batch([_args(p)], 1e-6, 10, precision="c32")


def test_groups_split_by_workspace(bk, batch):
    """A workspace bound smaller than the whole batch splits it into groups; results do not change."""
    from bdda_b200 import _lib
    args = [_args(p) for p in batch]
    full = bk.bl_bicgstab_jacobi_mvp_fft_batch(args, 1e-6, 200)
    ents = [bk._batch_entry(a) for a in args]
    one = int(_lib.load().bdda_batch_workspace_bytes(bk._batch_struct(ents[1:2], 0), 1, 0, 8, 200))
    split = bk.bl_bicgstab_jacobi_mvp_fft_batch(args, 1e-6, 200, max_bytes=one + 1)
    for (Xa, ia, ea), (Xb, ib, eb) in zip(full, split):   # groups of one run the one-problem solver
        assert ea < 1e-6 and eb < 1e-6 and abs(ia - ib) <= 3 and rel(Xa, Xb) < 1e-4
