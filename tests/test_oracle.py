"""The CPU oracle against the reference's golden vectors (no GPU needed).

The fixtures in tests/golden/ were produced by the live reference
(tests/golden/make_golden.py); the notebook values are the outputs recorded
in the reference's test_dda.ipynb.
"""
import numpy as np
import pytest
from scipy.spatial.transform import Rotation

from conftest import load_golden
from oracle import dda_oracle as O
from bdda_b200.inputs import lattice_index, lattice_points, load_geometry
import os

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def rel(a, b):
    return np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(np.max(np.abs(b)), 1e-300)


def test_green_tensor_matches_reference():
    g = load_golden("green_small")
    A = O.build_interaction_tensor(g["n"], float(g["lf"]), float(g["k"]))
    assert A.shape == g["A"].shape
    assert rel(A, g["A"]) < 1e-14
    At = O.fft_init(g["n"], 3, float(g["lf"]), float(g["k"]))
    assert rel(At, g["A_til"]) < 1e-14


def test_fft_init_rejects_f_not_3():
    with pytest.raises(ValueError):
        O.fft_init([2, 2, 2], 2, 0.1, 1.0)


def test_fft_mvp_matches_reference():
    g = load_golden("fft_mvp_small")
    At = O.fft_init(g["n"], 3, float(g["lf"]), float(g["k"]))
    assert rel(O.fft_mvp(g["n"], 3, At, g["P"]), g["Y"]) < 1e-14
    y1 = O.fft_mvp(g["n"], 3, At, g["p1"])
    assert y1.shape == g["y1"].shape and rel(y1, g["y1"]) < 1e-14


def test_scatter_index_and_block_mvp_match_reference():
    g = load_golden("block_mvp_small")
    idx = O.scatter_index(g["address"], 3)
    assert np.array_equal(idx, g["full_idx"])
    At = O.fft_init(g["n"], 3, float(g["lf"]), float(g["k"]))
    AS = O.block_mvp(g["n"], 3, At, idx, g["diag_A"], g["S"], 1.0 / g["diag_A"])
    assert rel(AS, g["AS"]) < 1e-14


@pytest.mark.parametrize("solver", ["bicgstab", "cocg"])
def test_solvers_match_reference(solver):
    g = load_golden("solver_small")
    At = O.fft_init(g["n"], 3, float(g["lf"]), float(g["k"]))
    fn = O.bicgstab if solver == "bicgstab" else O.cocg_rq
    hist = []
    X, it, err = fn(g["n"], 3, g["address"], At, g["diag_A"], g["B"], 1e-5, 200, history=hist)
    assert it == int(g[solver + "_iter_fin"])
    assert abs(err - float(g[solver + "_err_fin"])) <= 1e-9 * abs(float(g[solver + "_err_fin"]))
    # the reference printed the history to 4 decimals
    assert np.allclose(np.round(hist, 4), g[solver + "_history"], atol=0)
    assert rel(X, g[solver + "_X"]) < 1e-10


def test_padded_grid_gives_the_same_product():
    """Any cyclic length m >= 2n-1 reproduces the doubled-grid product."""
    rng = np.random.default_rng(5)
    n, lf, k = [5, 4, 6], 0.05, 7.0
    m = [9, 10, 15]     # 2n-1, 2n+2, 2n+3
    P = rng.standard_normal((3 * 120, 2)) + 1j * rng.standard_normal((3 * 120, 2))
    ref = O.fft_mvp(n, 3, O.fft_init(n, 3, lf, k), P)
    G = np.fft.fftn(O.sym6_to_full(O.green_components(n, lf, k, m)), axes=(0, 1, 2))
    grid = np.zeros(tuple(m) + (3, 2), complex)
    grid[:5, :4, :6] = P.reshape(5, 4, 6, 3, 2)
    out = np.fft.ifftn(G @ np.fft.fftn(grid, axes=(0, 1, 2)), axes=(0, 1, 2))[:5, :4, :6]
    assert rel(out.reshape(-1, 2), ref) < 1e-13


def test_direct_rows_match_fft_product():
    rng = np.random.default_rng(6)
    n, lf, k = [6, 5, 7], 0.04, 9.0
    nc = 210
    address = np.sort(rng.choice(nc, 150, replace=False))
    S = rng.standard_normal((450, 3)) + 1j * rng.standard_normal((450, 3))
    full = np.zeros((3 * nc, 3), complex)
    full[O.scatter_index(address, 3)] = S
    Y = O.fft_mvp(n, 3, O.fft_init(n, 3, lf, k), full)[O.scatter_index(address, 3)]
    rows = [0, 17, 149]
    d = O.direct_offdiag_rows(rows, lattice_index(address, n), lf, k, S)
    assert rel(d, Y.reshape(-1, 3, 3)[rows]) < 1e-12


def test_rotation_matches_scipy():
    rng = np.random.default_rng(7)
    e = rng.uniform(0, 2 * np.pi, (16, 3))
    R = Rotation.from_euler("ZYZ", e[:, ::-1] * -1.0).as_matrix()
    assert np.max(np.abs(O.lab_to_particle(e) - R)) < 1e-14


def _solve_case(rec, solver, tol, itermax):
    geo = rec
    n = geo["lattice_n"]
    lf = geo["lattice_lf"]
    address = geo["address"]
    pos = geo["grid"][address]
    g = O.incident_geometry(float(rec["wl_0"]), float(rec["m_m"]), rec["euler"])
    eper_r, _, diag = O.polarizability(rec["m_p_xyz"], float(rec["m_m"]), lf, g["k"], address.size)
    B = O.rhs(g["k"], g["u_inc"], g["e0_inc"], pos)
    At = O.fft_init(n, 3, lf, g["k"])
    fn = O.bicgstab if solver == "bicgstab" else O.cocg_rq
    hist = []
    X, it, err = fn(n, 3, address, At, diag, B, tol, itermax, history=hist)
    obs = O.observables(X, g, pos, eper_r, lf)
    return dict(X=X, it=it, err=err, hist=hist, obs=obs, diag=diag)


def test_test_dda_notebook_known_answers():
    """test_dda.ipynb: 17^3 lattice, 1,840 dipoles, BiCGSTAB tol 1e-2, L=10."""
    rec = load_geometry(os.path.join(GOLDEN, "kat_test_dda.npz"))
    assert list(rec["lattice_n"]) == [17, 17, 17]                       # test_dda.ipynb:92
    assert rec["address"].size == 1840
    res = _solve_case(rec, "bicgstab", 1e-2, 25)
    assert res["it"] == 1                                              # :189-191
    assert [round(h, 4) for h in res["hist"]] == [0.0156, 0.0002]
    # S_bk as printed by the notebook (test_dda.ipynb:316-321), 8 significant digits
    nb = np.array([0.00135109 + 0.00372118j, -0.00141074 + 0.0032077j, 0.00144375 + 0.00374011j,
                   -0.00083594 + 0.00331428j, -0.00124069 + 0.00324015j, -0.00053676 + 0.00336732j,
                   0.00109785 + 0.00367712j, 0.00171865 + 0.00379029j, 0.00151792 + 0.00375321j,
                   0.00119338 + 0.00369024j])
    assert np.allclose(res["obs"]["S_bk"], nb, rtol=0, atol=6e-9)
    # live reference values, full precision
    for key in ("C_abs", "C_ext", "S_fw_theta", "S_fw_phi", "S_bk"):
        assert rel(res["obs"][key], rec[key]) < 1e-12, key
    assert rel(res["diag"], rec["diag_A"]) < 1e-15
    # |Q_abs/Q_abs_mie - 1| printed at test_dda.ipynb:231-232 (Mie value from :208-209)
    r_ve = np.cbrt(3 * rec["lattice_lf"] ** 3 * 1840 / (4 * np.pi))
    q_abs = res["obs"]["C_abs"] / (np.pi * r_ve ** 2)
    printed = np.array([0.00234075, 0.00082194, 0.00247296, 0.00015358, 0.00059328, 0.00013724,
                        0.00211581, 0.00278785, 0.00257769, 0.00216351])
    assert np.allclose(np.abs(q_abs / 0.04493662949384336 - 1), printed, atol=6e-9)


# At tol 1e-5 the reference's own iterate moves by ~1e-5 relative (S_bk up to
# 2e-5) and by one iteration when B changes at the 1e-16 level, so there the
# check is: iterations within 1 and outputs within 1e-4.  Converged to 1e-11
# the outputs are fixed by the problem and must agree within 1e-8.
CFG1_CASES = [("cocg", 1e-5, ""), ("bicgstab", 1e-5, "bicgstab_tol5_"),
              ("cocg", 1e-11, "cocg_tight_"), ("bicgstab", 1e-11, "bicgstab_tight_")]


@pytest.mark.parametrize("solver,tol,tag", CFG1_CASES)
def test_config1_sphere_matches_reference(solver, tol, tag):
    """Sphere x=5, 28^3 lattice (9,445 dipoles), L=8 SO(3) orientations (seed 0)."""
    rec = load_geometry(os.path.join(GOLDEN, "geometry_cfg1.npz"))
    assert rec["address"].size == 9445
    res = _solve_case(rec, solver, tol, 300)
    assert abs(res["it"] - int(rec[tag + "iter_fin"])) <= 1
    bound = 1e-4 if tol > 1e-6 else 1e-8
    for key in ("C_abs", "C_ext", "S_fw_theta", "S_fw_phi", "S_bk"):
        assert rel(res["obs"][key], rec[tag + key]) < bound, key


def test_geometry_records_rebuild_reference_lattice():
    rec = load_geometry(os.path.join(GOLDEN, "kat_test_dda.npz"))
    pts = lattice_points(rec["x_axis"], rec["y_axis"], rec["z_axis"])
    assert pts.shape == (17 ** 3, 3)
    idx = lattice_index(rec["address"], rec["lattice_n"])
    assert np.allclose(pts[rec["address"]], np.column_stack(
        [rec["x_axis"][idx[:, 0]], rec["y_axis"][idx[:, 1]], rec["z_axis"][idx[:, 2]]]))
