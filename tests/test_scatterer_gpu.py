"""The bl_dda.scatterer drop-in end to end on the GPU (RHS, solve, observables)."""
import os

import numpy as np
import pytest

from oracle import dda_oracle as O
from bdda_b200.inputs import load_geometry

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def rel(a, b):
    return np.max(np.abs(np.asarray(a) - b)) / max(np.max(np.abs(b)), 1e-300)


def _dd(rec, m_p=None):
    from bl_dda import scatterer as sc
    sc.DiscreteDipoles.verbose = False
    target = sc.Target("gre", rec["lattice_n"], rec["lattice_lf"], rec["grid"], rec["is_in"],
                       rec["m_p_xyz"] if m_p is None else m_p)
    inc = sc.IncidentField(float(rec["wl_0"]), float(rec["m_m"]), rec["euler"])
    return sc.DiscreteDipoles(target, inc)


def test_notebook_case_through_public_api():
    """test_dda.ipynb cells 4-14 with the drop-in classes."""
    rec = load_geometry(os.path.join(GOLDEN, "kat_test_dda.npz"))
    dd = _dd(rec)
    dd.set_interaction_matrix()
    assert rel(dd.diag_A, rec["diag_A"]) < 1e-15
    pos = rec["grid"][rec["address"]]
    g = O.incident_geometry(float(rec["wl_0"]), float(rec["m_m"]), rec["euler"])
    assert rel(dd.B, O.rhs(g["k"], g["u_inc"], g["e0_inc"], pos)) < 1e-14
    dd.solve_matrix_equation()
    assert dd.converge and dd.iter_fin == 1
    assert rel(dd.compute_C_abs(), rec["C_abs"]) < 1e-10
    assert rel(dd.compute_C_ext(), rec["C_ext"]) < 1e-10
    st, sp = dd.compute_PCAS_observable_S_fw()
    assert rel(st, rec["S_fw_theta"]) < 1e-10 and rel(sp, rec["S_fw_phi"]) < 1e-10
    sbk = dd.compute_OCBS_observable_S_bk()
    assert rel(sbk, rec["S_bk"]) < 1e-10
    nb = np.array([0.00135109 + 0.00372118j, -0.00141074 + 0.0032077j, 0.00144375 + 0.00374011j,
                   -0.00083594 + 0.00331428j, -0.00124069 + 0.00324015j, -0.00053676 + 0.00336732j,
                   0.00109785 + 0.00367712j, 0.00171865 + 0.00379029j, 0.00151792 + 0.00375321j,
                   0.00119338 + 0.00369024j])                              # test_dda.ipynb:316-321
    assert np.allclose(sbk, nb, rtol=0, atol=6e-9)
    # reference attribute shapes
    assert dd.P.shape == (10, 1840, 3) and dd.E.shape == (10, 1840, 3)
    assert dd.E_inc.shape == (10, 1840, 3) and dd.X.shape == (5520, 10)


def test_config1_sphere_cocg_through_public_api():
    rec = load_geometry(os.path.join(GOLDEN, "geometry_cfg1.npz"))
    dd = _dd(rec)
    dd.tol, dd.itermax, dd.solver = 1e-5, 300, "cocg"
    dd.set_interaction_matrix()
    dd.solve_matrix_equation()
    assert dd.converge and abs(dd.iter_fin - int(rec["iter_fin"])) <= 1
    assert rel(dd.compute_C_ext(), rec["C_ext"]) < 1e-4
    assert rel(dd.compute_OCBS_observable_S_bk(), rec["S_bk"]) < 1e-4
    st, sp = dd.compute_PCAS_observable_S_fw()
    assert rel(st, rec["S_fw_theta"]) < 1e-4 and rel(sp, rec["S_fw_phi"]) < 1e-4


def test_non_absorbing_particle_has_zero_c_abs_and_unconverged_is_zero():
    rec = load_geometry(os.path.join(GOLDEN, "kat_test_dda.npz"))
    dd = _dd(rec, m_p=np.array([1.4, 1.4, 1.4]))
    dd.set_interaction_matrix()
    dd.solve_matrix_equation()
    assert np.all(dd.compute_C_abs() == 0.0)
    dd2 = _dd(rec)
    dd2.itermax, dd2.tol = 1, 1e-12
    dd2.set_interaction_matrix()
    dd2.solve_matrix_equation()
    assert not dd2.converge
    assert np.all(dd2.compute_C_ext() == 0.0)      # P stays zero, as in the reference


@pytest.mark.parametrize("solver,precision", [("bicgstab", None), ("cocg", None), ("bicgstab", "mixed"),
                                              ("bicgstab", "c64")])
def test_fused_solve_matches_the_separate_steps(solver, precision):
    """bdda_dda_solve (right-hand side formed in the prologue, observables in the
    epilogue) against polarizability + RHS kernels, the bl_krylov solver and the
    observables kernel run one after another on the same inputs."""
    from bl_krylov import bl_krylov as bk
    rec = load_geometry(os.path.join(GOLDEN, "geometry_cfg1.npz"))
    dd = _dd(rec)
    dd.tol, dd.itermax, dd.solver, dd.precision = 1e-6, 300, solver, precision
    dd.set_interaction_matrix()
    dd.solve_matrix_equation()
    obs_fused = dd.observables().copy()
    ref = _dd(rec)
    ref.set_interaction_matrix(green=dd.Au_til)
    ref._materialize()
    fn = bk.bl_cocg_rq_jacobi_mvp_fft if solver == "cocg" else bk.bl_bicgstab_jacobi_mvp_fft
    X, it, err = fn(ref.lattice_n, 3, ref._dev["occ"], ref.Au_til, ref._dev["diag"], ref._dev["B"], 1e-6, 300,
                    precision=precision)
    assert it == dd.iter_fin and abs(err - dd.err_fin) <= 1e-12 * err
    assert rel(dd.X, X.cpu().numpy()) < 1e-12
    ref._dev["X"] = X
    ref.converge = True
    assert rel(obs_fused, ref.observables()) < 1e-12
    assert rel(dd.diag_A, ref.diag_A) == 0.0 and rel(dd.eper_r, ref.eper_r) == 0.0


def test_more_than_64_orientations_are_solved_in_blocks():
    """L = 70: two blocks of 35 through the fused entry point, each the same as
    a solve of those 35 orientations alone."""
    from bdda_b200.inputs import so3_euler
    from bl_dda import scatterer as sc
    rec = load_geometry(os.path.join(GOLDEN, "kat_test_dda.npz"))
    euler = so3_euler(70, 9)
    sc.DiscreteDipoles.verbose = False
    target = sc.Target("gre", rec["lattice_n"], rec["lattice_lf"], rec["grid"], rec["is_in"], rec["m_p_xyz"])
    dd = sc.DiscreteDipoles(target, sc.IncidentField(float(rec["wl_0"]), float(rec["m_m"]), euler))
    dd.tol, dd.itermax = 1e-6, 200
    dd.set_interaction_matrix()
    dd.solve_matrix_equation()
    assert dd.converge and dd.X.shape == (3 * rec["address"].size, 70)
    obs = dd.observables()
    for l0, l1 in ((0, 35), (35, 70)):
        d = sc.DiscreteDipoles(target, sc.IncidentField(float(rec["wl_0"]), float(rec["m_m"]), euler[l0:l1]))
        d.tol, d.itermax = 1e-6, 200
        d.set_interaction_matrix(green=dd.Au_til)
        d.solve_matrix_equation()
        assert rel(dd.X[:, l0:l1], d.X) < 1e-13
        assert rel(obs[l0:l1], d.observables()) < 1e-13
