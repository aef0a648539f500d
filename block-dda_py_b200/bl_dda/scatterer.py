"""GPU drop-in for the reference module ``bl_dda.scatterer``.

``Target``, ``IncidentField`` and ``DiscreteDipoles`` keep the reference's
constructors, methods and attribute names (bl_dda/scatterer.py:8-227).  The
heavy state (Green's spectrum, diagonal, right-hand side, solution) lives on
the GPU; the reference's NumPy attributes (``B``, ``X``, ``P``, ``E``,
``E_inc``, ``diag_A`` ...) are produced on first access.  Added keywords are
optional and keep the reference's behaviour by default.
"""
from __future__ import annotations

import ctypes as C
import time

import numpy as np
import torch

from bdda_b200 import _lib
from bdda_b200.runtime import Occupancy, ptr, require_cuda, stream_ptr, to_device
from bl_krylov import bl_krylov
from mvp_fft.mvp_fft import fft_init


class _DdaProblem(C.Structure):
    """include/bdda.h: bdda_dda_problem."""
    _fields_ = [("n_occ", C.c_int), ("L", C.c_int), ("m_p_xyz", C.c_double * 6), ("m_m", C.c_double),
                ("lf", C.c_double), ("k", C.c_double), ("absorbing", C.c_int), ("pos", C.c_void_p),
                ("vec", C.c_void_p), ("e0", C.c_void_p)]


def _rot_z(t):
    c, s = np.cos(t), np.sin(t)
    R = np.zeros(t.shape + (3, 3))
    R[..., 0, 0], R[..., 0, 1], R[..., 1, 0], R[..., 1, 1], R[..., 2, 2] = c, -s, s, c, 1.0
    return R


def _rot_y(t):
    c, s = np.cos(t), np.sin(t)
    R = np.zeros(t.shape + (3, 3))
    R[..., 0, 0], R[..., 0, 2], R[..., 1, 1], R[..., 2, 0], R[..., 2, 2] = c, s, 1.0, -s, c
    return R


class Target:
    """Lattice geometry and refractive index of one particle (scatterer.py:8-28)."""

    def __init__(self, shape_name, lattice_n, lattice_lf, lattice_grid_points,
                 lattice_grid_points_is_in_target, m_p_xyz):
        self.shape_name = shape_name
        self.lattice_n = lattice_n
        self.lattice_lf = lattice_lf
        self.lattice_grid_points = lattice_grid_points
        self.lattice_grid_points_is_in_target = lattice_grid_points_is_in_target
        self.m_p_xyz = m_p_xyz
        self.lattice_address_in_target = np.where(lattice_grid_points_is_in_target)[0]
        self.lattice_pos_in_target = lattice_grid_points[self.lattice_address_in_target, :]
        self.num_element_occupy = self.lattice_address_in_target.size
        self.element_vol = self.lattice_lf ** 3
        self.m_p = np.ones_like(self.lattice_pos_in_target) * m_p_xyz
        self.eper_p = self.m_p ** 2
        self.total_vol = self.element_vol * self.num_element_occupy
        self.ve_radius = np.cbrt(3 * self.total_vol / (4 * np.pi))


class IncidentField:
    """Incident wave and scattering directions rotated into the particle frame (scatterer.py:31-85).

    The lab -> particle rotation is intrinsic ZYZ(-gamma, -beta, -alpha),
    i.e. Rz(-gamma) Ry(-beta) Rz(-alpha), per orientation.
    """

    def __init__(self, wl_0, m_m, euler_angles):
        self.wl_0 = wl_0
        self.m_m = m_m
        self.eper_m = m_m ** 2
        self.k = 2 * np.pi * m_m / wl_0
        self.euler_angles = euler_angles
        self.L = euler_angles.shape[0]
        ex, ey, ez = np.eye(3)
        self.e0_inc_pol_theta = 1 / np.sqrt(2)
        self.e0_inc_pol_phi = 1j / np.sqrt(2)
        e = np.asarray(euler_angles, dtype=np.float64)
        R = _rot_z(-e[:, 2]) @ _rot_y(-e[:, 1]) @ _rot_z(-e[:, 0])
        self.u_inc_vec_P = R @ ez
        self.theta_inc_vec_P = R @ ex
        self.phi_inc_vec_P = R @ ey
        self.e0_inc_vec_P = (self.e0_inc_pol_theta * self.theta_inc_vec_P
                             + self.e0_inc_pol_phi * self.phi_inc_vec_P)
        self.u_sca_fw_vec_P = R @ ez
        self.theta_sca_fw_vec_P = R @ ex
        self.phi_sca_fw_vec_P = R @ ey
        self.u_sca_bk_vec_P = R @ (-ez)
        self.theta_sca_bk_vec_P = R @ (-ex)
        self.phi_sca_bk_vec_P = R @ ey


class DiscreteDipoles(Target, IncidentField):
    """The DDA system of one particle for L orientations (scatterer.py:88-227).

    Solver settings as the reference: ``itermax = 25``, ``tol = 1e-2``.
    ``solver`` ("bicgstab", the reference's fixed choice, or "cocg") and
    ``precision`` ("c128" default, "c64") are extra, optional attributes.
    """

    verbose = True

    def __init__(self, target, incidentfield):
        Target.__init__(self, target.shape_name, target.lattice_n, target.lattice_lf,
                        target.lattice_grid_points, target.lattice_grid_points_is_in_target,
                        target.m_p_xyz)
        IncidentField.__init__(self, incidentfield.wl_0, incidentfield.m_m, incidentfield.euler_angles)
        self.device = require_cuda()
        self.dpl = (self.wl_0 / np.abs(np.max(self.m_p_xyz))) / self.lattice_lf
        self.f = 3
        self.itermax = 25
        self.tol = 1e-2
        self.converge = False
        self.solver = "bicgstab"
        self.precision = None
        self.iter_fin = None
        self.err_fin = None
        self.Au_til = None
        self._dev = {}
        self._host = {}
        self._obs = None
        if self.verbose:
            print("Number of dipoles per wavelength in the particle volume: dpl= {:}".format(self.dpl))

    # ---- device state --------------------------------------------------------
    def _geometry_to_device(self):
        if "pos" not in self._dev:
            self._dev["pos"] = to_device(self.lattice_pos_in_target, torch.float64, self.device)
        return self._dev["pos"]

    def _absorbing(self) -> int:
        er = (np.asarray(self.m_p_xyz).astype(np.complex128) ** 2) / self.eper_m
        return int(np.mean(er.imag) >= 1e-12)

    def _geometry_vectors(self):
        if "vec" not in self._dev:
            v = np.stack([self.u_inc_vec_P, self.u_sca_fw_vec_P, self.theta_sca_fw_vec_P,
                          self.phi_sca_fw_vec_P, self.u_sca_bk_vec_P, self.theta_sca_bk_vec_P,
                          self.phi_sca_bk_vec_P], axis=1).reshape(self.L, 21)
            self._dev["vec"] = to_device(v, torch.float64, self.device)
            self._dev["e0"] = to_device(self.e0_inc_vec_P, torch.complex128, self.device)
            self._dev["u_inc"] = to_device(self.u_inc_vec_P, torch.float64, self.device)
        return self._dev["vec"]

    def set_interaction_matrix(self, m=None, green=None):
        """Green's spectrum, and the diagonal and right-hand side on the GPU (scatterer.py:135-161).

        ``green`` (optional) is a spectrum from ``fft_init`` for the same
        lattice, spacing and wavenumber, reused instead of being rebuilt.
        diag_A and B are formed by the solve itself (``bdda_dda_solve``
        builds M^-1 B from the positions in its prologue and never stores B);
        reading ``diag_A`` or ``B`` before, or solving through another entry
        point, materialises them with the polarizability and RHS kernels.
        """
        if green is not None:
            if (green.plan.n != tuple(int(v) for v in self.lattice_n) or green.lf != float(self.lattice_lf)
                    or green.k != float(self.k)):
                raise ValueError("the given Green's spectrum belongs to another lattice or wavenumber")
            self.Au_til = green
        else:
            self.Au_til = fft_init(self.lattice_n, self.f, self.lattice_lf, self.k, m=m)
        if self._dev.get("occ") is None or self._dev["occ"].plan is not self.Au_til.plan:
            self._dev["occ"] = Occupancy(self.Au_til.plan, self.lattice_address_in_target)
        self._geometry_to_device()
        self._geometry_vectors()
        for key in ("diag", "eper", "B", "X", "obs"):
            self._dev.pop(key, None)
        self._host.clear()
        self._obs = None

    def _m_p_doubles(self):
        mp = np.asarray(self.m_p_xyz).astype(np.complex128)
        return [float(v) for z in mp for v in (z.real, z.imag)]

    def _materialize(self):
        """diag_A, eps_r and B as device arrays (polarizability and RHS kernels)."""
        if "diag" in self._dev and "B" in self._dev:
            return
        if self.Au_til is None:
            raise ValueError("call set_interaction_matrix() first")
        lib = _lib.load()
        N, L = self.num_element_occupy, self.L
        if "diag" not in self._dev or "eper" not in self._dev:
            diag = torch.empty(3 * N, dtype=torch.complex128, device=self.device)
            eper = torch.empty(3 * N, dtype=torch.complex128, device=self.device)
            mpd = (C.c_double * 6)(*self._m_p_doubles())
            _lib.check(lib.bdda_polarizability(N, mpd, float(self.m_m), float(self.lattice_lf), float(self.k),
                                               ptr(diag), ptr(eper), stream_ptr(self.device)),
                       "bdda_polarizability")
            self._dev.update(diag=diag, eper=eper)
        B = torch.empty((3 * N, L), dtype=torch.complex128, device=self.device)
        _lib.check(lib.bdda_incident_rhs(N, L, float(self.k), ptr(self._geometry_to_device()),
                                         ptr(self._dev["u_inc"]), ptr(self._dev["e0"]), ptr(B),
                                         stream_ptr(self.device)), "bdda_incident_rhs")
        self._dev["B"] = B

    def _fused_solve(self, X0, solver, mode):
        """set-up + solve + observables in one library call per block of <= 64 orientations."""
        lib = _lib.load()
        N, L = self.num_element_occupy, self.L
        g = self.Au_til
        plan = g.plan
        occ = self._dev["occ"]
        dev = self.device
        need64 = mode != _lib.BATCH_C64
        need32 = mode != _lib.BATCH_C128
        diag = torch.empty(3 * N, dtype=torch.complex128, device=dev)
        eper = torch.empty(3 * N, dtype=torch.complex128, device=dev)
        X = torch.empty((3 * N, L), dtype=torch.complex128, device=dev)
        obs = torch.empty((L, 12), dtype=torch.float64, device=dev)
        X0d = None if X0 is None else to_device(X0, torch.complex128, dev).reshape(3 * N, L)
        nblk = (L + 63) // 64
        bounds = [(b * L // nblk, (b + 1) * L // nblk) for b in range(nblk)]
        iters, errs = [], []
        vec, e0 = self._dev["vec"], self._dev["e0"]
        itermax = int(self.itermax)
        for l0, l1 in bounds:
            Lb = l1 - l0
            prob = _DdaProblem()
            prob.n_occ, prob.L = N, Lb
            prob.m_p_xyz = (C.c_double * 6)(*self._m_p_doubles())
            prob.m_m, prob.lf, prob.k = float(self.m_m), float(self.lattice_lf), float(self.k)
            prob.absorbing = self._absorbing()
            prob.pos = ptr(self._geometry_to_device())
            vb = vec[l0:l1].contiguous()
            eb = e0[l0:l1].contiguous()
            prob.vec, prob.e0 = ptr(vb), ptr(eb)
            Xb = X if nblk == 1 else torch.empty((3 * N, Lb), dtype=torch.complex128, device=dev)
            ob = obs if nblk == 1 else torch.empty((Lb, 12), dtype=torch.float64, device=dev)
            X0b = None if X0d is None else (X0d if nblk == 1 else X0d[:, l0:l1].contiguous())
            nbytes = int(lib.bdda_dda_workspace_bytes(plan.handle, mode, Lb, N))
            work = torch.empty(max(nbytes, 16), dtype=torch.uint8, device=dev)
            hist = (C.c_double * max(itermax, 1))()
            it = C.c_int(0)
            err = C.c_double(float("inf"))
            status = lib.bdda_dda_solve(plan.handle, C.byref(prob), solver, mode,
                                        ptr(g.ghat(_lib.C128)) if need64 else None,
                                        ptr(g.ghat(_lib.C64)) if need32 else None, ptr(occ.cell_map), ptr(X0b),
                                        float(self.tol), itermax, 20, ptr(Xb), ptr(diag), ptr(eper), ptr(ob),
                                        C.byref(it), C.byref(err), hist, ptr(work), nbytes, stream_ptr(dev))
            if status == _lib.BREAKDOWN:
                raise np.linalg.LinAlgError("Singular matrix")
            _lib.check(status, "bdda_dda_solve")
            del work
            if nblk > 1:
                X[:, l0:l1] = Xb
                obs[l0:l1] = ob
            iters.append(it.value)
            errs.append(err.value)
        self._dev.update(diag=diag, eper=eper, X=X, obs=obs)
        # one block: the solver's own values; several: the largest (a bound on the
        # residual of the whole block, whose columns were solved in groups of <= 64)
        return max(iters), max(errs)

    def solve_matrix_equation(self, X0=None, solver=None, precision=None):
        """Block solve to ``self.tol`` within ``self.itermax`` (scatterer.py:164-184).

        The complex128 (default), complex64 and "mixed" forms run the fused
        entry point bdda_dda_solve: right-hand side, solve and observables in
        one call.  Other ``precision`` forms go through ``bl_krylov``.  More
        than 64 orientations are solved in blocks of at most 64.
        """
        solver = solver or self.solver
        precision = precision if precision is not None else self.precision
        start = time.time()
        if self.verbose:
            print("Starting block-%s iterative solver..." % ("BiCGStab" if solver == "bicgstab" else "COCG-rq"))
        if self.Au_til is None:
            raise ValueError("call set_interaction_matrix() first")
        key = "c128" if precision is None else str(precision).lower()
        modes = {"c128": _lib.BATCH_C128, "fp64": _lib.BATCH_C128, "complex128": _lib.BATCH_C128,
                 "c64": _lib.BATCH_C64, "fp32": _lib.BATCH_C64, "complex64": _lib.BATCH_C64,
                 "mixed": _lib.BATCH_MIXED}
        kind = _lib.COCG_RQ if solver == "cocg" else _lib.BICGSTAB
        if key in modes:
            iter_fin, err_fin = self._fused_solve(X0, kind, modes[key])
        else:
            self._materialize()
            fn = (bl_krylov.bl_cocg_rq_jacobi_mvp_fft if solver == "cocg"
                  else bl_krylov.bl_bicgstab_jacobi_mvp_fft)
            X, iter_fin, err_fin = fn(self.lattice_n, self.f, self._dev["occ"], self.Au_til,
                                      self._dev["diag"], self._dev["B"], self.tol, self.itermax, X0=X0,
                                      precision=precision)
            self._dev["X"] = X
            self._dev.pop("obs", None)
        self.iter_fin, self.err_fin = iter_fin, err_fin
        self._host.pop("X", None)
        self._obs = None
        elapsed = time.time() - start
        self.converge = bool(err_fin < self.tol)
        if self.converge and self.verbose:
            print("block-BiCGStab converged! (iter_fin={:}, err_fin={:.4f}, solver time={:.1f}s)".format(
                iter_fin, err_fin, elapsed))

    # ---- reference attributes, produced on access -------------------------------
    def _np(self, key, fn):
        if key not in self._host:
            self._host[key] = fn()
        return self._host[key]

    def _dev_array(self, key):
        if key not in self._dev:
            self._materialize()
        return self._dev[key]

    @property
    def eper_r(self):
        return self._np("eper_r", lambda: self._dev_array("eper").cpu().numpy().reshape(-1, 3))

    @property
    def diag_A(self):
        return self._np("diag_A", lambda: self._dev_array("diag").cpu().numpy())

    @property
    def alpha_E(self):
        return self._np("alpha_E", lambda: (1.0 / self.diag_A).reshape(-1, 3))

    @property
    def B(self):
        return self._np("B", lambda: self._dev_array("B").cpu().numpy())

    @property
    def E_inc(self):
        return self._np("E_inc", lambda: self.B.T.reshape(self.L, self.num_element_occupy, 3))

    @property
    def e_inc_phase(self):
        return self._np("e_inc_phase", lambda: np.exp(1j * self.k * (self.u_inc_vec_P @ self.lattice_pos_in_target.T)))

    @property
    def X(self):
        if "X" not in self._dev:
            return np.zeros((3 * self.num_element_occupy, self.L), dtype=np.complex128)
        return self._np("X", lambda: self._dev["X"].cpu().numpy())

    @property
    def P(self):
        if not self.converge:
            return np.zeros((self.L, self.num_element_occupy, 3), dtype=np.complex128)
        return self._np("P", lambda: self.X.T.reshape(self.L, self.num_element_occupy, 3))

    @property
    def E(self):
        if not self.converge:
            return np.zeros((self.L, self.num_element_occupy, 3), dtype=np.complex128)
        return self._np("E", lambda: self.P * (4 * np.pi) / ((self.eper_r[np.newaxis] - 1) * self.element_vol))

    # ---- observables ---------------------------------------------------------------
    def observables(self) -> np.ndarray:
        """(L, 12) = C_abs, C_ext, S_fw_theta (re, im), S_fw_phi, S_bk_theta, S_bk_phi, S_bk.

        Computed in one pass on the GPU from the solution.  Like the
        reference, a solve that did not converge leaves P = E = 0.
        """
        if self._obs is None and "obs" in self._dev:   # from the fused solve (zeros if not converged)
            self._obs = self._dev["obs"].cpu().numpy()
        if self._obs is None:
            lib = _lib.load()
            N, L = self.num_element_occupy, self.L
            X = self._dev.get("X") if self.converge else None
            if X is None:
                X = torch.zeros((3 * N, L), dtype=torch.complex128, device=self.device)
            out = torch.empty((L, 12), dtype=torch.float64, device=self.device)
            work = torch.empty(max(int(lib.bdda_observables_workspace_bytes(L)), 16), dtype=torch.uint8,
                               device=self.device)
            _lib.check(lib.bdda_observables(N, L, float(self.k), float(self.lattice_lf), self._absorbing(),
                                            ptr(self._geometry_to_device()), ptr(self._dev_array("eper")), ptr(X),
                                            ptr(self._geometry_vectors()), ptr(self._dev["e0"]), ptr(out),
                                            ptr(work), stream_ptr(self.device)), "bdda_observables")
            self._obs = out.cpu().numpy()
        return self._obs

    def compute_C_abs(self):
        self.C_abs = self.observables()[:, 0].copy()
        return self.C_abs

    def compute_C_ext(self):
        self.C_ext = self.observables()[:, 1].copy()
        return self.C_ext

    def compute_PCAS_observable_S_fw(self):
        o = self.observables()
        self.S_fw_PCAS_theta = o[:, 2] + 1j * o[:, 3]
        self.S_fw_PCAS_phi = o[:, 4] + 1j * o[:, 5]
        return self.S_fw_PCAS_theta, self.S_fw_PCAS_phi

    def compute_OCBS_observable_S_bk(self):
        o = self.observables()
        self.S_bk_OCBS_theta = o[:, 6] + 1j * o[:, 7]
        self.S_bk_OCBS_phi = o[:, 8] + 1j * o[:, 9]
        self.S_bk_OCBS = o[:, 10] + 1j * o[:, 11]
        return self.S_bk_OCBS


def solve_matrix_equations(dds, X0s=None, precision=None, graph=True):
    """``solve_matrix_equation`` for many ``DiscreteDipoles`` in one batched call.

    No counterpart in the reference, which solves one particle, wavelength
    and orientation block at a time (run_dda.py:56-65).  Every object must
    have had ``set_interaction_matrix()``; they may differ in lattice,
    wavelength and refractive index but share L (8, 16, 32 or 64), ``tol``
    and ``itermax``.  Block-BiCGSTAB (the reference's solver) through
    ``bl_krylov.bl_bicgstab_jacobi_mvp_fft_batch``; ``precision`` as there
    (default: each object's ``precision``, which must agree).  Sets
    ``X``/``P``/``E``, ``iter_fin``, ``err_fin`` and ``converge`` of each.
    """
    dds = list(dds)
    if not dds:
        return
    tols = {float(d.tol) for d in dds}
    itms = {int(d.itermax) for d in dds}
    if len(tols) != 1 or len(itms) != 1:
        raise ValueError("batched objects must share tol and itermax")
    if precision is None:
        precs = {d.precision for d in dds}
        if len(precs) != 1:
            raise ValueError("batched objects must share precision")
        precision = precs.pop()
    probs = []
    for i, d in enumerate(dds):
        if d.Au_til is None:
            raise ValueError("call set_interaction_matrix() first")
        d._materialize()
        p = (d.lattice_n, d._dev["occ"], d.Au_til, d._dev["diag"], d._dev["B"])
        x0 = None if X0s is None else X0s[i]
        probs.append(p if x0 is None else p + (x0,))
    start = time.time()
    res = bl_krylov.bl_bicgstab_jacobi_mvp_fft_batch(probs, tols.pop(), itms.pop(), precision=precision,
                                                     graph=graph)
    for d, (X, it, err) in zip(dds, res):
        d.iter_fin, d.err_fin = it, err
        d._dev["X"] = X
        d._dev.pop("obs", None)
        d._host.pop("X", None)
        d._obs = None
        d.converge = bool(err < d.tol)
    if DiscreteDipoles.verbose:
        print("batched block-BiCGStab: %d problems, %d converged, solver time=%.1fs"
              % (len(dds), sum(d.converge for d in dds), time.time() - start))
