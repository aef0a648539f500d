"""Parameter sweeps with resumable result shards (the reference's run_dda.py).

The reference's driver (run_dda.py:74-146) walks the product of shapes
(r_v_base x bc x ab x beta), (wl_0, m_m) pairs and particle indices m_p, and
for every condition

* builds the GRE lattice once per shape with ``default_rng(RNG_SEED)``
  (run_dda.py:21-35);
* solves up to ``MAX_TRY`` times, each try with fresh Euler angles from one
  ``default_rng(RNG_SEED + 1)`` per condition (alpha, gamma ~ U[0, 2 pi),
  beta ~ U[0, pi), drawn in that order; run_dda.py:38-70), keeping the first
  try that converges, else NaN observables with the last try's angles;
* writes C_abs, C_ext, S_fw (theta, phi), S_bk per orientation, the angles,
  r_ve and the Mie values of the volume-equivalent sphere into an HDF5 file
  of 7-D arrays [pair, m_p, r_v, bc, ab, beta, orientation] (layout:
  dda_results/create_h5py.ipynb), skipping conditions already written
  (run_dda.py:102-105).

Here each condition goes to its own ``.npz`` shard (h5py is not part of
this stack), written to a temporary name and renamed, so an interrupted
sweep leaves only whole shards and resumes by skipping them; a shard is
written for a condition that failed every try too (NaN observables), as the
reference marks those done.  :func:`load_results` assembles the shards into
the reference's 7-D arrays.  The solves run on the GPU; all conditions of a
shape that share a try are solved together (one batched block-BiCGSTAB
call, problems grouped by lattice size), the Green's spectrum of each
(wl_0, m_m) is built once per shape and shared by its m_p conditions, and
the lattice can be built on the GPU (:mod:`bdda_b200.geometry`).
"""
from __future__ import annotations

import datetime
import itertools
import os
from dataclasses import dataclass, field

import numpy as np

from .mie import mie_q_and_s
from .shapes import gre_geometry

# per-orientation outputs, with the reference's dataset names
ORIENTATION_KEYS = ("C_abs", "C_ext", "S_fw_PCAS_theta", "S_fw_PCAS_phi", "S_bk_OCBS")
CONDITION_KEYS = ("C_abs_mie", "C_ext_mie", "S_fw_PCAS_mie", "S_bk_OCBS_mie")
COMPLEX_KEYS = ("S_fw_PCAS_theta", "S_fw_PCAS_phi", "S_bk_OCBS", "S_fw_PCAS_mie", "S_bk_OCBS_mie")


@dataclass
class SweepSpec:
    """The sweep's parameter lists (the ``target`` group of the reference's file)."""
    wl_m_m_pairs: np.ndarray                      # (N_pairs, 2): wl_0 [um], m_m
    m_p_xyz_list: np.ndarray                      # (N_m_p, 3) complex
    r_v_base_list: np.ndarray
    bc_ratio_list: np.ndarray
    ab_ratio_list: np.ndarray
    gre_beta_list: np.ndarray
    num_orientations: int
    rng_seed: int = 12345                         # run_dda.py:11
    max_try: int = 4                              # run_dda.py:12
    lattice_lf: float | None = None               # None: the shape model's default spacing
    extra: dict = field(default_factory=dict)

    def __post_init__(self):
        self.wl_m_m_pairs = np.asarray(self.wl_m_m_pairs, dtype=np.float64).reshape(-1, 2)
        self.m_p_xyz_list = np.asarray(self.m_p_xyz_list, dtype=np.complex128).reshape(-1, 3)
        for name in ("r_v_base_list", "bc_ratio_list", "ab_ratio_list", "gre_beta_list"):
            setattr(self, name, np.asarray(getattr(self, name), dtype=np.float64).ravel())
        self.num_orientations = int(self.num_orientations)

    @property
    def shape_geo(self):
        return (len(self.r_v_base_list), len(self.bc_ratio_list), len(self.ab_ratio_list),
                len(self.gre_beta_list))

    @property
    def shape_cond(self):
        return (len(self.wl_m_m_pairs), len(self.m_p_xyz_list)) + self.shape_geo

    def shapes(self):
        """(shape index (i_rv, i_bc, i_ab, i_bt), (r_v_base, bc, ab, beta)) in the reference's loop order."""
        for (i, rv), (j, bc), (k, ab), (m, bt) in itertools.product(
                enumerate(self.r_v_base_list), enumerate(self.bc_ratio_list),
                enumerate(self.ab_ratio_list), enumerate(self.gre_beta_list)):
            yield (i, j, k, m), (float(rv), float(bc), float(ab), float(bt))

    def as_record(self) -> dict:
        return dict(wl_m_m_pairs=self.wl_m_m_pairs, m_p_xyz_list=self.m_p_xyz_list,
                    r_v_base_list=self.r_v_base_list, bc_ratio_list=self.bc_ratio_list,
                    ab_ratio_list=self.ab_ratio_list, gre_beta_list=self.gre_beta_list,
                    num_orientations=self.num_orientations, rng_seed=self.rng_seed, max_try=self.max_try,
                    lattice_lf=np.nan if self.lattice_lf is None else self.lattice_lf)

    def same_as(self, rec: dict) -> bool:
        mine = self.as_record()
        return all(np.array_equal(np.asarray(mine[k]), np.asarray(rec[k]), equal_nan=True) for k in mine)


def euler_tries(num_orientations: int, seed: int, max_try: int) -> list[np.ndarray]:
    """The angles of each try of one condition (run_dda.py:45-53): one generator, L draws per column."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(max_try):
        a = rng.uniform(0, 2 * np.pi, num_orientations)
        b = rng.uniform(0, np.pi, num_orientations)
        g = rng.uniform(0, 2 * np.pi, num_orientations)
        out.append(np.column_stack([a, b, g]))
    return out


def shard_name(idx6) -> str:
    return "cond_p%d_m%d_r%d_b%d_a%d_t%d.npz" % tuple(int(i) for i in idx6)


def _log(msg: str) -> None:
    print(f"[{datetime.datetime.now():%H:%M:%S}] {msg}", flush=True)


def gpu_solve(items, tol=None, itermax=None, precision=None, batched=True):
    """Solve conditions on the GPU: ``items`` = [(target, wl_0, m_m, euler)].

    Returns one ``(converged, obs)`` per item, obs the (L, 12) observables of
    ``DiscreteDipoles.observables``.  Items with the same (wl_0, m_m) on the
    same lattice share one Green's spectrum; with ``batched`` all are solved
    by one batched block-BiCGSTAB call when L is 8, 16, 32 or 64.
    """
    from bl_dda import scatterer as sc
    dds, greens = [], {}
    for target, wl_0, m_m, euler in items:
        d = sc.DiscreteDipoles(target, sc.IncidentField(wl_0, m_m, euler))
        if tol is not None:
            d.tol = tol
        if itermax is not None:
            d.itermax = itermax
        d.precision = precision
        key = (id(target.lattice_grid_points), float(wl_0), float(m_m), float(target.lattice_lf))
        d.set_interaction_matrix(green=greens.get(key))
        greens[key] = d.Au_til
        dds.append(d)
    L = dds[0].L if dds else 0
    if batched and len(dds) > 1 and L in (8, 16, 32, 64):
        sc.solve_matrix_equations(dds)
    else:
        for d in dds:
            d.solve_matrix_equation()
    return [(bool(d.converge), d.observables().copy(), int(d.iter_fin)) for d in dds]


class Sweep:
    """Run (or resume) a sweep into ``out_dir``.

    ``solve(items) -> [(converged, obs (L, 12), iter_fin)]`` solves a list of
    conditions (default :func:`gpu_solve`; tests pass a stand-in).
    ``mask_fn`` decides the occupied cells of a lattice (default: host k-d
    tree; :func:`bdda_b200.geometry.inside_from_gpu` on the GPU).
    """

    def __init__(self, spec: SweepSpec, out_dir: str, solve=None, mask_fn=None, tol=None, itermax=None,
                 precision=None, batched=True, verbose=True):
        self.spec = spec
        self.out_dir = out_dir
        self.mask_fn = mask_fn
        self.verbose = verbose
        if solve is None:
            def solve(items):
                return gpu_solve(items, tol=tol, itermax=itermax, precision=precision, batched=batched)
        self.solve = solve
        os.makedirs(out_dir, exist_ok=True)
        spec_path = os.path.join(out_dir, "sweep_spec.npz")
        if os.path.exists(spec_path):
            with np.load(spec_path, allow_pickle=False) as z:
                if not spec.same_as({k: z[k] for k in z.files}):
                    raise ValueError("%s holds a sweep with other parameters" % out_dir)
        else:
            _atomic_savez(spec_path, spec.as_record())

    def done(self, idx6) -> bool:
        return os.path.exists(os.path.join(self.out_dir, shard_name(idx6)))

    def pending(self) -> list[tuple]:
        P, M = self.spec.shape_cond[:2]
        return [(p, m) + s for s, _ in self.spec.shapes() for p in range(P) for m in range(M)
                if not self.done((p, m) + s)]

    def run(self, max_conditions: int | None = None) -> int:
        """Solve every pending condition (at most ``max_conditions``); returns how many were written."""
        spec = self.spec
        written = 0
        tries = euler_tries(spec.num_orientations, spec.rng_seed + 1, spec.max_try)
        for sidx, (rv, bc, ab, bt) in spec.shapes():
            todo = [(p, m) for p in range(len(spec.wl_m_m_pairs)) for m in range(len(spec.m_p_xyz_list))
                    if not self.done((p, m) + sidx)]
            if max_conditions is not None:
                todo = todo[:max(0, max_conditions - written)]
            if not todo:
                if self.verbose:
                    _log("Skip: shape=%s (all conditions computed)" % (sidx,))
                continue
            geo = gre_geometry(rv, bc, ab, bt, spec.rng_seed, lattice_lf=spec.lattice_lf, mask_fn=self.mask_fn)
            written += self._run_shape(sidx, geo, todo, tries)
            if max_conditions is not None and written >= max_conditions:
                break
        return written

    def _run_shape(self, sidx, geo, todo, tries) -> int:
        from bl_dda.scatterer import Target
        spec = self.spec
        targets = {m: Target(geo["name"], geo["lattice_n"], geo["lattice_lf"], geo["grid"], geo["is_in"],
                             spec.m_p_xyz_list[m]) for m in {m for _, m in todo}}
        left = list(todo)
        result = {}
        for i_try, euler in enumerate(tries, 1):
            if not left:
                break
            items = [(targets[m], float(spec.wl_m_m_pairs[p, 0]), float(spec.wl_m_m_pairs[p, 1]), euler)
                     for p, m in left]
            sols = self.solve(items)
            nxt = []
            for (p, m), (conv, obs, it) in zip(left, sols):
                if self.verbose:
                    _log("    pair=%d m_p=%d shape=%s try %d/%d: %s (iter_fin=%d)"
                         % (p, m, sidx, i_try, spec.max_try, "converged" if conv else "not converged", it))
                if conv:
                    result[(p, m)] = (euler, obs, True, i_try)
                else:
                    result[(p, m)] = (euler, None, False, i_try)
                    nxt.append((p, m))
            left = nxt
        for (p, m), (euler, obs, conv, i_try) in result.items():
            self._write((p, m) + sidx, geo, euler, obs, conv, i_try)
        return len(result)

    def _write(self, idx6, geo, euler, obs, converged, tries):
        spec = self.spec
        p, m = idx6[:2]
        wl_0, m_m = (float(v) for v in spec.wl_m_m_pairs[p])
        L = spec.num_orientations
        if converged:
            out = {"C_abs": obs[:, 0], "C_ext": obs[:, 1], "S_fw_PCAS_theta": obs[:, 2] + 1j * obs[:, 3],
                   "S_fw_PCAS_phi": obs[:, 4] + 1j * obs[:, 5], "S_bk_OCBS": obs[:, 10] + 1j * obs[:, 11]}
        else:   # run_dda.py:68-70
            out = {k: np.full(L, np.nan + (0j if k in COMPLEX_KEYS else 0.0)) for k in ORIENTATION_KEYS}
        r_ve = geo["r_ve"]
        m_p_avg = complex(np.mean(spec.m_p_xyz_list[m]))
        _, q_abs, q_ext, s_fw, s_bk = mie_q_and_s(wl_0, m_m, r_ve, m_p_avg)
        out.update(C_abs_mie=q_abs * np.pi * r_ve ** 2, C_ext_mie=q_ext * np.pi * r_ve ** 2,
                   S_fw_PCAS_mie=s_fw, S_bk_OCBS_mie=s_bk)
        out.update(Euler_angles=euler, r_ve=r_ve, converged=converged, tries=tries, idx6=np.array(idx6),
                   wl_0=wl_0, m_m=m_m, m_p_xyz=spec.m_p_xyz_list[m], shape_name=geo["name"],
                   lattice_n=geo["lattice_n"], lattice_lf=geo["lattice_lf"], n_dipoles=geo["address"].size)
        _atomic_savez(os.path.join(self.out_dir, shard_name(idx6)), out)
        if self.verbose:
            vals = " ".join("%s(mean)=%.4g" % (k, np.nanmean(out[k]).real) for k in ORIENTATION_KEYS[1:])
            _log("  wrote %s: %s" % (shard_name(idx6), vals))


def _atomic_savez(path: str, rec: dict) -> None:
    tmp = path + ".part.npz"
    np.savez(tmp, **rec)
    os.replace(tmp, path)


def load_results(out_dir: str) -> dict:
    """The shards of a sweep as the reference's 7-D datasets (``simulated_data``).

    Returns the parameter lists plus ``r_ve`` (shape_geo), ``Euler_angles``
    (shape_cond + (L, 3)), the per-orientation datasets (shape_cond + (L,)),
    the Mie datasets (shape_cond) and ``done`` (shape_cond, bool).  Conditions
    without a shard hold NaN.
    """
    with np.load(os.path.join(out_dir, "sweep_spec.npz"), allow_pickle=False) as z:
        rec = {k: z[k] for k in z.files}
    spec = SweepSpec(rec["wl_m_m_pairs"], rec["m_p_xyz_list"], rec["r_v_base_list"], rec["bc_ratio_list"],
                     rec["ab_ratio_list"], rec["gre_beta_list"], int(rec["num_orientations"]),
                     int(rec["rng_seed"]), int(rec["max_try"]))
    sc, L = spec.shape_cond, spec.num_orientations
    out = dict(spec.as_record())
    out["r_ve"] = np.full(spec.shape_geo, np.nan)
    out["Euler_angles"] = np.full(sc + (L, 3), np.nan)
    for k in ORIENTATION_KEYS:
        out[k] = np.full(sc + (L,), np.nan + (0j if k in COMPLEX_KEYS else 0.0))
    for k in CONDITION_KEYS:
        out[k] = np.full(sc, np.nan + (0j if k in COMPLEX_KEYS else 0.0))
    out["done"] = np.zeros(sc, dtype=bool)
    out["converged"] = np.zeros(sc, dtype=bool)
    for name in os.listdir(out_dir):
        if not (name.startswith("cond_") and name.endswith(".npz")) or name.endswith(".part.npz"):
            continue
        with np.load(os.path.join(out_dir, name), allow_pickle=False) as z:
            idx = tuple(int(i) for i in z["idx6"])
            out["r_ve"][idx[2:]] = float(z["r_ve"])
            out["Euler_angles"][idx] = z["Euler_angles"]
            for k in ORIENTATION_KEYS + CONDITION_KEYS:
                out[k][idx] = z[k]
            out["done"][idx] = True
            out["converged"][idx] = bool(z["converged"])
    return out
