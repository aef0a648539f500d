"""Seeded inputs of the workloads: lattice geometry records and orientations.

Geometry records (``.npz``) hold what the reference's shape model produces
for one particle (shape_model/gaussian_ellipsoid.py:150-237): the lattice
size, spacing, the three axis coordinate arrays (np.arange(-lim, lim, lf)),
and the occupancy mask packed to bits.  They are generated once from the
reference and shipped as data, so the GPU path and the oracle see identical
dipoles.
"""
from __future__ import annotations

import numpy as np


def so3_euler(L: int, seed: int) -> np.ndarray:
    """SO(3)-uniform ZYZ Euler angles (L, 3): alpha, gamma ~ U[0, 2pi), beta = arccos U[-1, 1].

    Drawn in the column order alpha, beta, gamma from ``default_rng(seed)``.
    """
    rng = np.random.default_rng(seed)
    a = rng.uniform(0.0, 2 * np.pi, L)
    b = np.arccos(rng.uniform(-1.0, 1.0, L))
    g = rng.uniform(0.0, 2 * np.pi, L)
    return np.column_stack([a, b, g])


def load_geometry(path: str) -> dict:
    """Read a geometry record; adds ``is_in`` (bool, Nc), ``address`` and ``grid``."""
    with np.load(path, allow_pickle=False) as z:
        rec = {k: z[k] for k in z.files}
    n = [int(v) for v in rec["lattice_n"]]
    nc = int(rec["n_cells"])
    is_in = np.unpackbits(rec["mask_bits"])[:nc].astype(bool)
    rec["is_in"] = is_in
    rec["address"] = np.where(is_in)[0]
    rec["lattice_n"] = np.array(n)
    rec["lattice_lf"] = float(rec["lattice_lf"])
    rec["grid"] = lattice_points(rec["x_axis"], rec["y_axis"], rec["z_axis"])
    return rec


def lattice_points(x_axis, y_axis, z_axis) -> np.ndarray:
    """(Nx*Ny*Nz, 3) cell centres in C order, as the reference's meshgrid ravel."""
    X, Y, Z = np.meshgrid(x_axis, y_axis, z_axis, indexing="ij")
    return np.column_stack([X.ravel(), Y.ravel(), Z.ravel()])


def lattice_index(address, n) -> np.ndarray:
    """Integer (ix, iy, iz) of each occupied cell address."""
    address = np.asarray(address, dtype=np.int64)
    ny, nz = int(n[1]), int(n[2])
    return np.column_stack([address // (ny * nz), (address // nz) % ny, address % nz])
