"""Gaussian-random-ellipsoid (GRE) particles on a cubic dipole lattice.

Input generation for the batched sweeps and the warm-start training data: a
restatement of the reference's GRE shape model (shape_model/
gaussian_ellipsoid.py:73-237, after Muinonen & Pieniluoma 2011, JQSRT):

1. base ellipsoid with semi-axes a = b ab, b = c bc, c = (r_v^3 / (ab bc^2))^(1/3)
   (gaussian_ellipsoid.py:95-98);
2. a Gaussian random field s on a (theta, phi) grid of the base surface with
   covariance beta^2 exp(-|r_i - r_j|^2 / (2 lc^2)), lc = 0.3 c, drawn with
   numpy's multivariate_normal(method="eigh") (:100-121), interpolated by a
   bicubic spline onto a finer grid (:123-131);
3. the surface displaced along the base normal by h0 (exp(s) - beta^2/2 - 1),
   h0 = c^2 / a (:133-142);
4. the enclosing cuboid lattice np.arange(-lim, lim, lf) per axis, lim the
   largest |coordinate| plus lf (:150-180);
5. cells within distance_factor lf of the surface points are "near"; a cell
   is inside when, along each of the three axes, near cells lie on both sides
   of it, the near cell itself excluded (:183-237).

The draws of step 2 consume the generator exactly as the reference does, so a
given seed gives the reference's surface.  ``coarse`` lowers the covariance
grid (fewer than the reference's 25 x 100 nodes) for cheap training shapes.
"""
from __future__ import annotations

import numpy as np
import scipy.interpolate
import scipy.spatial


def gre_axes(r_v: float, ab: float, bc: float) -> tuple[float, float, float]:
    c = np.cbrt(r_v ** 3 / (ab * bc ** 2))
    b = c * bc
    return b * ab, b, c


def gre_surface(r_v: float, ab: float, bc: float, beta: float, rng: np.random.Generator,
                coarse: tuple[int, int] = (25, 100)) -> np.ndarray:
    """(N, 3) points on the deformed surface."""
    a, b, c = gre_axes(r_v, ab, bc)
    h0 = c * c / a
    lc = 0.3 * c
    n_t, n_p = coarse
    th = np.linspace(0.0, np.pi, n_t)
    ph = np.linspace(0.0, 2.0 * np.pi, n_p)
    T, P = np.meshgrid(th, ph, indexing="ij")
    nodes = np.stack([a * np.sin(T) * np.cos(P), b * np.sin(T) * np.sin(P), c * np.cos(T)], -1).reshape(-1, 3)
    diff = nodes[:, None, :] - nodes[None, :, :]
    d2 = diff[..., 0] ** 2 + diff[..., 1] ** 2 + diff[..., 2] ** 2
    cov = beta ** 2 * np.exp(-0.5 * d2 / lc ** 2)
    s = rng.multivariate_normal(np.zeros(nodes.shape[0]), cov, size=1, method="eigh").reshape(n_t, n_p)
    spline = scipy.interpolate.RectBivariateSpline(th, ph, s)
    k = int(4 * np.cbrt(bc * ab))
    th2 = np.linspace(0.0, np.pi, k * n_t)
    ph2 = np.linspace(0.0, 2.0 * np.pi, k * n_p)
    s2 = spline(th2, ph2)
    T2, P2 = np.meshgrid(th2, ph2, indexing="ij")
    base = np.stack([a * np.sin(T2) * np.cos(P2), b * np.sin(T2) * np.sin(P2), c * np.cos(T2)], -1)
    normal = base / np.array([a * a, b * b, c * c])
    normal /= np.linalg.norm(normal, axis=-1, keepdims=True)
    shift = h0 * (np.exp(s2) - 0.5 * beta ** 2 - 1.0)
    return (base + shift[..., None] * normal).reshape(-1, 3)


def inside_mask(near: np.ndarray) -> np.ndarray:
    """Cells with near cells on both sides along every axis, the near cell itself excluded."""
    ni = near.astype(np.int32)
    inside = np.ones(near.shape, dtype=bool)
    for ax in range(3):
        fwd = np.cumsum(ni, axis=ax) - ni
        rev = np.flip(np.cumsum(np.flip(ni, ax), axis=ax), ax) - ni
        inside &= (fwd >= 1) & (rev >= 1)
    return inside


def reference_spacing(r_v_base: float, bc: float, ab: float) -> tuple[float, float]:
    """Default lattice spacing and near-surface distance factor of the reference's
    shape model for these axes (gaussian_ellipsoid.py:64-70)."""
    c = np.cbrt(r_v_base ** 3 / (ab * bc ** 2))
    lf = (1 / 75) * np.sqrt(c / 0.05) * (ab * bc) ** (1 / 5)
    dfac = 3 ** 0.5 / 2 * (bc * ab * (c / 0.1)) ** (1 / 6)
    return float(lf), float(dfac)


def gre_name(r_v_base: float, ab: float, bc: float, beta: float) -> str:
    """The reference's shape name string (gaussian_ellipsoid.py:86-89)."""
    return ("GRE_shape__r_v_base={:.2f}um__ab_ratio={:.1f}"
            "__bc_ratio={:.1f}__beta={:.2f}".format(r_v_base, ab, bc, beta))


def lattice_axes(surf: np.ndarray, lf: float) -> list[np.ndarray]:
    """Cell centres per axis of the cuboid enclosing the surface (gaussian_ellipsoid.py:150-180)."""
    lim = np.max(np.abs(surf), axis=0) + lf
    return [np.arange(-lim[i], lim[i], lf) for i in range(3)]


def gre_geometry(r_v_base: float, bc: float, ab: float, beta: float, seed: int, lattice_lf: float | None = None,
                 mask_fn=None, workers: int = -1) -> dict:
    """The reference's geometry pipeline for one shape (run_dda.py:21-35).

    Same arguments and defaults as ``gaussian_ellipsoid_shape_model(r_v_base,
    bc_ratio, ab_ratio, beta)`` followed by the surface draw from
    ``default_rng(seed)``, the enclosing lattice, the nearest-surface distance
    and the three-axis inside test.  ``lattice_lf`` overrides the default
    spacing.  ``mask_fn(axes, surf, thr) -> inside (Nx, Ny, Nz) bool`` decides
    the occupied cells (default: a k-d tree and cumulative sums on the host;
    :func:`bdda_b200.geometry.inside_from_gpu` runs both on the GPU).  Returns
    ``name, lattice_n, lattice_lf, x_axis, y_axis, z_axis, is_in, address,
    grid, r_ve``.
    """
    lf0, dfac = reference_spacing(r_v_base, bc, ab)
    lf = lf0 if lattice_lf is None else float(lattice_lf)
    rng = np.random.default_rng(seed)
    surf = gre_surface(r_v_base, ab, bc, beta, rng)
    axes = lattice_axes(surf, lf)
    n = np.array([len(v) for v in axes], dtype=np.int64)
    thr = dfac * lf
    if mask_fn is None:
        is_in = inside_mask(host_near_surface(axes, surf, thr, workers)).ravel()
    else:
        is_in = np.asarray(mask_fn(axes, surf, thr), dtype=bool).ravel()
    X, Y, Z = np.meshgrid(*axes, indexing="ij")
    grid = np.column_stack([X.ravel(), Y.ravel(), Z.ravel()])
    n_in = int(is_in.sum())
    return dict(name=gre_name(r_v_base, ab, bc, beta), lattice_n=n, lattice_lf=lf, x_axis=axes[0],
                y_axis=axes[1], z_axis=axes[2], is_in=is_in, address=np.flatnonzero(is_in), grid=grid,
                r_ve=float(np.cbrt(3.0 * lf ** 3 * n_in / (4 * np.pi))))


def host_near_surface(axes, surf: np.ndarray, thr: float, workers: int = -1) -> np.ndarray:
    """Cells whose centre lies closer than ``thr`` to a surface point (k-d tree, host)."""
    X, Y, Z = np.meshgrid(*axes, indexing="ij")
    grid = np.column_stack([X.ravel(), Y.ravel(), Z.ravel()])
    dist, _ = scipy.spatial.cKDTree(surf).query(grid, k=1, distance_upper_bound=thr, workers=workers)
    return (dist < thr).reshape(tuple(len(v) for v in axes))


def gre_particle(x: float, ab: float, bc: float, beta: float, seed: int, wl_0: float = 1.0, m_m: float = 1.0,
                 ppl: float = 16.0, coarse: tuple[int, int] = (25, 100), workers: int = -1,
                 mask_fn=None) -> dict:
    """GRE of size parameter x = 2 pi r_v / lambda_m on a lattice of spacing lambda_m / ppl.

    Returns a geometry record like :func:`bdda_b200.inputs.load_geometry`:
    ``lattice_n``, ``lattice_lf``, the axis arrays, ``is_in``, ``address``,
    ``grid`` (cell centres) plus the shape parameters.  ``workers``: threads
    of the nearest-surface query (-1: all cores); ``mask_fn`` as for
    :func:`gre_geometry` (the GPU decides the occupied cells).
    """
    lam = wl_0 / m_m
    r_v = x * lam / (2.0 * np.pi)
    lf = lam / ppl
    rng = np.random.default_rng(seed)
    surf = gre_surface(r_v, ab, bc, beta, rng, coarse)
    lim = np.max(np.abs(surf), axis=0) + lf
    axes = [np.arange(-lim[i], lim[i], lf) for i in range(3)]
    n = np.array([len(v) for v in axes], dtype=np.int64)
    X, Y, Z = np.meshgrid(*axes, indexing="ij")
    grid = np.column_stack([X.ravel(), Y.ravel(), Z.ravel()])
    a, b, c = gre_axes(r_v, ab, bc)
    dfac = np.sqrt(3.0) / 2.0 * (bc * ab * (c / 0.1)) ** (1.0 / 6.0)
    thr = dfac * lf
    if mask_fn is None:
        dist, _ = scipy.spatial.cKDTree(surf).query(grid, k=1, distance_upper_bound=thr, workers=workers)
        is_in = inside_mask((dist < thr).reshape(tuple(n))).ravel()
    else:
        is_in = np.asarray(mask_fn(axes, surf, thr), dtype=bool).ravel()
    return dict(lattice_n=n, lattice_lf=float(lf), x_axis=axes[0], y_axis=axes[1], z_axis=axes[2],
                is_in=is_in, address=np.flatnonzero(is_in), grid=grid, wl_0=float(wl_0), m_m=float(m_m),
                x=float(x), ab=float(ab), bc=float(bc), beta=float(beta), seed=int(seed))
