// GRE lattice occupancy on the GPU: near-surface cells and the three-axis
// inside test of the reference's shape model
// (shape_model/gaussian_ellipsoid.py:182-237).
//
// The reference queries a k-d tree for the distance of every lattice cell to
// the nearest surface point and marks a cell "near" when that distance is
// below distance_factor * lattice_lf; a cell is inside when, along each of
// the three axes, a near cell lies strictly before it and one strictly after
// it (cumulative sums along the axis minus the cell itself, both >= 1).
//
// Here the surface points arrive sorted into a uniform grid of bins whose
// edge h is at least the threshold, so a point closer than the threshold lies
// in the cell's bin or one of its 26 neighbours.  One thread per lattice cell
// scans those 27 bins and stops at the first point within the threshold.  The
// distance is evaluated as the k-d tree does, sqrt((dx^2 + dy^2) + dz^2) in
// double precision with separately rounded products and sums (no fused
// multiply-add), so the comparison with the threshold decides exactly as the
// reference's does.  Then, per line along each axis, the first and last near
// index; a cell is inside when it lies strictly between them on all three of
// its lines.  The cell coordinates are the reference's own axis arrays
// (np.arange values), passed in, not recomputed.
#include "bdda_internal.h"

namespace bdda {
namespace {

constexpr int kGeoThreads = 256;

__global__ void near_kernel(int nx, int ny, int nz, const double* __restrict__ xs, const double* __restrict__ ys,
                            const double* __restrict__ zs, const double* __restrict__ pts,
                            const int32_t* __restrict__ bin_start, int nbx, int nby, int nbz, double ox,
                            double oy, double oz, double inv_h, double thr, uint8_t* __restrict__ near) {
  const int64_t nc = (int64_t)nx * ny * nz;
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < nc; c += (int64_t)gridDim.x * blockDim.x) {
    const int k = (int)(c % nz);
    const int64_t ij = c / nz;
    const int j = (int)(ij % ny);
    const int i = (int)(ij / ny);
    const double x = xs[i], y = ys[j], z = zs[k];
    // bin of the cell; a point within thr <= h is at most one bin away per
    // axis (clamped first: cells far outside the bins find nothing)
    const int bx = (int)fmin(fmax(floor((x - ox) * inv_h), -2.0), (double)nbx + 1.0);
    const int by = (int)fmin(fmax(floor((y - oy) * inv_h), -2.0), (double)nby + 1.0);
    const int bz = (int)fmin(fmax(floor((z - oz) * inv_h), -2.0), (double)nbz + 1.0);
    uint8_t hit = 0;
    for (int u = max(bx - 1, 0); u <= min(bx + 1, nbx - 1) && !hit; ++u) {
      for (int v = max(by - 1, 0); v <= min(by + 1, nby - 1) && !hit; ++v) {
        const int64_t row = ((int64_t)u * nby + v) * nbz;
        const int w0 = max(bz - 1, 0), w1 = min(bz + 1, nbz - 1);
        if (w0 > w1) continue;
        // bins w0..w1 of this (u, v) row are contiguous in the sorted points
        const int p0 = bin_start[row + w0], p1 = bin_start[row + w1 + 1];
        for (int p = p0; p < p1; ++p) {
          const double dx = __dsub_rn(x, pts[3 * (int64_t)p]);
          const double dy = __dsub_rn(y, pts[3 * (int64_t)p + 1]);
          const double dz = __dsub_rn(z, pts[3 * (int64_t)p + 2]);
          const double d2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
          if (sqrt(d2) < thr) { hit = 1; break; }
        }
      }
    }
    near[c] = hit;
  }
}

// First and last near index along one axis for every line of that axis.
// axis 0: lines (j, k), index i; axis 1: lines (i, k), index j; axis 2: lines (i, j), index k.
__global__ void line_extent_kernel(int nx, int ny, int nz, int axis, const uint8_t* __restrict__ near,
                                   int2* __restrict__ ext) {
  const int n_ax = axis == 0 ? nx : axis == 1 ? ny : nz;
  const int64_t lines = (int64_t)nx * ny * nz / n_ax;
  for (int64_t l = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; l < lines; l += (int64_t)gridDim.x * blockDim.x) {
    int64_t base, stride;
    if (axis == 0) {        // l = j * nz + k
      base = l;
      stride = (int64_t)ny * nz;
    } else if (axis == 1) {  // l = i * nz + k
      const int64_t i = l / nz, k = l % nz;
      base = i * (int64_t)ny * nz + k;
      stride = nz;
    } else {                 // l = i * ny + j
      base = l * nz;
      stride = 1;
    }
    int first = n_ax, last = -1;
    for (int t = 0; t < n_ax; ++t) {
      if (near[base + t * stride]) {
        if (first == n_ax) first = t;
        last = t;
      }
    }
    ext[l] = make_int2(first, last);
  }
}

__global__ void inside_kernel(int nx, int ny, int nz, const int2* __restrict__ ex, const int2* __restrict__ ey,
                              const int2* __restrict__ ez, uint8_t* __restrict__ inside) {
  const int64_t nc = (int64_t)nx * ny * nz;
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < nc; c += (int64_t)gridDim.x * blockDim.x) {
    const int k = (int)(c % nz);
    const int64_t ij = c / nz;
    const int j = (int)(ij % ny);
    const int i = (int)(ij / ny);
    const int2 a = ex[(int64_t)j * nz + k], b = ey[(int64_t)i * nz + k], d = ez[ij];
    inside[c] = (a.x < i && i < a.y && b.x < j && j < b.y && d.x < k && k < d.y) ? 1 : 0;
  }
}

int grid_for(int64_t n) {
  const int64_t blocks = (n + kGeoThreads - 1) / kGeoThreads;
  return (int)(blocks < 148 * 16 ? (blocks > 0 ? blocks : 1) : 148 * 16);
}

}  // namespace
}  // namespace bdda

using namespace bdda;

extern "C" {

size_t bdda_gre_occupancy_workspace_bytes(int nx, int ny, int nz) {
  if (nx < 1 || ny < 1 || nz < 1) return 0;
  return sizeof(int2) * ((size_t)ny * nz + (size_t)nx * nz + (size_t)nx * ny);
}

int bdda_gre_occupancy(int nx, int ny, int nz, const double* xs, const double* ys, const double* zs, int npts,
                       const double* pts, const int32_t* bin_start, int nbx, int nby, int nbz, double ox,
                       double oy, double oz, double h, double thr, uint8_t* near, uint8_t* inside, void* work,
                       size_t work_bytes, void* stream) {
  if (nx < 1 || ny < 1 || nz < 1 || npts < 0 || nbx < 1 || nby < 1 || nbz < 1 || !(h > 0.0) ||
      !(thr >= 0.0) || thr > h || !xs || !ys || !zs || !bin_start || !near || !inside || (npts > 0 && !pts))
    return BDDA_BAD_ARG;
  if (!work || work_bytes < bdda_gre_occupancy_workspace_bytes(nx, ny, nz)) return BDDA_NO_WORKSPACE;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int64_t nc = (int64_t)nx * ny * nz;
  near_kernel<<<grid_for(nc), kGeoThreads, 0, st>>>(nx, ny, nz, xs, ys, zs, pts, bin_start, nbx, nby, nbz, ox, oy,
                                                    oz, 1.0 / h, thr, near);
  BDDA_CUDA_TRY(cudaGetLastError());
  int2* ex = static_cast<int2*>(work);
  int2* ey = ex + (size_t)ny * nz;
  int2* ez = ey + (size_t)nx * nz;
  line_extent_kernel<<<grid_for((int64_t)ny * nz), kGeoThreads, 0, st>>>(nx, ny, nz, 0, near, ex);
  line_extent_kernel<<<grid_for((int64_t)nx * nz), kGeoThreads, 0, st>>>(nx, ny, nz, 1, near, ey);
  line_extent_kernel<<<grid_for((int64_t)nx * ny), kGeoThreads, 0, st>>>(nx, ny, nz, 2, near, ez);
  inside_kernel<<<grid_for(nc), kGeoThreads, 0, st>>>(nx, ny, nz, ex, ey, ez, inside);
  BDDA_CUDA_TRY(cudaGetLastError());
  count_launch(5);
  return BDDA_OK;
}

}  // extern "C"
