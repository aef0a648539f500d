// One-CTA dense algebra on L x L complex matrices (L <= 64) in shared memory.
//
// These replace the reference's numpy.linalg calls on the small block
// matrices (bl_krylov/bl_krylov.py:92,101,104,113,167,184): LU with partial
// pivoting for solve(), and a Cholesky-based QR for qr().  All threads of
// the CTA must call each routine; matrices are row-major double2.
#pragma once
#include <cuda_runtime.h>

namespace bdda {

__device__ __forceinline__ double2 zmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 zmulc(double2 a, double2 b) {   // conj(a) * b
  return make_double2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ double2 zsub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 zadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 zdiv(double2 a, double2 b) {
  // Smith's algorithm
  if (fabs(b.x) >= fabs(b.y)) {
    const double r = b.y / b.x, d = b.x + r * b.y;
    return make_double2((a.x + a.y * r) / d, (a.y - a.x * r) / d);
  }
  const double r = b.x / b.y, d = b.y + r * b.x;
  return make_double2((a.x * r + a.y) / d, (a.y * r - a.x) / d);
}
__device__ __forceinline__ bool zfinite(double2 a) { return isfinite(a.x) && isfinite(a.y); }

__device__ __forceinline__ void block_copy(double2* dst, const double2* src, int n) {
  for (int e = threadIdx.x; e < n; e += blockDim.x) dst[e] = src[e];
}

// In-place LU with partial pivoting (row interchanges recorded in piv, in
// order).  Pivot choice as LAPACK's izamax: largest |re| + |im|, first on
// ties.  *bad becomes 1 for an exactly zero pivot (singular) and 2 for a
// non-finite one (the matrix holds NaN/Inf).
static __device__ void lu_factor(double2* a, int L, int* piv, int* bad) {
  __shared__ double sbest[32];
  __shared__ int sidx[32];
  for (int k = 0; k < L; ++k) {
    if (threadIdx.x < 32) {
      double best = -1.0;
      int bi = k;
      for (int i = k + threadIdx.x; i < L; i += 32) {
        const double2 v = a[i * L + k];
        const double m = fabs(v.x) + fabs(v.y);
        if (m > best || (m != m)) { best = (m != m) ? INFINITY : m; bi = i; }
      }
      sbest[threadIdx.x] = best;
      sidx[threadIdx.x] = bi;
      __syncwarp();
      if (threadIdx.x == 0) {
        double b = -1.0;
        int id = k;
        for (int w = 0; w < 32; ++w)
          if (sbest[w] > b || (sbest[w] == b && sidx[w] < id)) { b = sbest[w]; id = sidx[w]; }
        piv[k] = id;
        if (!isfinite(b)) *bad = 2;
        else if (!(b > 0.0) && *bad == 0) *bad = 1;
      }
    }
    __syncthreads();
    const int p = piv[k];
    if (p != k)
      for (int j = threadIdx.x; j < L; j += blockDim.x) {
        const double2 t = a[k * L + j];
        a[k * L + j] = a[p * L + j];
        a[p * L + j] = t;
      }
    __syncthreads();
    const double2 d = a[k * L + k];
    if (!(*bad))
      for (int i = k + 1 + threadIdx.x; i < L; i += blockDim.x) a[i * L + k] = zdiv(a[i * L + k], d);
    __syncthreads();
    const int m = L - k - 1;
    for (int e = threadIdx.x; e < m * m; e += blockDim.x) {
      const int i = k + 1 + e / m, j = k + 1 + e % m;
      a[i * L + j] = zsub(a[i * L + j], zmul(a[i * L + k], a[k * L + j]));
    }
    __syncthreads();
  }
}

// b (L x ncol) <- A^-1 b from lu_factor's output
static __device__ void lu_solve(const double2* lu, const int* piv, int L, double2* b, int ncol) {
  for (int k = 0; k < L; ++k) {
    const int p = piv[k];
    if (p != k)
      for (int j = threadIdx.x; j < ncol; j += blockDim.x) {
        const double2 t = b[k * ncol + j];
        b[k * ncol + j] = b[p * ncol + j];
        b[p * ncol + j] = t;
      }
    __syncthreads();
  }
  for (int k = 0; k < L; ++k) {            // unit lower
    const int m = L - k - 1;
    for (int e = threadIdx.x; e < m * ncol; e += blockDim.x) {
      const int i = k + 1 + e / ncol, j = e % ncol;
      b[i * ncol + j] = zsub(b[i * ncol + j], zmul(lu[i * L + k], b[k * ncol + j]));
    }
    __syncthreads();
  }
  for (int k = L - 1; k >= 0; --k) {       // upper
    const double2 d = lu[k * L + k];
    for (int j = threadIdx.x; j < ncol; j += blockDim.x) b[k * ncol + j] = zdiv(b[k * ncol + j], d);
    __syncthreads();
    for (int e = threadIdx.x; e < k * ncol; e += blockDim.x) {
      const int i = e / ncol, j = e % ncol;
      b[i * ncol + j] = zsub(b[i * ncol + j], zmul(lu[i * L + k], b[k * ncol + j]));
    }
    __syncthreads();
  }
}

// Hermitian positive definite g -> upper R with R^H R = g (lower part zeroed).
static __device__ void chol_upper(double2* g, int L, int* bad) {
  for (int k = 0; k < L; ++k) {
    if (threadIdx.x == 0) {
      const double d = g[k * L + k].x;
      if (!isfinite(d)) *bad = 2;
      else if (!(d > 0.0) && *bad == 0) *bad = 1;
      g[k * L + k] = make_double2(sqrt(fmax(d, 0.0)), 0.0);
    }
    __syncthreads();
    const double rkk = g[k * L + k].x;
    if (!(*bad))
      for (int j = k + 1 + threadIdx.x; j < L; j += blockDim.x)
        g[k * L + j] = make_double2(g[k * L + j].x / rkk, g[k * L + j].y / rkk);
    __syncthreads();
    const int m = L - k - 1;
    for (int e = threadIdx.x; e < m * m; e += blockDim.x) {
      const int i = k + 1 + e / m, j = k + 1 + e % m;
      if (j >= i) g[i * L + j] = zsub(g[i * L + j], zmulc(g[k * L + i], g[k * L + j]));
    }
    __syncthreads();
  }
  for (int e = threadIdx.x; e < L * L; e += blockDim.x)
    if (e / L > e % L) g[e] = make_double2(0.0, 0.0);
  __syncthreads();
}

// x <- R^-1 for upper-triangular R (x must not alias r)
static __device__ void tri_upper_inv(const double2* r, int L, double2* x) {
  for (int e = threadIdx.x; e < L * L; e += blockDim.x)
    x[e] = make_double2((e / L == e % L) ? 1.0 : 0.0, 0.0);
  __syncthreads();
  for (int k = L - 1; k >= 0; --k) {
    const double2 d = r[k * L + k];
    for (int j = threadIdx.x; j < L; j += blockDim.x) x[k * L + j] = zdiv(x[k * L + j], d);
    __syncthreads();
    for (int e = threadIdx.x; e < k * L; e += blockDim.x) {
      const int i = e / L, j = e % L;
      x[i * L + j] = zsub(x[i * L + j], zmul(r[i * L + k], x[k * L + j]));
    }
    __syncthreads();
  }
}

// c = op(a) b with op = transpose (TA) or identity; c must not alias a or b
template <bool TA>
static __device__ void small_matmul(const double2* a, const double2* b, double2* c, int L) {
  for (int e = threadIdx.x; e < L * L; e += blockDim.x) {
    const int i = e / L, j = e % L;
    double2 s = make_double2(0.0, 0.0);
    for (int m = 0; m < L; ++m) s = zadd(s, zmul(TA ? a[m * L + i] : a[i * L + m], b[m * L + j]));
    c[e] = s;
  }
  __syncthreads();
}

}  // namespace bdda
