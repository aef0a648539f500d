// Solver state and the one-CTA L x L step bodies of block-BiCGSTAB, shared
// by the one-problem solver (bdda_solver.cu) and the batched solver
// (bdda_batch.cu).
#pragma once
#include "bdda_blas.cuh"
#include "bdda_small.cuh"

namespace bdda {

constexpr int kSmallMats = 16;

struct SolverState {
  double2 zeta, negzeta;
  double red[4];
  double bnorm;
  double err;
  int bad;      // 1: zero pivot (singular small system), 2: non-finite values
  int iter;     // iterations done (the graph-driven loop's counter)
};

// ---- one-CTA step kernels -------------------------------------------------------
struct SmallPtrs {
  double2 *g2, *lu, *alpha, *negalpha, *beta, *tmp, *xi, *tau, *qq, *rinv, *alphaxi, *r;
  int* piv;
};

__host__ __device__ inline SmallPtrs small_ptrs(unsigned char* base) {
  double2* m = reinterpret_cast<double2*>(base);
  const size_t S = (size_t)kMaxL * kMaxL;
  SmallPtrs s;
  s.g2 = m;            // two matrices
  s.lu = m + 2 * S;
  s.alpha = m + 3 * S;
  s.negalpha = m + 4 * S;
  s.beta = m + 5 * S;
  s.tmp = m + 6 * S;   // two matrices
  s.xi = m + 8 * S;
  s.tau = m + 9 * S;
  s.qq = m + 10 * S;
  s.rinv = m + 11 * S;
  s.alphaxi = m + 12 * S;
  s.r = m + 13 * S;
  s.piv = reinterpret_cast<int*>(m + kSmallMats * S);
  return s;
}

__device__ __forceinline__ void flag_nonfinite(const double2* a, int n, SolverState* st) {
  for (int e = threadIdx.x; e < n; e += blockDim.x)
    if (!zfinite(a[e])) atomicCAS(&st->bad, 0, 2);
  __syncthreads();
}

// ||.|| from a sum of squares; optionally the initial residual norm
__device__ __forceinline__ void norm_body(const double* partial, int nblk, SolverState* st, int set_bnorm) {
  double s = 0.0;
  for (int b = threadIdx.x; b < nblk; b += blockDim.x) s += partial[b];
  __shared__ double red[32];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    const double nrm = sqrt(t);
    if (set_bnorm) st->bnorm = nrm;
    st->err = nrm / st->bnorm;
    if (!isfinite(st->err)) atomicCAS(&st->bad, 0, 2);
  }
}

// BiCGSTAB: LU(RV), alpha = RV^-1 (R0^H R)   (bl_krylov.py:166-167)
__device__ __forceinline__ void bicg_alpha_body(const SmallPtrs& s, int L, SolverState* st, double2* sm) {
  double2* a = sm;
  double2* b = sm + L * L;
  __shared__ int piv[kMaxL];
  __shared__ int bad;
  if (threadIdx.x == 0) bad = 0;
  block_copy(a, s.g2, L * L);
  block_copy(b, s.g2 + L * L, L * L);
  __syncthreads();
  lu_factor(a, L, piv, &bad);
  if (!bad) lu_solve(a, piv, L, b, L);
  for (int e = threadIdx.x; e < L * L; e += blockDim.x) {
    s.lu[e] = a[e];
    s.alpha[e] = b[e];
    s.negalpha[e] = make_double2(-b[e].x, -b[e].y);
  }
  for (int e = threadIdx.x; e < L; e += blockDim.x) s.piv[e] = piv[e];
  __syncthreads();
  if (threadIdx.x == 0 && bad == 1) atomicExch(&st->bad, 1);
  if (threadIdx.x == 0 && bad == 2) atomicCAS(&st->bad, 0, 2);
  flag_nonfinite(b, L * L, st);
}

// BiCGSTAB: zeta = tr(Z^H T) / tr(Z^H Z); beta = RV^-1 (-R0^H Z)   (bl_krylov.py:173,184)
__device__ __forceinline__ void bicg_zeta_beta_body(const SmallPtrs& s, int L, const double* dot_partial, int nblk,
                                                    SolverState* st, double2* sm) {
  double2* a = sm;
  double2* b = sm + L * L;
  __shared__ int piv[kMaxL];
  __shared__ double tot[3];
  __shared__ int singular;
  if (threadIdx.x == 0) singular = (st->bad == 1);
  if (threadIdx.x < 3) {
    double acc = 0.0;
    for (int k = 0; k < nblk; ++k) acc += dot_partial[k * 3 + threadIdx.x];
    tot[threadIdx.x] = acc;
  }
  block_copy(a, s.lu, L * L);
  for (int e = threadIdx.x; e < L * L; e += blockDim.x) b[e] = make_double2(-s.g2[e].x, -s.g2[e].y);
  for (int e = threadIdx.x; e < L; e += blockDim.x) piv[e] = s.piv[e];
  __syncthreads();
  if (threadIdx.x == 0) {
    const double2 z = make_double2(tot[0] / tot[2], tot[1] / tot[2]);
    st->zeta = z;
    st->negzeta = make_double2(-z.x, -z.y);
    if (!zfinite(z)) atomicCAS(&st->bad, 0, 2);
  }
  __syncthreads();
  if (!singular) lu_solve(a, piv, L, b, L);
  block_copy(s.beta, b, L * L);
}

}  // namespace bdda
