// Tall-skinny block kernels for the block Krylov solvers.
//
// Block vectors are (n, L) row-major complex (n = 3 N_occ rows).  Three
// kernel families cover every non-FFT step of block-BiCGSTAB and
// block-COCG-rq (bl_krylov/bl_krylov.py:98-116, 161-185):
//   gram    G_k = op(A)^T B_k   (op = conj or identity), FP64 accumulation,
//           per-CTA partials + deterministic reduction
//   update  out = a0*Y0 + a1*Y1 + (X1 + c2*X2) M, optional ||out||_F^2
//           (coefficients read from device memory, never from the host)
//   small   one-CTA dense L x L algebra: LU with partial pivoting, Cholesky,
//           triangular inverse, products (bdda_small.cu)
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "bdda_fft.cuh"

namespace bdda {

constexpr int kMaxL = 64;          // right-hand sides per block solve
constexpr int kRedBlocks = 296;    // CTAs of the reduction kernels (2 per SM)

__device__ __forceinline__ double2 to_d2(double2 v) { return v; }
__device__ __forceinline__ double2 to_d2(float2 v) { return make_double2(v.x, v.y); }
template <typename T> __device__ __forceinline__ T from_d2(double2 v);
template <> __device__ __forceinline__ double2 from_d2<double2>(double2 v) { return v; }
template <> __device__ __forceinline__ float2 from_d2<float2>(double2 v) {
  return make_float2((float)v.x, (float)v.y);
}

// block-wide sum of one double per thread; result valid in thread 0
__device__ __forceinline__ double block_sum(double v) {
  __shared__ double red[32];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) red[w] = v;
  __syncthreads();
  v = 0.0;
  if (w == 0) {
    const int nw = (blockDim.x + 31) >> 5;
    v = l < nw ? red[l] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  }
  return v;
}

struct GramArgs {
  int64_t n;
  int L;
  int nB;
  const void* A;
  const void* B[2];
  double2* partial;   // [gridDim.x][nB][L][L]
};

struct UpdateArgs {
  int64_t n;
  int L;
  const void* Y0; const double2* a0;   // a0 == nullptr means 1
  const void* Y1; const double2* a1;
  const void* X1; const void* X2; const double2* c2;
  const double2* M;                    // L x L row-major, nullptr = no product
  void* out;
  double* norm_partial;                // [gridDim.x] sum |out|^2, or nullptr
};

struct DotArgs {
  int64_t n;          // elements (rows * L)
  const void* A;
  const void* B;
  double* partial;    // [gridDim.x][3]: Re sum conj(A) B, Im sum conj(A) B, sum |A|^2
};

// Host-side launchers (bdda_blas.cu)
void set_fixed_blas(int on);
template <typename T> int gram(const GramArgs& g, bool conj, double2* out, cudaStream_t st);
template <typename T> int update(const UpdateArgs& u, cudaStream_t st);
template <typename T> int dots(const DotArgs& d, cudaStream_t st);
// sum of a partial array into out[0..width) (width values per CTA partial)
int reduce_partials(const double* partial, int nblk, int width, double* out, cudaStream_t st);

}  // namespace bdda
