// Tall-skinny block kernels: Gram products, fused block updates, dots.
#include <climits>
#include <type_traits>

#include "bdda_blas.cuh"
#include "bdda_blas_dev.cuh"
#include "bdda_internal.h"

namespace bdda {

// L-specialised Gram / update kernels on (tests switch them off to compare).
static int g_fixed_blas = 1;

// ---- Gram: G_k[i][j] = sum_r op(A[r][i]) B_k[r][j] ---------------------------
template <typename T, bool CONJ, int TM, int NB>
__global__ void __launch_bounds__(256) gram_kernel(GramArgs g) {
  constexpr int RCH = 16;
  const int L = g.L;
  const int nt = (L + TM - 1) / TM;
  const int t = threadIdx.x;
  const int ty = t / nt, tx = t - ty * nt;
  const bool active = ty < nt;
  extern __shared__ double2 gsh[];
  double2* sA = gsh;
  double2* sB = gsh + RCH * L;
  double2 acc[NB][TM][TM];
#pragma unroll
  for (int k = 0; k < NB; ++k)
#pragma unroll
    for (int i = 0; i < TM; ++i)
#pragma unroll
      for (int j = 0; j < TM; ++j) acc[k][i][j] = make_double2(0.0, 0.0);
  const int64_t chunk = (g.n + gridDim.x - 1) / gridDim.x;
  const int64_t r0 = blockIdx.x * chunk;
  const int64_t r1 = min(g.n, r0 + chunk);
  const T* A = static_cast<const T*>(g.A);
  for (int64_t rb = r0; rb < r1; rb += RCH) {
    const int rows = (int)min((int64_t)RCH, r1 - rb);
    for (int e = t; e < RCH * L; e += blockDim.x) {
      const int r = e / L;
      double2 v = make_double2(0.0, 0.0);
      if (r < rows) {
        v = ld_as<double2>(A, rb * L + e);
        if (CONJ) v.y = -v.y;
      }
      sA[e] = v;
#pragma unroll
      for (int k = 0; k < NB; ++k)
        sB[k * RCH * L + e] = r < rows ? ld_as<double2>(static_cast<const T*>(g.B[k]), rb * L + e)
                                       : make_double2(0.0, 0.0);
    }
    __syncthreads();
    if (active) {
      for (int r = 0; r < rows; ++r) {
        double2 a[TM], b[NB][TM];
#pragma unroll
        for (int ii = 0; ii < TM; ++ii) {
          const int i = ty * TM + ii;
          a[ii] = i < L ? sA[r * L + i] : make_double2(0.0, 0.0);
        }
#pragma unroll
        for (int k = 0; k < NB; ++k)
#pragma unroll
          for (int jj = 0; jj < TM; ++jj) {
            const int j = tx * TM + jj;
            b[k][jj] = j < L ? sB[k * RCH * L + r * L + j] : make_double2(0.0, 0.0);
          }
#pragma unroll
        for (int k = 0; k < NB; ++k)
#pragma unroll
          for (int ii = 0; ii < TM; ++ii)
#pragma unroll
            for (int jj = 0; jj < TM; ++jj) acc[k][ii][jj] = cfma(a[ii], b[k][jj], acc[k][ii][jj]);
      }
    }
    __syncthreads();
  }
  if (active) {
#pragma unroll
    for (int k = 0; k < NB; ++k)
#pragma unroll
      for (int ii = 0; ii < TM; ++ii)
#pragma unroll
        for (int jj = 0; jj < TM; ++jj) {
          const int i = ty * TM + ii, j = tx * TM + jj;
          if (i < L && j < L) g.partial[(((int64_t)blockIdx.x * NB + k) * L + i) * L + j] = acc[k][ii][jj];
        }
  }
}

__global__ void gram_reduce_kernel(const double2* partial, int nblk, int width, double2* out) {
  gram_reduce_body(partial, nblk, width, out, blockIdx.x * blockDim.x + threadIdx.x);
}

template <typename T, bool CONJ, int L, int NB>
__global__ void __launch_bounds__(256) gram_fixed_kernel(GramArgs g) {
  extern __shared__ __align__(16) unsigned char gfs[];
  gram_fixed_body<T, CONJ, L, NB>(g, blockIdx.x, gridDim.x, gfs);
}

template <typename T, bool CONJ, int L>
static int gram_fixed(const GramArgs& g, double2* out, cudaStream_t st) {
  const size_t smem = (size_t)2 * (1 + g.nB) * 16 * L * sizeof(T);
  if (g.nB == 1) {
    auto k = gram_fixed_kernel<T, CONJ, L, 1>;
    BDDA_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k<<<kRedBlocks, 256, smem, st>>>(g);
  } else {
    auto k = gram_fixed_kernel<T, CONJ, L, 2>;
    BDDA_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k<<<kRedBlocks, 256, smem, st>>>(g);
  }
  BDDA_CUDA_TRY(cudaGetLastError());
  const int width = g.nB * L * L;
  gram_reduce_kernel<<<(width + 255) / 256, 256, 0, st>>>(g.partial, kRedBlocks, width, out);
  BDDA_CUDA_TRY(cudaGetLastError());
  count_launch(2);
  return BDDA_OK;
}

template <typename T, bool CONJ, int TM>
static int gram_tm(const GramArgs& g, double2* out, cudaStream_t st) {
  constexpr int RCH = 16;
  const size_t smem = (size_t)RCH * g.L * (1 + g.nB) * sizeof(double2);
  if (g.nB == 1) {
    auto k = gram_kernel<T, CONJ, TM, 1>;
    BDDA_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k<<<kRedBlocks, 256, smem, st>>>(g);
  } else {
    auto k = gram_kernel<T, CONJ, TM, 2>;
    BDDA_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k<<<kRedBlocks, 256, smem, st>>>(g);
  }
  BDDA_CUDA_TRY(cudaGetLastError());
  count_launch(2);
  const int width = g.nB * g.L * g.L;
  gram_reduce_kernel<<<(width + 255) / 256, 256, 0, st>>>(g.partial, kRedBlocks, width, out);
  BDDA_CUDA_TRY(cudaGetLastError());
  return BDDA_OK;
}

template <typename T>
int gram(const GramArgs& g, bool conj, double2* out, cudaStream_t st) {
  if (g.L < 1 || g.L > kMaxL || g.nB < 1 || g.nB > 2) return BDDA_BAD_ARG;
  const bool aligned = ((reinterpret_cast<uintptr_t>(g.A) | reinterpret_cast<uintptr_t>(g.B[0]) |
                         reinterpret_cast<uintptr_t>(g.nB > 1 ? g.B[1] : g.B[0])) & 15) == 0;
  if (aligned && g_fixed_blas) {
#define BDDA_GRAM_L(LL) \
  if (g.L == LL) return conj ? gram_fixed<T, true, LL>(g, out, st) : gram_fixed<T, false, LL>(g, out, st);
    BDDA_GRAM_L(8) BDDA_GRAM_L(16) BDDA_GRAM_L(32) BDDA_GRAM_L(64)
#undef BDDA_GRAM_L
  }
  const int tm = g.L <= 16 ? 1 : (g.L <= 32 ? 2 : 4);
  if (conj) {
    if (tm == 1) return gram_tm<T, true, 1>(g, out, st);
    if (tm == 2) return gram_tm<T, true, 2>(g, out, st);
    return gram_tm<T, true, 4>(g, out, st);
  }
  if (tm == 1) return gram_tm<T, false, 1>(g, out, st);
  if (tm == 2) return gram_tm<T, false, 2>(g, out, st);
  return gram_tm<T, false, 4>(g, out, st);
}

// ---- fused block update -------------------------------------------------------
// out = a0*Y0 + a1*Y1 + (X1 + c2*X2) M, arithmetic in A (double2 for c128,
// float2 for c64 vectors), optional per-CTA partial of ||out||_F^2.
template <typename T, typename A, int TN>
__global__ void __launch_bounds__(256) update_kernel(UpdateArgs u) {
  const int L = u.L;
  const int ncg = (L + TN - 1) / TN;
  const int RCH = blockDim.x / ncg;
  extern __shared__ __align__(16) unsigned char ush[];
  A* sM = reinterpret_cast<A*>(ush);
  A* sX = sM + (u.M ? L * L : 0);
  const int t = threadIdx.x;
  const int rr = t / ncg, cg = t - rr * ncg;
  const bool active = rr < RCH;
  const A one = conv_acc<A>(make_double2(1.0, 0.0));
  const A a0 = u.a0 ? conv_acc<A>(*u.a0) : one;
  const A a1 = u.a1 ? conv_acc<A>(*u.a1) : one;
  const A c2 = u.c2 ? conv_acc<A>(*u.c2) : one;
  const T* Y0 = static_cast<const T*>(u.Y0);
  const T* Y1 = static_cast<const T*>(u.Y1);
  const T* X1 = static_cast<const T*>(u.X1);
  const T* X2 = static_cast<const T*>(u.X2);
  T* out = static_cast<T*>(u.out);
  if (u.M)
    for (int e = t; e < L * L; e += blockDim.x) sM[e] = conv_acc<A>(u.M[e]);
  double nrm = 0.0;
  for (int64_t rb = (int64_t)blockIdx.x * RCH; rb < u.n; rb += (int64_t)gridDim.x * RCH) {
    if (u.M) {
      __syncthreads();
      for (int e = t; e < RCH * L; e += blockDim.x) {
        const int64_t row = rb + e / L;
        A v = conv_acc<A>(make_double2(0.0, 0.0));
        if (row < u.n) {
          v = ld_as<A>(X1, rb * L + e);
          if (X2) {
            const A w = ld_as<A>(X2, rb * L + e);
            v = cfma(c2, w, v);
          }
        }
        sX[e] = v;
      }
      __syncthreads();
    }
    const int64_t row = rb + rr;
    if (active && row < u.n) {
      A acc[TN];
#pragma unroll
      for (int jj = 0; jj < TN; ++jj) {
        const int j = cg * TN + jj;
        acc[jj] = conv_acc<A>(make_double2(0.0, 0.0));
        if (j < L) {
          if (Y0) acc[jj] = cfma(a0, ld_as<A>(Y0, row * L + j), acc[jj]);
          if (Y1) acc[jj] = cfma(a1, ld_as<A>(Y1, row * L + j), acc[jj]);
        }
      }
      if (u.M) {
        for (int i = 0; i < L; ++i) {
          const A x = sX[rr * L + i];
#pragma unroll
          for (int jj = 0; jj < TN; ++jj) {
            const int j = cg * TN + jj;
            if (j < L) acc[jj] = cfma(x, sM[i * L + j], acc[jj]);
          }
        }
      }
#pragma unroll
      for (int jj = 0; jj < TN; ++jj) {
        const int j = cg * TN + jj;
        if (j < L) {
          const T v = st_as<T>(acc[jj]);
          out[row * L + j] = v;
          const double2 vd = to_d2(v);
          nrm += vd.x * vd.x + vd.y * vd.y;
        }
      }
    }
  }
  if (u.norm_partial) {
    const double s = block_sum(nrm);
    if (threadIdx.x == 0) u.norm_partial[blockIdx.x] = s;
  }
}

template <typename T, typename A, int L>
__global__ void __launch_bounds__(256) update_fixed_kernel(UpdateArgs u) {
  extern __shared__ __align__(16) unsigned char ufs[];
  update_fixed_body<T, A, L>(u, blockIdx.x, gridDim.x, ufs);
}

template <typename T, typename A, int L>
static int update_fixed(const UpdateArgs& u, cudaStream_t st) {
  constexpr int TC = L >= 64 ? 4 : (L >= 32 ? 2 : 1);
  constexpr int RB = (256 / (L / TC)) * 2;
  const size_t smem = u.M ? ((size_t)L * L + (size_t)RB * L) * sizeof(A) : 0;
  auto k = update_fixed_kernel<T, A, L>;
  BDDA_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k<<<kRedBlocks, 256, smem, st>>>(u);
  BDDA_CUDA_TRY(cudaGetLastError());
  count_launch();
  return BDDA_OK;
}

template <typename T, typename A, int TN>
static int update_tn(const UpdateArgs& u, cudaStream_t st) {
  const int ncg = (u.L + TN - 1) / TN;
  const int rch = 256 / ncg;
  const size_t smem = ((u.M ? (size_t)u.L * u.L : 0) + (u.M ? (size_t)rch * u.L : 0)) * sizeof(A);
  auto k = update_kernel<T, A, TN>;
  BDDA_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k<<<kRedBlocks, 256, smem, st>>>(u);
  BDDA_CUDA_TRY(cudaGetLastError());
  count_launch();
  return BDDA_OK;
}

template <typename T>
int update(const UpdateArgs& u, cudaStream_t st) {
  if (u.L < 1 || u.L > kMaxL || !u.out) return BDDA_BAD_ARG;
  typedef typename std::conditional<std::is_same<T, float2>::value, float2, double2>::type A;
  if (g_fixed_blas) {
    if (u.L == 64) return update_fixed<T, A, 64>(u, st);
    if (u.L == 32) return update_fixed<T, A, 32>(u, st);
    if (u.L == 16) return update_fixed<T, A, 16>(u, st);
    if (u.L == 8) return update_fixed<T, A, 8>(u, st);
  }
  if (u.L >= 32) return update_tn<T, A, 4>(u, st);
  if (u.L >= 16) return update_tn<T, A, 2>(u, st);
  return update_tn<T, A, 1>(u, st);
}

template <typename T>
__global__ void __launch_bounds__(256) dots_kernel(DotArgs d) {
  dots_body<T>(d, blockIdx.x, gridDim.x);
}

template <typename T>
int dots(const DotArgs& d, cudaStream_t st) {
  dots_kernel<T><<<kRedBlocks, 256, 0, st>>>(d);
  BDDA_CUDA_TRY(cudaGetLastError());
  count_launch();
  return BDDA_OK;
}

__global__ void reduce_partials_kernel(const double* partial, int nblk, int width, double* out) {
  for (int w = 0; w < width; ++w) {
    double s = 0.0;
    for (int b = threadIdx.x; b < nblk; b += blockDim.x) s += partial[(int64_t)b * width + w];
    s = block_sum(s);
    if (threadIdx.x == 0) out[w] = s;
    __syncthreads();
  }
}

int reduce_partials(const double* partial, int nblk, int width, double* out, cudaStream_t st) {
  reduce_partials_kernel<<<1, 256, 0, st>>>(partial, nblk, width, out);
  BDDA_CUDA_TRY(cudaGetLastError());
  count_launch();
  return BDDA_OK;
}

void set_fixed_blas(int on) { g_fixed_blas = on ? 1 : 0; }

template int gram<double2>(const GramArgs&, bool, double2*, cudaStream_t);
template int gram<float2>(const GramArgs&, bool, double2*, cudaStream_t);
template int update<double2>(const UpdateArgs&, cudaStream_t);
template int update<float2>(const UpdateArgs&, cudaStream_t);
template int dots<double2>(const DotArgs&, cudaStream_t);
template int dots<float2>(const DotArgs&, cudaStream_t);

}  // namespace bdda
