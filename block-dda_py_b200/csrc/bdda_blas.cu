// Tall-skinny block kernels: Gram products, fused block updates, dots.
#include <climits>
#include <type_traits>

#include "bdda_blas.cuh"
#include "bdda_internal.h"

namespace bdda {

// L-specialised Gram / update kernels on (tests switch them off to compare).
static int g_fixed_blas = 1;

template <typename A> __device__ __forceinline__ A conv_acc(double2 v);
template <> __device__ __forceinline__ double2 conv_acc<double2>(double2 v) { return v; }
template <> __device__ __forceinline__ float2 conv_acc<float2>(double2 v) {
  return make_float2((float)v.x, (float)v.y);
}
template <typename A> __device__ __forceinline__ A load_acc(const double2* v) { return conv_acc<A>(*v); }
__device__ __forceinline__ double2 up(double2 v) { return v; }
__device__ __forceinline__ float2 up_f(float2 v) { return v; }

template <typename A, typename T> __device__ __forceinline__ A ld_as(const T* p, int64_t i);
template <> __device__ __forceinline__ double2 ld_as<double2, double2>(const double2* p, int64_t i) { return p[i]; }
template <> __device__ __forceinline__ double2 ld_as<double2, float2>(const float2* p, int64_t i) {
  const float2 v = p[i];
  return make_double2(v.x, v.y);
}
template <> __device__ __forceinline__ float2 ld_as<float2, float2>(const float2* p, int64_t i) { return p[i]; }

template <typename T, typename A> __device__ __forceinline__ T st_as(A v);
template <> __device__ __forceinline__ double2 st_as<double2, double2>(double2 v) { return v; }
template <> __device__ __forceinline__ float2 st_as<float2, float2>(float2 v) { return v; }
template <> __device__ __forceinline__ float2 st_as<float2, double2>(double2 v) {
  return make_float2((float)v.x, (float)v.y);
}

__device__ __forceinline__ double2 cfma(double2 a, double2 b, double2 c) {
  return make_double2(fma(a.x, b.x, fma(-a.y, b.y, c.x)), fma(a.x, b.y, fma(a.y, b.x, c.y)));
}
__device__ __forceinline__ float2 cfma(float2 a, float2 b, float2 c) {
  return make_float2(fmaf(a.x, b.x, fmaf(-a.y, b.y, c.x)), fmaf(a.x, b.y, fmaf(a.y, b.x, c.y)));
}

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
  const int o = blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= width) return;
  double2 s = make_double2(0.0, 0.0);
  for (int b = 0; b < nblk; ++b) {
    const double2 v = partial[(int64_t)b * width + o];
    s.x += v.x;
    s.y += v.y;
  }
  out[o] = s;
}

// ---- Gram, specialised on L: split-K over row chunks, register tiles --------
// Each CTA reduces a contiguous range of rows into a full L x L partial (per
// B matrix); row chunks of RCH rows are double-buffered in shared memory with
// cp.async so the next chunk streams in while the current one is consumed.
__device__ __forceinline__ void cp_async16_g(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit_g() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait_g() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

template <typename T, int L, int RCH>
__device__ __forceinline__ void stage_rows(T* dst, const T* src, int64_t rb, int64_t r1) {
  // rows [rb, min(rb + RCH, r1)) of an (n, L) block, 16-byte granules; the rest zeroed
  constexpr int BYTES = RCH * L * (int)sizeof(T);
  const int64_t rows = min((int64_t)RCH, r1 - rb);
  const int valid = (int)(rows * L * (int)sizeof(T));
  const char* s = reinterpret_cast<const char*>(src + rb * L);
  char* d = reinterpret_cast<char*>(dst);
  for (int off = threadIdx.x * 16; off < BYTES; off += blockDim.x * 16) {
    if (off < valid) cp_async16_g(d + off, s + off);
    else *reinterpret_cast<uint4*>(d + off) = make_uint4(0, 0, 0, 0);
  }
}

template <typename T, bool CONJ, int L, int NB>
__global__ void __launch_bounds__(256) gram_fixed_kernel(GramArgs g) {
  constexpr int TM = L >= 64 ? 4 : (L >= 32 ? 2 : 1);
  constexpr int NT = L / TM;                       // thread grid side
  constexpr int RCH = 16;
  constexpr int CH = RCH * L;
  extern __shared__ __align__(16) unsigned char gfs[];
  T* buf = reinterpret_cast<T*>(gfs);               // [2][1 + NB][CH]
  const int t = threadIdx.x;
  const int ty = t / NT, tx = t - ty * NT;
  const bool active = ty < NT;
  double2 acc[NB][TM][TM];
#pragma unroll
  for (int k = 0; k < NB; ++k)
#pragma unroll
    for (int i = 0; i < TM; ++i)
#pragma unroll
      for (int j = 0; j < TM; ++j) acc[k][i][j] = make_double2(0.0, 0.0);
  const int64_t nchunks = (g.n + RCH - 1) / RCH;
  const int64_t per = (nchunks + gridDim.x - 1) / gridDim.x;
  const int64_t c0 = blockIdx.x * per, c1 = min(nchunks, c0 + per);
  const T* A = static_cast<const T*>(g.A);
  auto stage = [&](int64_t ck, int slot) {
    T* b = buf + slot * (1 + NB) * CH;
    stage_rows<T, L, RCH>(b, A, ck * RCH, g.n);
#pragma unroll
    for (int k = 0; k < NB; ++k) stage_rows<T, L, RCH>(b + (1 + k) * CH, static_cast<const T*>(g.B[k]), ck * RCH, g.n);
  };
  if (c0 < c1) stage(c0, 0);
  cp_async_commit_g();
  for (int64_t ck = c0; ck < c1; ++ck) {
    const int slot = (int)((ck - c0) & 1);
    if (ck + 1 < c1) stage(ck + 1, slot ^ 1);
    cp_async_commit_g();
    cp_async_wait_g<1>();
    __syncthreads();
    const T* sA = buf + slot * (1 + NB) * CH;
    if (active) {
#pragma unroll 4
      for (int r = 0; r < RCH; ++r) {
        double2 a[TM], b[NB][TM];
#pragma unroll
        for (int ii = 0; ii < TM; ++ii) {
          a[ii] = to_d2(sA[r * L + ty * TM + ii]);
          if (CONJ) a[ii].y = -a[ii].y;
        }
#pragma unroll
        for (int k = 0; k < NB; ++k)
#pragma unroll
          for (int jj = 0; jj < TM; ++jj) b[k][jj] = to_d2(sA[(1 + k) * CH + r * L + tx * TM + jj]);
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
  cp_async_wait_g<0>();
  if (active) {
#pragma unroll
    for (int k = 0; k < NB; ++k)
#pragma unroll
      for (int ii = 0; ii < TM; ++ii)
#pragma unroll
        for (int jj = 0; jj < TM; ++jj)
          g.partial[(((int64_t)blockIdx.x * NB + k) * L + ty * TM + ii) * L + tx * TM + jj] = acc[k][ii][jj];
  }
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

// ---- block update, specialised on L ---------------------------------------------
// out = a0 Y0 + a1 Y1 + (X1 + c2 X2) M.  M lives in shared memory for the
// whole kernel; X row blocks of RB rows are staged per iteration; each thread
// owns TR rows x TC columns of the output block.
template <typename T, typename A, int L>
__global__ void __launch_bounds__(256) update_fixed_kernel(UpdateArgs u) {
  constexpr int TC = L >= 64 ? 4 : (L >= 32 ? 2 : 1);
  constexpr int NCG = L / TC;
  constexpr int NRG = 256 / NCG;
  constexpr int TR = 2;
  constexpr int RB = NRG * TR;
  extern __shared__ __align__(16) unsigned char ufs[];
  A* sM = reinterpret_cast<A*>(ufs);
  A* sX = sM + (u.M ? L * L : 0);
  const int t = threadIdx.x;
  const int rg = t / NCG, cg = t - rg * NCG;
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
    for (int e = t; e < L * L; e += 256) sM[e] = conv_acc<A>(u.M[e]);
  double nrm = 0.0;
  for (int64_t rb = (int64_t)blockIdx.x * RB; rb < u.n; rb += (int64_t)gridDim.x * RB) {
    if (u.M) {
      __syncthreads();
      for (int e = t; e < RB * L; e += 256) {
        const int64_t row = rb + e / L;
        A v = conv_acc<A>(make_double2(0.0, 0.0));
        if (row < u.n) {
          v = ld_as<A>(X1, rb * L + e);
          if (X2) v = cfma(c2, ld_as<A>(X2, rb * L + e), v);
        }
        sX[e] = v;
      }
      __syncthreads();
    }
    A acc[TR][TC];
#pragma unroll
    for (int ii = 0; ii < TR; ++ii) {
      const int64_t row = rb + rg * TR + ii;
#pragma unroll
      for (int jj = 0; jj < TC; ++jj) {
        acc[ii][jj] = conv_acc<A>(make_double2(0.0, 0.0));
        if (row < u.n) {
          const int64_t idx = row * L + cg * TC + jj;
          if (Y0) acc[ii][jj] = cfma(a0, ld_as<A>(Y0, idx), acc[ii][jj]);
          if (Y1) acc[ii][jj] = cfma(a1, ld_as<A>(Y1, idx), acc[ii][jj]);
        }
      }
    }
    if (u.M) {
#pragma unroll 8
      for (int i = 0; i < L; ++i) {
        A x[TR], m[TC];
#pragma unroll
        for (int ii = 0; ii < TR; ++ii) x[ii] = sX[(rg * TR + ii) * L + i];
#pragma unroll
        for (int jj = 0; jj < TC; ++jj) m[jj] = sM[i * L + cg * TC + jj];
#pragma unroll
        for (int ii = 0; ii < TR; ++ii)
#pragma unroll
          for (int jj = 0; jj < TC; ++jj) acc[ii][jj] = cfma(x[ii], m[jj], acc[ii][jj]);
      }
    }
#pragma unroll
    for (int ii = 0; ii < TR; ++ii) {
      const int64_t row = rb + rg * TR + ii;
      if (row < u.n) {
#pragma unroll
        for (int jj = 0; jj < TC; ++jj) {
          const T v = st_as<T>(acc[ii][jj]);
          out[row * L + cg * TC + jj] = v;
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

// ---- Frobenius dots: sum conj(A) B and sum |A|^2 ------------------------------
template <typename T>
__global__ void __launch_bounds__(256) dots_kernel(DotArgs d) {
  const T* A = static_cast<const T*>(d.A);
  const T* B = static_cast<const T*>(d.B);
  double re = 0.0, im = 0.0, aa = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < d.n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double2 a = to_d2(A[i]), b = to_d2(B[i]);
    re += a.x * b.x + a.y * b.y;
    im += a.x * b.y - a.y * b.x;
    aa += a.x * a.x + a.y * a.y;
  }
  re = block_sum(re);
  im = block_sum(im);
  aa = block_sum(aa);
  if (threadIdx.x == 0) {
    d.partial[blockIdx.x * 3 + 0] = re;
    d.partial[blockIdx.x * 3 + 1] = im;
    d.partial[blockIdx.x * 3 + 2] = aa;
  }
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
