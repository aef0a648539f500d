// Device bodies of the L-specialised block kernels, shared by the
// one-problem kernels (bdda_blas.cu) and the batched persistent kernels
// (bdda_batch.cu).  Each body handles split index bid of nblk for one
// problem's arguments.
#pragma once
#include "bdda_blas.cuh"

namespace bdda {

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

// Per-element reduction of gram partials: out[o] = sum_b partial[b][o].
__device__ __forceinline__ void gram_reduce_body(const double2* partial, int nblk, int width, double2* out, int o) {
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
// A thread owns rows ty + NT i and columns tx + NT j of the L x L tile, so the
// 32 lanes of a warp read consecutive 16-byte words of a staged row (no
// shared-memory bank conflicts).
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
__device__ __forceinline__ void gram_fixed_body(const GramArgs& g, int64_t bid, int64_t nblk, unsigned char* gfs) {
  constexpr int TM = L >= 64 ? 4 : (L >= 32 ? 2 : 1);
  constexpr int NT = L / TM;                       // thread grid side
  constexpr int RCH = 16;
  constexpr int CH = RCH * L;
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
  const int64_t per = (nchunks + nblk - 1) / nblk;
  const int64_t c0 = bid * per, c1 = min(nchunks, c0 + per);
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
          a[ii] = to_d2(sA[r * L + ty + NT * ii]);
          if (CONJ) a[ii].y = -a[ii].y;
        }
#pragma unroll
        for (int k = 0; k < NB; ++k)
#pragma unroll
          for (int jj = 0; jj < TM; ++jj) b[k][jj] = to_d2(sA[(1 + k) * CH + r * L + tx + NT * jj]);
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
          g.partial[((bid * NB + k) * L + ty + NT * ii) * L + tx + NT * jj] = acc[k][ii][jj];
  }
}

// ---- block update, specialised on L ---------------------------------------------
// out = a0 Y0 + a1 Y1 + (X1 + c2 X2) M.  M lives in shared memory for the
// whole kernel; X row blocks of RB rows are staged per iteration; each thread
// owns TR rows x TC columns (cg + NCG j) of the output block, so lanes read
// consecutive 16-byte words of M (no shared-memory bank conflicts).
template <typename T, typename A, int L>
__device__ __forceinline__ void update_fixed_body(const UpdateArgs& u, int64_t bid, int64_t nblk, unsigned char* ufs) {
  constexpr int TC = L >= 64 ? 4 : (L >= 32 ? 2 : 1);
  constexpr int NCG = L / TC;
  constexpr int NRG = 256 / NCG;
  constexpr int TR = 2;
  constexpr int RB = NRG * TR;
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
  for (int64_t rb = bid * RB; rb < u.n; rb += nblk * RB) {
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
          const int64_t idx = row * L + cg + NCG * jj;
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
        for (int jj = 0; jj < TC; ++jj) m[jj] = sM[i * L + cg + NCG * jj];
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
          out[row * L + cg + NCG * jj] = v;
          const double2 vd = to_d2(v);
          nrm += vd.x * vd.x + vd.y * vd.y;
        }
      }
    }
  }
  if (u.norm_partial) {
    const double s = block_sum(nrm);
    if (threadIdx.x == 0) u.norm_partial[bid] = s;
  }
}

// ---- Frobenius dots: sum conj(A) B and sum |A|^2 ------------------------------
template <typename T>
__device__ __forceinline__ void dots_body(const DotArgs& d, int64_t bid, int64_t nblk) {
  const T* A = static_cast<const T*>(d.A);
  const T* B = static_cast<const T*>(d.B);
  double re = 0.0, im = 0.0, aa = 0.0;
  for (int64_t i = bid * (int64_t)blockDim.x + threadIdx.x; i < d.n; i += nblk * blockDim.x) {
    const double2 a = to_d2(A[i]), b = to_d2(B[i]);
    re += a.x * b.x + a.y * b.y;
    im += a.x * b.y - a.y * b.x;
    aa += a.x * a.x + a.y * a.y;
  }
  re = block_sum(re);
  im = block_sum(im);
  aa = block_sum(aa);
  if (threadIdx.x == 0) {
    d.partial[bid * 3 + 0] = re;
    d.partial[bid * 3 + 1] = im;
    d.partial[bid * 3 + 2] = aa;
  }
}

}  // namespace bdda
