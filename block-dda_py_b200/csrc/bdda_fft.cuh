// Mixed-radix pencil FFT building blocks for the doubled-grid block MVP.
//
// A "pencil" is one line of a 3-D grid along the axis being transformed.  A
// CTA stages one pencil x one column tile in shared memory as [row][W]
// complex values (W = 3 components x LT right-hand sides) and runs the
// radix stages there; every global access is a run of LT contiguous complex
// values, so all five passes of the MVP read and write whole sectors.
//
// Forward transforms are decimation-in-frequency (natural order in,
// digit-reversed order out); inverse transforms are decimation-in-time
// (digit-reversed in, natural out).  Spectra therefore stay in digit-reversed
// order in HBM between passes and no permutation pass is ever needed; the
// Green's tensor spectrum is built by the same forward stages, so it is
// stored in the same order.  Transforms are unnormalised; the 1/(Mx My Mz)
// of the inverse FFT is applied once, in the last pass.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace bdda {

constexpr int kMaxStages = 12;

template <typename T> struct real_of;
template <> struct real_of<double2> { typedef double type; };
template <> struct real_of<float2> { typedef float type; };

template <typename T> __host__ __device__ __forceinline__ T mkc(typename real_of<T>::type re,
                                                               typename real_of<T>::type im) {
  T r; r.x = re; r.y = im; return r;
}
template <typename T> __device__ __forceinline__ T cadd(T a, T b) { return mkc<T>(a.x + b.x, a.y + b.y); }
template <typename T> __device__ __forceinline__ T csub(T a, T b) { return mkc<T>(a.x - b.x, a.y - b.y); }
template <typename T> __device__ __forceinline__ T cmul(T a, T b) {
  return mkc<T>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
template <typename T> __device__ __forceinline__ T cmulc(T a, T b) {
  return mkc<T>(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
template <typename T> __device__ __forceinline__ T cscale(T a, typename real_of<T>::type s) {
  return mkc<T>(a.x * s, a.y * s);
}
// multiply by -i for a forward transform, by +i for an inverse one
template <bool INV, typename T> __device__ __forceinline__ T mul_mi(T a) {
  return INV ? mkc<T>(-a.y, a.x) : mkc<T>(a.y, -a.x);
}

// cos / sin of 2*pi*j/R for the odd radices (values from the definition,
// 25 significant digits, rounded by the compiler to the working precision)
template <int R> __device__ __forceinline__ constexpr double root_cos(int j);
template <int R> __device__ __forceinline__ constexpr double root_sin(int j);
template <> __device__ __forceinline__ constexpr double root_cos<3>(int j) { return j == 0 ? 1.0 : -0.5; }
template <> __device__ __forceinline__ constexpr double root_sin<3>(int j) {
  return j == 0 ? 0.0 : (j == 1 ? 0.8660254037844386467637232 : -0.8660254037844386467637232);
}
template <> __device__ __forceinline__ constexpr double root_cos<5>(int j) {
  return j == 0 ? 1.0 : (j == 1 || j == 4) ? 0.3090169943749474241022934 : -0.8090169943749474241022934;
}
template <> __device__ __forceinline__ constexpr double root_sin<5>(int j) {
  return j == 0 ? 0.0 : j == 1 ? 0.9510565162951535721164393 : j == 2 ? 0.587785252292473129168706
       : j == 3 ? -0.587785252292473129168706 : -0.9510565162951535721164393;
}
template <> __device__ __forceinline__ constexpr double root_cos<7>(int j) {
  return j == 0 ? 1.0 : (j == 1 || j == 6) ? 0.6234898018587335305250049
       : (j == 2 || j == 5) ? -0.2225209339563144042889026 : -0.9009688679024191262361023;
}
template <> __device__ __forceinline__ constexpr double root_sin<7>(int j) {
  return j == 0 ? 0.0 : j == 1 ? 0.7818314824680298087084445 : j == 2 ? 0.9749279121818236070181317
       : j == 3 ? 0.4338837391175581204757683 : j == 4 ? -0.4338837391175581204757683
       : j == 5 ? -0.9749279121818236070181317 : -0.7818314824680298087084445;
}

// ---- small DFTs on registers: y_q = sum_p v_p exp(-+2 pi i p q / R) ----------
template <bool INV, typename T> __device__ __forceinline__ void dft2(T* v) {
  T a = v[0], b = v[1];
  v[0] = cadd(a, b); v[1] = csub(a, b);
}
template <bool INV, typename T> __device__ __forceinline__ void dft4(T* v) {
  T a = cadd(v[0], v[2]), b = csub(v[0], v[2]);
  T c = cadd(v[1], v[3]), d = mul_mi<INV>(csub(v[1], v[3]));
  v[0] = cadd(a, c); v[2] = csub(a, c);
  v[1] = cadd(b, d); v[3] = csub(b, d);
}
template <bool INV, typename T> __device__ __forceinline__ void dft8(T* v) {
  typedef typename real_of<T>::type R;
  const R h = R(0.7071067811865475244008444);
  T e[4] = {v[0], v[2], v[4], v[6]};
  T o[4] = {v[1], v[3], v[5], v[7]};
  dft4<INV>(e); dft4<INV>(o);
  T t1, t3;
  if (!INV) {   // w = exp(-i pi/4), w^3 = exp(-3 i pi/4)
    t1 = mkc<T>(h * (o[1].x + o[1].y), h * (o[1].y - o[1].x));
    t3 = mkc<T>(h * (o[3].y - o[3].x), -h * (o[3].x + o[3].y));
  } else {      // w = exp(+i pi/4), w^3 = exp(+3 i pi/4)
    t1 = mkc<T>(h * (o[1].x - o[1].y), h * (o[1].x + o[1].y));
    t3 = mkc<T>(-h * (o[3].x + o[3].y), h * (o[3].x - o[3].y));
  }
  T t2 = mul_mi<INV>(o[2]);
  v[0] = cadd(e[0], o[0]); v[4] = csub(e[0], o[0]);
  v[1] = cadd(e[1], t1);   v[5] = csub(e[1], t1);
  v[2] = cadd(e[2], t2);   v[6] = csub(e[2], t2);
  v[3] = cadd(e[3], t3);   v[7] = csub(e[3], t3);
}
// odd R: pair p with R-p so that only (R-1)^2/2 real products per component remain
template <int R, bool INV, typename T> __device__ __forceinline__ void dft_odd(T* v) {
  typedef typename real_of<T>::type F;
  constexpr int H = (R - 1) / 2;
  T a[H], b[H];
#pragma unroll
  for (int k = 1; k <= H; ++k) { a[k - 1] = cadd(v[k], v[R - k]); b[k - 1] = csub(v[k], v[R - k]); }
  T y[R];
  y[0] = v[0];
#pragma unroll
  for (int k = 0; k < H; ++k) y[0] = cadd(y[0], a[k]);
#pragma unroll
  for (int q = 1; q <= H; ++q) {
    T re = v[0], im = mkc<T>(F(0), F(0));
#pragma unroll
    for (int k = 1; k <= H; ++k) {
      const F c = F(root_cos<R>((q * k) % R));
      const F s = F(root_sin<R>((q * k) % R));
      re = mkc<T>(re.x + a[k - 1].x * c, re.y + a[k - 1].y * c);
      im = mkc<T>(im.x + b[k - 1].x * s, im.y + b[k - 1].y * s);
    }
    const T mi = mkc<T>(im.y, -im.x);   // -i * im
    y[q] = INV ? csub(re, mi) : cadd(re, mi);
    y[R - q] = INV ? cadd(re, mi) : csub(re, mi);
  }
#pragma unroll
  for (int q = 0; q < R; ++q) v[q] = y[q];
}

template <int R, bool INV, typename T> __device__ __forceinline__ void dft(T* v) {
  if constexpr (R == 2) dft2<INV>(v);
  else if constexpr (R == 4) dft4<INV>(v);
  else if constexpr (R == 8) dft8<INV>(v);
  else dft_odd<R, INV>(v);
}

// ---- one radix-R butterfly on shared memory ---------------------------------
// DIF (forward):   v = x[q*stride]; v = DFT(v); v[q] *= w^(q*tws); store
// DIT (inverse):   v = x[q*stride]; v[q] *= conj(w^(q*tws)); v = IDFT(v); store
template <int R, typename T> __device__ __forceinline__ void bfly_dif(T* p, int stride, const T* tw, int tws) {
  T v[R];
#pragma unroll
  for (int q = 0; q < R; ++q) v[q] = p[q * stride];
  dft<R, false>(v);
  if (tws) {
#pragma unroll
    for (int q = 1; q < R; ++q) v[q] = cmul(v[q], tw[q * tws]);
  }
#pragma unroll
  for (int q = 0; q < R; ++q) p[q * stride] = v[q];
}
template <int R, typename T> __device__ __forceinline__ void bfly_dit(T* p, int stride, const T* tw, int tws) {
  T v[R];
#pragma unroll
  for (int q = 0; q < R; ++q) v[q] = p[q * stride];
  if (tws) {
#pragma unroll
    for (int q = 1; q < R; ++q) v[q] = cmulc(v[q], tw[q * tws]);
  }
  dft<R, true>(v);
#pragma unroll
  for (int q = 0; q < R; ++q) p[q * stride] = v[q];
}

template <int R, bool INV, typename T>
__device__ __forceinline__ void bfly(T* p, int stride, const T* tw, int tws) {
  if constexpr (INV) bfly_dit<R>(p, stride, tw, tws);
  else bfly_dif<R>(p, stride, tw, tws);
}

// Per-axis FFT description, passed by value to the kernels.
struct AxisFFT {
  int M;                  // cyclic length
  int nst;                // number of radix stages
  int rad[kMaxStages];    // stage radices (DIF order)
  int blk[kMaxStages];    // sub-transform length entering each DIF stage
};

// Run all stages of a length-M transform on a [M][W] shared-memory tile.
// Thread jobs are (butterfly, column) pairs with the column fastest, so a
// quarter-warp touches contiguous 16-byte words (no bank conflicts).
template <bool INV, int W, typename T>
__device__ __forceinline__ void fft_stages(T* sm, const T* tw, const AxisFFT& ax) {
  const int M = ax.M;
  for (int si = 0; si < ax.nst; ++si) {
    const int s = INV ? ax.nst - 1 - si : si;
    const int r = ax.rad[s];
    const int B = ax.blk[s];
    const int span = B / r;
    const int tstep = M / B;
    const int njobs = (M / r) * W;
    for (int job = threadIdx.x; job < njobs; job += blockDim.x) {
      const int col = job % W;
      const int t = job / W;
      const int b = t / span;
      const int j = t - b * span;
      T* p = sm + (b * B + j) * W + col;
      const int stride = span * W;
      const int tws = j * tstep;
      switch (r) {
        case 2: bfly<2, INV>(p, stride, tw, tws); break;
        case 3: bfly<3, INV>(p, stride, tw, tws); break;
        case 4: bfly<4, INV>(p, stride, tw, tws); break;
        case 5: bfly<5, INV>(p, stride, tw, tws); break;
        case 7: bfly<7, INV>(p, stride, tw, tws); break;
        default: bfly<8, INV>(p, stride, tw, tws); break;
      }
    }
    __syncthreads();
  }
}

}  // namespace bdda
