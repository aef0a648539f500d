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

// cos / sin of 2*pi*j/R for the odd and composite radices (values from the
// definition, 25 significant digits, rounded by the compiler to the working
// precision)
template <int R> __device__ __forceinline__ constexpr double root_cos(int j);
template <int R> __device__ __forceinline__ constexpr double root_sin(int j);
template <> __device__ __forceinline__ constexpr double root_cos<3>(int j) {
  constexpr double t[3] = {1.000000000000000000000000, -0.5000000000000000000000000, -0.5000000000000000000000000};
  return t[j];
}
template <> __device__ __forceinline__ constexpr double root_sin<3>(int j) {
  constexpr double t[3] = {0.0, 0.8660254037844386467637232, -0.8660254037844386467637232};
  return t[j];
}
template <> __device__ __forceinline__ constexpr double root_cos<5>(int j) {
  constexpr double t[5] = {1.000000000000000000000000, 0.3090169943749474241022934, -0.8090169943749474241022934, -0.8090169943749474241022934, 0.3090169943749474241022934};
  return t[j];
}
template <> __device__ __forceinline__ constexpr double root_sin<5>(int j) {
  constexpr double t[5] = {0.0, 0.9510565162951535721164393, 0.5877852522924731291687060, -0.5877852522924731291687060, -0.9510565162951535721164393};
  return t[j];
}
template <> __device__ __forceinline__ constexpr double root_cos<6>(int j) {
  constexpr double t[6] = {1.000000000000000000000000, 0.5000000000000000000000000, -0.5000000000000000000000000, -1.000000000000000000000000, -0.5000000000000000000000000, 0.5000000000000000000000000};
  return t[j];
}
template <> __device__ __forceinline__ constexpr double root_sin<6>(int j) {
  constexpr double t[6] = {0.0, 0.8660254037844386467637232, 0.8660254037844386467637232, 0.0, -0.8660254037844386467637232, -0.8660254037844386467637232};
  return t[j];
}
template <> __device__ __forceinline__ constexpr double root_cos<7>(int j) {
  constexpr double t[7] = {1.000000000000000000000000, 0.6234898018587335305250049, -0.2225209339563144042889026, -0.9009688679024191262361023, -0.9009688679024191262361023, -0.2225209339563144042889026, 0.6234898018587335305250049};
  return t[j];
}
template <> __device__ __forceinline__ constexpr double root_sin<7>(int j) {
  constexpr double t[7] = {0.0, 0.7818314824680298087084445, 0.9749279121818236070181317, 0.4338837391175581204757683, -0.4338837391175581204757683, -0.9749279121818236070181317, -0.7818314824680298087084445};
  return t[j];
}
template <> __device__ __forceinline__ constexpr double root_cos<9>(int j) {
  constexpr double t[9] = {1.000000000000000000000000, 0.7660444431189780352023927, 0.1736481776669303488517166, -0.5000000000000000000000000, -0.9396926207859083840541093, -0.9396926207859083840541093, -0.5000000000000000000000000, 0.1736481776669303488517166, 0.7660444431189780352023927};
  return t[j];
}
template <> __device__ __forceinline__ constexpr double root_sin<9>(int j) {
  constexpr double t[9] = {0.0, 0.6427876096865393263226434, 0.9848077530122080593667430, 0.8660254037844386467637232, 0.3420201433256687330440996, -0.3420201433256687330440996, -0.8660254037844386467637232, -0.9848077530122080593667430, -0.6427876096865393263226434};
  return t[j];
}
template <> __device__ __forceinline__ constexpr double root_cos<10>(int j) {
  constexpr double t[10] = {1.000000000000000000000000, 0.8090169943749474241022934, 0.3090169943749474241022934, -0.3090169943749474241022934, -0.8090169943749474241022934, -1.000000000000000000000000, -0.8090169943749474241022934, -0.3090169943749474241022934, 0.3090169943749474241022934, 0.8090169943749474241022934};
  return t[j];
}
template <> __device__ __forceinline__ constexpr double root_sin<10>(int j) {
  constexpr double t[10] = {0.0, 0.5877852522924731291687060, 0.9510565162951535721164393, 0.9510565162951535721164393, 0.5877852522924731291687060, 0.0, -0.5877852522924731291687060, -0.9510565162951535721164393, -0.9510565162951535721164393, -0.5877852522924731291687060};
  return t[j];
}
template <> __device__ __forceinline__ constexpr double root_cos<12>(int j) {
  constexpr double t[12] = {1.000000000000000000000000, 0.8660254037844386467637232, 0.5000000000000000000000000, 0.0, -0.5000000000000000000000000, -0.8660254037844386467637232, -1.000000000000000000000000, -0.8660254037844386467637232, -0.5000000000000000000000000, 0.0, 0.5000000000000000000000000, 0.8660254037844386467637232};
  return t[j];
}
template <> __device__ __forceinline__ constexpr double root_sin<12>(int j) {
  constexpr double t[12] = {0.0, 0.5000000000000000000000000, 0.8660254037844386467637232, 1.000000000000000000000000, 0.8660254037844386467637232, 0.5000000000000000000000000, 0.0, -0.5000000000000000000000000, -0.8660254037844386467637232, -1.000000000000000000000000, -0.8660254037844386467637232, -0.5000000000000000000000000};
  return t[j];
}
template <> __device__ __forceinline__ constexpr double root_cos<14>(int j) {
  constexpr double t[14] = {1.000000000000000000000000, 0.9009688679024191262361023, 0.6234898018587335305250049, 0.2225209339563144042889026, -0.2225209339563144042889026, -0.6234898018587335305250049, -0.9009688679024191262361023, -1.000000000000000000000000, -0.9009688679024191262361023, -0.6234898018587335305250049, -0.2225209339563144042889026, 0.2225209339563144042889026, 0.6234898018587335305250049, 0.9009688679024191262361023};
  return t[j];
}
template <> __device__ __forceinline__ constexpr double root_sin<14>(int j) {
  constexpr double t[14] = {0.0, 0.4338837391175581204757683, 0.7818314824680298087084445, 0.9749279121818236070181317, 0.9749279121818236070181317, 0.7818314824680298087084445, 0.4338837391175581204757683, 0.0, -0.4338837391175581204757683, -0.7818314824680298087084445, -0.9749279121818236070181317, -0.9749279121818236070181317, -0.7818314824680298087084445, -0.4338837391175581204757683};
  return t[j];
}
template <> __device__ __forceinline__ constexpr double root_cos<16>(int j) {
  constexpr double t[16] = {1.000000000000000000000000, 0.9238795325112867561281832, 0.7071067811865475244008444, 0.3826834323650897717284600, 0.0, -0.3826834323650897717284600, -0.7071067811865475244008444, -0.9238795325112867561281832, -1.000000000000000000000000, -0.9238795325112867561281832, -0.7071067811865475244008444, -0.3826834323650897717284600, 0.0, 0.3826834323650897717284600, 0.7071067811865475244008444, 0.9238795325112867561281832};
  return t[j];
}
template <> __device__ __forceinline__ constexpr double root_sin<16>(int j) {
  constexpr double t[16] = {0.0, 0.3826834323650897717284600, 0.7071067811865475244008444, 0.9238795325112867561281832, 1.000000000000000000000000, 0.9238795325112867561281832, 0.7071067811865475244008444, 0.3826834323650897717284600, 0.0, -0.3826834323650897717284600, -0.7071067811865475244008444, -0.9238795325112867561281832, -1.000000000000000000000000, -0.9238795325112867561281832, -0.7071067811865475244008444, -0.3826834323650897717284600};
  return t[j];
}

template <> __device__ __forceinline__ constexpr double root_cos<24>(int j) {
  constexpr double t[24] = {1.000000000000000000000000, 0.9659258262890682867497432, 0.8660254037844386467637232, 0.7071067811865475244008444, 0.5000000000000000000000000, 0.2588190451025207623488988, 0.0, -0.2588190451025207623488988, -0.5000000000000000000000000, -0.7071067811865475244008444, -0.8660254037844386467637232, -0.9659258262890682867497432, -1.000000000000000000000000, -0.9659258262890682867497432, -0.8660254037844386467637232, -0.7071067811865475244008444, -0.5000000000000000000000000, -0.2588190451025207623488988, 0.0, 0.2588190451025207623488988, 0.5000000000000000000000000, 0.7071067811865475244008444, 0.8660254037844386467637232, 0.9659258262890682867497432};
  return t[j];
}
template <> __device__ __forceinline__ constexpr double root_sin<24>(int j) {
  constexpr double t[24] = {0.0, 0.2588190451025207623488988, 0.5000000000000000000000000, 0.7071067811865475244008444, 0.8660254037844386467637232, 0.9659258262890682867497432, 1.000000000000000000000000, 0.9659258262890682867497432, 0.8660254037844386467637232, 0.7071067811865475244008444, 0.5000000000000000000000000, 0.2588190451025207623488988, 0.0, -0.2588190451025207623488988, -0.5000000000000000000000000, -0.7071067811865475244008444, -0.8660254037844386467637232, -0.9659258262890682867497432, -1.000000000000000000000000, -0.9659258262890682867497432, -0.8660254037844386467637232, -0.7071067811865475244008444, -0.5000000000000000000000000, -0.2588190451025207623488988};
  return t[j];
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

template <int R, bool INV, typename T> __device__ __forceinline__ void dft(T* v);

// v *= exp(-+2 pi i m / R) for a compile-time-known m (after unrolling);
// the four quarter turns are exact swaps / negations
template <int R, bool INV, typename T> __device__ __forceinline__ T twiddle_const(T v, int m) {
  typedef typename real_of<T>::type F;
  m %= R;
  if (m == 0) return v;
  if (4 * m == R) return mul_mi<INV>(v);
  if (2 * m == R) return mkc<T>(-v.x, -v.y);
  if (4 * m == 3 * R) return mul_mi<!INV>(v);
  const F c = F(root_cos<R>(m));
  const F s = INV ? F(root_sin<R>(m)) : F(-root_sin<R>(m));
  return mkc<T>(v.x * c - v.y * s, v.x * s + v.y * c);
}

// Cooley-Tukey on registers for R = A * B: x[n1 + A n2] -> X[k2 + B k1]
template <int A, int B, bool INV, typename T> __device__ __forceinline__ void dft_ab(T* v) {
  constexpr int R = A * B;
  T u[R];
#pragma unroll
  for (int n1 = 0; n1 < A; ++n1) {
    T t[B];
#pragma unroll
    for (int n2 = 0; n2 < B; ++n2) t[n2] = v[n1 + A * n2];
    dft<B, INV>(t);
#pragma unroll
    for (int k2 = 0; k2 < B; ++k2) u[n1 * B + k2] = twiddle_const<R, INV>(t[k2], n1 * k2);
  }
#pragma unroll
  for (int k2 = 0; k2 < B; ++k2) {
    T t[A];
#pragma unroll
    for (int n1 = 0; n1 < A; ++n1) t[n1] = u[n1 * B + k2];
    dft<A, INV>(t);
#pragma unroll
    for (int k1 = 0; k1 < A; ++k1) v[k2 + B * k1] = t[k1];
  }
}

template <int R, bool INV, typename T> __device__ __forceinline__ void dft(T* v) {
  if constexpr (R == 2) dft2<INV>(v);
  else if constexpr (R == 4) dft4<INV>(v);
  else if constexpr (R == 8) dft8<INV>(v);
  else if constexpr (R == 3 || R == 5 || R == 7) dft_odd<R, INV>(v);
  else if constexpr (R == 6) dft_ab<2, 3, INV>(v);
  else if constexpr (R == 9) dft_ab<3, 3, INV>(v);
  else if constexpr (R == 10) dft_ab<2, 5, INV>(v);
  else if constexpr (R == 12) dft_ab<4, 3, INV>(v);
  else if constexpr (R == 14) dft_ab<2, 7, INV>(v);
  else if constexpr (R == 16) dft_ab<4, 4, INV>(v);
  else if constexpr (R == 24) dft_ab<8, 3, INV>(v);
  else static_assert(R == 2, "unsupported radix");
}

// Per-axis FFT description, passed by value to the kernels.
struct AxisFFT {
  int M;                  // cyclic length
  int nst;                // number of radix stages
  int rad[kMaxStages];    // stage radices (DIF order)
  int blk[kMaxStages];    // sub-transform length entering each DIF stage
};

}  // namespace bdda
