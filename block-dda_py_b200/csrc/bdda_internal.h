// Internal declarations shared by the translation units of libbdda.so.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "../../include/bdda.h"
#include "bdda_fft.cuh"

struct bdda_plan {
  int n[3];
  bdda::AxisFFT ax[3];
  // byte offsets into the device table buffer
  size_t tw64_off[3];   // double2[M]: exp(-2 pi i k / M)
  size_t tw32_off[3];   // float2[M]: the same, rounded
  size_t rev_off[3];    // int32[M]: stored position -> frequency index
  size_t err_off;       // uint32: bounded waits of the plan's kernels that gave up
  size_t table_bytes;
  std::vector<unsigned char> host_tables;
  void* dev_tables;
};

namespace bdda {

// Kernel launches issued by the library (all threads, all devices).
void count_launch(int n = 1);
// Optional per-pass timing of every block MVP (events on the launching stream).
bool profiling();
// pass 0..5: before Z, after Z, Y, X, Y^-1, Z^-1; prec tags the product (0 c128, 1 c64)
void profile_mark(int pass, cudaStream_t st, int prec = 0);

#define BDDA_CUDA_TRY(expr)                      \
  do {                                           \
    cudaError_t e_ = (expr);                     \
    if (e_ != cudaSuccess) return BDDA_CUDA_ERROR; \
  } while (0)

inline int64_t cells(const bdda_plan* p) { return (int64_t)p->n[0] * p->n[1] * p->n[2]; }
inline int64_t grid_points(const bdda_plan* p) {
  return (int64_t)p->ax[0].M * p->ax[1].M * p->ax[2].M;
}
inline size_t cplx_bytes(int prec) { return prec == BDDA_C64 ? 8 : 16; }

template <typename T>
inline const T* table_ptr(const bdda_plan* p, size_t off) {
  return reinterpret_cast<const T*>(static_cast<const unsigned char*>(p->dev_tables) + off);
}
inline unsigned int* plan_err(const bdda_plan* p) {
  return p->dev_tables ? reinterpret_cast<unsigned int*>(static_cast<unsigned char*>(p->dev_tables) + p->err_off)
                       : nullptr;
}

// Residual replacement drop and divergence factor of the mixed-form
// BiCGSTAB (bdda_tune_mixed).
double mixed_replace_drop();
double mixed_diverge_factor();

// Launch the block MVP in one precision (defined in bdda_mvp.cu).
template <typename T>
int block_mvp_impl(const bdda_plan* plan, int L, const T* ghat, const int32_t* cell_map,
                   const T* diag, const T* jpre, const T* S, T* out, T* work, cudaStream_t st);
// The complex64 block MVP of a complex128 vector: the Z pass gathers S
// rounding to complex64, the Z^-1 epilogue reads S the same way and writes
// out widened to complex128 (the same values as rounding S into a complex64
// copy and widening a complex64 result, without the copies).
int block_mvp_wide(const bdda_plan* plan, int L, const float2* ghat, const int32_t* cell_map, const float2* diag,
                   const float2* jpre, const double2* S, double2* out, float2* work, cudaStream_t st);

}  // namespace bdda
