// Register-bound variants of the complex64 pencil kernels of the x=20
// particle's 192 x 224 x 350 grid: 3 and 4 resident CTAs of 256 threads per
// SM (at most 85 / 64 registers) for the latency-bound forward and inverse
// passes, 3 for the X pass.  The unbounded ones are in bdda_fixed_b.cu; the
// autotuner picks per pass.
#include "bdda_fixed.cuh"

namespace bdda {

static const FixedKernel kTableC[] = {
    BDDA_FIXED(float2, 1, K_CONV, 8, 3, 8, 8, 3, 1),
    BDDA_FIXED(float2, 1, K_FWD, 8, 3, 8, 7, 4, 1),
    BDDA_FIXED(float2, 1, K_INV, 8, 3, 8, 7, 4, 1),
    BDDA_FIXED(float2, 1, K_FWD, 8, 3, 10, 7, 5, 1),
    BDDA_FIXED(float2, 1, K_INV, 8, 3, 10, 7, 5, 1),
    BDDA_FIXED(float2, 1, K_FWD, 8, 4, 8, 7, 4, 1),
    BDDA_FIXED(float2, 1, K_INV, 8, 4, 8, 7, 4, 1),
    BDDA_FIXED(float2, 1, K_FWD, 8, 4, 10, 7, 5, 1),
    BDDA_FIXED(float2, 1, K_INV, 8, 4, 10, 7, 5, 1),
};

const FixedKernel* fixed_table_c(int* n) {
  *n = (int)(sizeof(kTableC) / sizeof(kTableC[0]));
  return kTableC;
}

}  // namespace bdda
