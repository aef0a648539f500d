// Complex64 pencil kernels of the x=20 particle's 192 x 224 x 350 grid with
// CTA sizes other than 256 threads: the X pass [8,8,3] at tile width 8 has
// 576 butterfly jobs per radix-8 stage (2.25 rounds of 256 threads; 3 of 192,
// 2 of 288), [10,7,5] fits 224 threads better.  The autotuner picks.
#include "bdda_fixed.cuh"

namespace bdda {

static const FixedKernel kTableE[] = {
    BDDA_FIXED_NT(float2, 1, K_CONV, 8, 5, 192, 8, 8, 3, 1),
    BDDA_FIXED_NT(float2, 1, K_CONV, 8, 3, 288, 8, 8, 3, 1),
    BDDA_FIXED_NT(float2, 1, K_FWD, 8, 4, 224, 10, 7, 5, 1),
    BDDA_FIXED_NT(float2, 1, K_INV, 8, 4, 224, 10, 7, 5, 1),
};

const FixedKernel* fixed_table_e(int* n) {
  *n = (int)(sizeof(kTableE) / sizeof(kTableE[0]));
  return kTableE;
}

}  // namespace bdda
