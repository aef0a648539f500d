// Specialised complex64 pencil kernels for the radix sequences of the
// shipped workloads: the x=20 particle's 192 x 224 x 350 grid ([8,8,3] X
// pass, [8,7,4] and [10,7,5] forward / inverse) and the x=5 sphere's 56^3
// grid ([7,4,2] X pass, [8,7] forward / inverse).
#include "bdda_fixed.cuh"

namespace bdda {

static const FixedKernel kTableB[] = {
    BDDA_FIXED(float2, 1, K_CONV, 8, 1, 8, 8, 3, 1),
    BDDA_FIXED(float2, 1, K_FWD, 8, 1, 8, 7, 4, 1),
    BDDA_FIXED(float2, 1, K_INV, 8, 1, 8, 7, 4, 1),
    BDDA_FIXED(float2, 1, K_FWD, 8, 1, 10, 7, 5, 1),
    BDDA_FIXED(float2, 1, K_INV, 8, 1, 10, 7, 5, 1),
    BDDA_FIXED(float2, 1, K_CONV, 8, 1, 7, 4, 2, 1),
    BDDA_FIXED(float2, 1, K_FWD, 8, 1, 8, 7, 1, 1),
    BDDA_FIXED(float2, 1, K_INV, 8, 1, 8, 7, 1, 1),
};

const FixedKernel* fixed_table_b(int* n) {
  *n = (int)(sizeof(kTableB) / sizeof(kTableB[0]));
  return kTableB;
}

}  // namespace bdda
