// Specialised complex128 pencil kernels for the radix sequences of the
// shipped workloads: the x=20 particle's 192 x 224 x 350 grid ([8,8,3] X
// pass, [8,7,4] and [10,7,5] forward / inverse) and the x=5 sphere's 56^3
// grid ([7,4,2] X pass, [8,7] forward / inverse).  Each is compiled with two
// register bounds (3 and 4 resident CTAs per SM); the autotuner picks.
#include "bdda_fixed.cuh"

namespace bdda {

#define BDDA_FIXED2(KIND, LT, R0, R1, R2, R3) \
  BDDA_FIXED(double2, 0, KIND, LT, 3, R0, R1, R2, R3), BDDA_FIXED(double2, 0, KIND, LT, 4, R0, R1, R2, R3)

static const FixedKernel kTableA[] = {
    BDDA_FIXED2(K_CONV, 4, 8, 8, 3, 1),
    BDDA_FIXED2(K_FWD, 4, 8, 7, 4, 1),
    BDDA_FIXED2(K_INV, 4, 8, 7, 4, 1),
    BDDA_FIXED2(K_FWD, 4, 10, 7, 5, 1),
    BDDA_FIXED2(K_INV, 4, 10, 7, 5, 1),
    BDDA_FIXED2(K_CONV, 8, 7, 4, 2, 1),
    BDDA_FIXED2(K_FWD, 8, 8, 7, 1, 1),
    BDDA_FIXED2(K_INV, 8, 8, 7, 1, 1),
};

const FixedKernel* fixed_table_a(int* n) {
  *n = (int)(sizeof(kTableA) / sizeof(kTableA[0]));
  return kTableA;
}

}  // namespace bdda
