// Column-pair complex64 kernels of the forward and inverse Y and Z passes of
// the x=20 particle's 192 x 224 x 350 grid ([8,7,4] and [10,7,5] at tile
// width 8).  The autotuner picks among these and the one-column kernels.
#include "bdda_fixed.cuh"

namespace bdda {

static const FixedKernel kTableG[] = {
    BDDA_FIXED_PAIR(1, K_FWD, 8, 3, 256, 8, 7, 4, 1),
    BDDA_FIXED_PAIR(1, K_INV, 8, 3, 256, 8, 7, 4, 1),
    BDDA_FIXED_PAIR(1, K_FWD, 8, 4, 192, 8, 7, 4, 1),
    BDDA_FIXED_PAIR(1, K_INV, 8, 4, 192, 8, 7, 4, 1),
    BDDA_FIXED_PAIR(1, K_FWD, 8, 3, 224, 10, 7, 5, 1),
    BDDA_FIXED_PAIR(1, K_INV, 8, 3, 224, 10, 7, 5, 1),
    BDDA_FIXED_PAIR(1, K_INV, 8, 4, 224, 10, 7, 5, 1),
};

const FixedKernel* fixed_table_g(int* n) {
  *n = (int)(sizeof(kTableG) / sizeof(kTableG[0]));
  return kTableG;
}

}  // namespace bdda
