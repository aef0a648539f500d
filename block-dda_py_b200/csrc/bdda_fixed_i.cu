// Pencil kernels whose tile is filled by a bulk tensor copy (TMA) instead of
// the first stage's global loads: the dense-source passes of the x=20
// particle's 192 x 224 x 350 grid (Y and Y^-1 [8,7,4], X [8,8,3], Z^-1
// [10,7,5]), at the CTA shapes of their plain counterparts.  Measured per
// pass by the autotuner against those.
#include "bdda_fixed.cuh"

namespace bdda {

static const FixedKernel kTableI[] = {
    // complex64, column pairs, tile width 8
    BDDA_FIXED_TMA_PAIR(1, K_FWD, 8, 3, 256, 8, 7, 4, 1),
    BDDA_FIXED_TMA_PAIR(1, K_FWD, 8, 4, 192, 8, 7, 4, 1),
    BDDA_FIXED_TMA_PAIR(1, K_INV, 8, 3, 256, 8, 7, 4, 1),
    BDDA_FIXED_TMA_PAIR(1, K_INV, 8, 4, 192, 8, 7, 4, 1),
    BDDA_FIXED_TMA_PAIR(1, K_INV, 8, 3, 224, 10, 7, 5, 1),
    BDDA_FIXED_TMA_PAIR(1, K_INV, 8, 4, 224, 10, 7, 5, 1),
    BDDA_FIXED_TMA_PAIR(1, K_CONV, 8, 4, 160, 8, 8, 3, 1),
    BDDA_FIXED_TMA_PAIR(1, K_CONV, 8, 3, 192, 8, 8, 3, 1),
    // complex128, tile width 4 (and 8 for the X pass)
    BDDA_FIXED_TMA_NT(double2, 0, K_FWD, 4, 2, 384, 8, 7, 4, 1),
    BDDA_FIXED_TMA_NT(double2, 0, K_INV, 4, 2, 384, 8, 7, 4, 1),
    BDDA_FIXED_TMA(double2, 0, K_FWD, 4, 4, 8, 7, 4, 1),
    BDDA_FIXED_TMA(double2, 0, K_INV, 4, 4, 8, 7, 4, 1),
    BDDA_FIXED_TMA(double2, 0, K_FWD, 4, 3, 8, 7, 4, 1),
    BDDA_FIXED_TMA(double2, 0, K_INV, 4, 3, 8, 7, 4, 1),
    BDDA_FIXED_TMA_NT(double2, 0, K_INV, 4, 3, 224, 10, 7, 5, 1),
    BDDA_FIXED_TMA_NT(double2, 0, K_CONV, 4, 2, 288, 8, 8, 3, 1),
    BDDA_FIXED_TMA_NT(double2, 0, K_CONV, 8, 2, 288, 8, 8, 3, 1),
};

const FixedKernel* fixed_table_i(int* n) {
  *n = (int)(sizeof(kTableI) / sizeof(kTableI[0]));
  return kTableI;
}

}  // namespace bdda
