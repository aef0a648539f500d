// Two-stage X-pass kernels (bdda_xconv.cuh) for the x=20 particle's 192-point
// x axis, plan radices [8,8,3], as 24 x 8: complex128 and complex64 at two
// tile widths and both intermediate layouts, with and without the TMA-filled
// tile.  The autotuner times them beside the plan-stage kernels.
#include "bdda_xconv.cuh"

namespace bdda {

static const FixedKernel kTableJ[] = {
    BDDA_XCONV2(double2, 0, 8, 2, 192, 24, 8, 8, 8, 3, 1, 0),
    BDDA_XCONV2(double2, 0, 8, 2, 192, 24, 8, 8, 8, 3, 0, 0),
    BDDA_XCONV2(double2, 0, 8, 2, 192, 24, 8, 8, 8, 3, 1, 1),
    BDDA_XCONV2(double2, 0, 4, 3, 96, 24, 8, 8, 8, 3, 1, 0),
    BDDA_XCONV2(float2, 1, 8, 3, 192, 24, 8, 8, 8, 3, 1, 0),
    BDDA_XCONV2(float2, 1, 8, 3, 192, 24, 8, 8, 8, 3, 1, 1),
    BDDA_XCONV2(float2, 1, 8, 3, 192, 24, 8, 8, 8, 3, 0, 1),
    BDDA_XCONV2(float2, 1, 4, 4, 96, 24, 8, 8, 8, 3, 1, 1),
};

const FixedKernel* fixed_table_j(int* n) {
  *n = (int)(sizeof(kTableJ) / sizeof(kTableJ[0]));
  return kTableJ;
}

}  // namespace bdda
