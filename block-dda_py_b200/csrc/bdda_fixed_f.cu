// Column-pair complex64 kernels of the X pass of the x=20 particle's
// 192 x 224 x 350 grid, radices [8,8,3] at tile width 8: a radix-8 stage has
// 288 pair jobs (one round of 288 threads, three of 96), the Green middle
// 256.  Pair jobs take about 90 registers; the CTA sizes below let four CTAs
// (the shared-memory limit) or two of 288 threads stay resident without
// spilling.  CTA sizes are whole warps: the variant id counts warps.  The
// autotuner picks among these and the one-column kernels.
#include "bdda_fixed.cuh"

namespace bdda {

static const FixedKernel kTableF[] = {
    BDDA_FIXED_PAIR(1, K_CONV, 8, 1, 288, 8, 8, 3, 1),
    BDDA_FIXED_PAIR(1, K_CONV, 8, 4, 160, 8, 8, 3, 1),
    BDDA_FIXED_PAIR(1, K_CONV, 8, 5, 96, 8, 8, 3, 1),
    BDDA_FIXED_PAIR(1, K_CONV, 8, 4, 128, 8, 8, 3, 1),
    BDDA_FIXED_PAIR(1, K_CONV, 8, 3, 192, 8, 8, 3, 1),
};

const FixedKernel* fixed_table_f(int* n) {
  *n = (int)(sizeof(kTableF) / sizeof(kTableF[0]));
  return kTableF;
}

}  // namespace bdda
