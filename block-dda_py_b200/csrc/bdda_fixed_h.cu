// X-pass kernels of the x=20 particle's 192 x 224 x 350 grid ([8,8,3]) with
// wider column tiles: complex128 at tile width 8 (24 columns) and complex64
// column pairs at tile width 16 (48 columns).  A wider tile stages the
// pencil's twiddles and Green's tensor entries (6 per frequency) once for
// more right-hand sides; it holds fewer CTAs per SM.  The autotuner times
// them beside the narrower tiles and keeps the fastest.
#include "bdda_fixed.cuh"

namespace bdda {

static const FixedKernel kTableH[] = {
    BDDA_FIXED_NT(double2, 0, K_CONV, 8, 2, 288, 8, 8, 3, 1),
    BDDA_FIXED_NT(double2, 0, K_CONV, 8, 2, 192, 8, 8, 3, 1),
    BDDA_FIXED_PAIR(1, K_CONV, 16, 2, 288, 8, 8, 3, 1),
    BDDA_FIXED_PAIR(1, K_CONV, 16, 2, 192, 8, 8, 3, 1),
};

const FixedKernel* fixed_table_h(int* n) {
  *n = (int)(sizeof(kTableH) / sizeof(kTableH[0]));
  return kTableH;
}

}  // namespace bdda
