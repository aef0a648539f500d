// Complex128 pencil kernels of the x=20 particle's 192 x 224 x 350 grid with
// CTA sizes other than 256 threads, chosen so that each stage's butterfly jobs
// fill whole rounds of threads (256 threads leave the X pass's radix-8 stages
// at 288 jobs = 1.125 rounds, i.e. 56 % busy): X pass [8,8,3] with 288
// threads, [8,7,4] with 384, [10,7,5] with 224.  The autotuner picks.
#include "bdda_fixed.cuh"

namespace bdda {

static const FixedKernel kTableD[] = {
    BDDA_FIXED_NT(double2, 0, K_CONV, 4, 2, 288, 8, 8, 3, 1),
    BDDA_FIXED_NT(double2, 0, K_CONV, 4, 3, 288, 8, 8, 3, 1),
    BDDA_FIXED_NT(double2, 0, K_FWD, 4, 2, 384, 8, 7, 4, 1),
    BDDA_FIXED_NT(double2, 0, K_INV, 4, 2, 384, 8, 7, 4, 1),
    BDDA_FIXED_NT(double2, 0, K_FWD, 4, 3, 224, 10, 7, 5, 1),
    BDDA_FIXED_NT(double2, 0, K_INV, 4, 3, 224, 10, 7, 5, 1),
    BDDA_FIXED_NT(double2, 0, K_FWD, 4, 4, 224, 10, 7, 5, 1),
    BDDA_FIXED_NT(double2, 0, K_INV, 4, 4, 224, 10, 7, 5, 1),
};

const FixedKernel* fixed_table_d(int* n) {
  *n = (int)(sizeof(kTableD) / sizeof(kTableD[0]));
  return kTableD;
}

}  // namespace bdda
