// Block MVP for callers that cannot allocate device memory.
//
// bdda_block_mvp needs a scratch field buffer of bdda_mvp_workspace_bytes()
// that the caller allocates.  Some callers cannot call cudaMalloc: a plugin
// hosted by an application whose own allocator owns every byte of device
// memory and forbids libraries from allocating behind its back, or code on a
// latency-critical path that cannot accept the device-wide synchronisation
// cudaMalloc / cudaFree may imply.  bdda_block_mvp_noalloc runs the same
// product with its scratch in a fixed static device array instead.
//
// Costs and rules of that array:
//  - it is kNoAllocScratchBytes (64 MiB) and every GPU that loads this
//    library holds it until the process exits;
//  - every call on a device shares it, so calls that overlap on the GPU (on
//    different streams, or from different host threads) race on it; run them
//    one after another;
//  - it keeps whatever the last call left; nothing in it has to start at
//    zero, because each product writes every scratch element before reading it;
//  - the first call on a device looks up the array's device address with that
//    device current (cudaGetSymbolAddress); make that first call before any
//    stream capture.  The address is kept for the life of the process, so
//    cudaDeviceReset on a device that has called this entry point is not
//    supported (the reset unloads the array; a later call would use a stale
//    address).
#include <mutex>

#include "bdda_internal.h"

namespace {

constexpr size_t kNoAllocScratchBytes = (size_t)64 << 20;
__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
void* g_noalloc_addr[kMaxDevices] = {};

// Device address of the scratch array on the current device, set up once per device.
int noalloc_scratch(void** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return BDDA_CUDA_ERROR;
  if (dev < 0 || dev >= kMaxDevices) return BDDA_BAD_ARG;
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_addr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return BDDA_CUDA_ERROR;
    g_noalloc_addr[dev] = p;
  }
  *out = g_noalloc_addr[dev];
  return BDDA_OK;
}

}  // namespace

extern "C" {

size_t bdda_block_mvp_noalloc_max_bytes(void) { return kNoAllocScratchBytes; }

int bdda_block_mvp_noalloc_fits(const bdda_plan* plan, int prec, int L) {
  if (!plan || L < 1) return 0;
  const size_t need = bdda_mvp_workspace_bytes(plan, prec, L);
  return need > 0 && need <= kNoAllocScratchBytes ? 1 : 0;
}

int bdda_block_mvp_noalloc(const bdda_plan* plan, int prec, int L, const void* ghat, const int32_t* cell_map,
                           const void* diag, const void* jpre, const void* S, void* out, void* stream) {
  if (!plan || L < 1) return BDDA_BAD_ARG;
  if (!bdda_block_mvp_noalloc_fits(plan, prec, L)) return BDDA_BAD_ARG;   // scratch would not hold the field
  if (!ghat || !cell_map || !diag || !jpre || !S || !out) return BDDA_BAD_ARG;
  void* scratch = nullptr;
  const int s = noalloc_scratch(&scratch);
  if (s != BDDA_OK) return s;
  return bdda_block_mvp(plan, prec, L, ghat, cell_map, diag, jpre, S, out, scratch, stream);
}

}  // extern "C"
