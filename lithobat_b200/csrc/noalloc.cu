// litho_abbe_noalloc: the Abbe image pipeline with no caller workspace.
//
// Some callers cannot allocate device memory for a workspace: a host process
// whose device memory is entirely pre-reserved by another allocator (a
// serving engine's memory pool, a framework's caching allocator it must not
// bypass), or a latency-critical loop that must never pay cudaMalloc's
// implicit device synchronisation. For them this entry point runs the same
// kernels as litho_abbe() on a fixed scratch buffer that lives in the
// library's own device image: a file-scope __device__ array of
// LITHO_NOALLOC_SCRATCH_BYTES, resident on every GPU that loads the library
// until the process exits.
//
// The array's name is only a host-side stand-in in host code; its device
// address is looked up once per device with cudaGetSymbolAddress (with that
// device current) on the first call made on the device, and cached.
#include <mutex>

#include "common.cuh"

namespace {

__device__ __align__(256) unsigned char g_noalloc_scratch[LITHO_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
void* g_scratch_dev[kMaxDevices] = {nullptr};
std::mutex g_scratch_mu;

// Device address of the scratch array on the current device (set-up on the
// first call per device). Returns a LITHO_* / CUDA status.
int scratch_for_current_device(void** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return (int)e;
  if (dev < 0 || dev >= kMaxDevices) return LITHO_E_DEVICE;
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_dev[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return (int)e;
    if (!p) return LITHO_E_DEVICE;
    g_scratch_dev[dev] = p;
  }
  *out = g_scratch_dev[dev];
  return LITHO_OK;
}

}  // namespace

extern "C" int litho_abbe_noalloc(const LithoAbbePlan* plan, const void* plan_blob_dev, const void* mask_dev,
                                  float* image_dev, float* peak_dev, cudaStream_t stream) {
  size_t need = 0;
  int st = litho_abbe_workspace(plan, &need);
  if (st) return st;
  if (need > (size_t)LITHO_NOALLOC_SCRATCH_BYTES) return LITHO_E_SCRATCH;
  void* scratch = nullptr;
  st = scratch_for_current_device(&scratch);
  if (st) return st;
  // litho_abbe clears the status word it keeps in the scratch and overwrites
  // every other byte it reads, so stale contents of a previous call are safe.
  return litho_abbe(plan, plan_blob_dev, mask_dev, image_dev, peak_dev, scratch,
                    (size_t)LITHO_NOALLOC_SCRATCH_BYTES, stream);
}

extern "C" int litho_abbe_noalloc_status(const LithoAbbePlan* plan, cudaStream_t stream) {
  void* scratch = nullptr;
  const int st = scratch_for_current_device(&scratch);
  if (st) return st;
  return litho_abbe_status(plan, scratch, stream);
}
