// Bounded device waits: the test hooks of the failure reporting.
//
// Every wait inside a kernel on an mbarrier (bulk copies landing, tensor-core
// MMAs completing) is bounded by a clock budget; a wait that gives up records
// LITHO_E_TIMEOUT in the status word of the call's workspace, drains what its
// block already has in flight, and lets the block exit. These two entry
// points let a test exercise that path without faulting or hanging a GPU.
#include "common.cuh"

namespace litho {
cudaError_t set_wait_limit_band(long long cycles);
cudaError_t set_wait_limit_synth(long long cycles);
cudaError_t set_wait_limit_gram(long long cycles);
cudaError_t set_wait_limit_queue(long long cycles);

// One thread waits, within `cycles`, on an mbarrier that nothing arrives at,
// and records the outcome the way the pipeline kernels do.
__global__ void k_wait_probe(int* status, long long cycles) {
  __shared__ uint64_t bar;
  if (threadIdx.x != 0) return;
  mbar_init(&bar, 1);
  fence_mbar_init();
  if (!mbar_wait_for(&bar, 0, cycles)) atomicExch(status, LITHO_E_TIMEOUT);
}
}  // namespace litho

using namespace litho;

extern "C" int litho_set_wait_limit(long long cycles) {
  if (cycles < 0) return LITHO_E_SIZE;
  const long long c = cycles == 0 ? kWaitCycles : cycles;
  cudaError_t e;
  if ((e = set_wait_limit_band(c)) != cudaSuccess) return (int)e;
  if ((e = set_wait_limit_synth(c)) != cudaSuccess) return (int)e;
  if ((e = set_wait_limit_gram(c)) != cudaSuccess) return (int)e;
  if ((e = set_wait_limit_queue(c)) != cudaSuccess) return (int)e;
  return LITHO_OK;
}

extern "C" int litho_wait_probe(int* status_dev, long long cycles, cudaStream_t s) {
  if (!status_dev) return LITHO_E_NULL;
  if (cycles < 1 || cycles > kWaitCycles) return LITHO_E_SIZE;
  if ((uintptr_t)status_dev & 3) return LITHO_E_ALIGN;
  k_wait_probe<<<1, 32, 0, s>>>(status_dev, cycles);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? LITHO_OK : (int)e;
}
