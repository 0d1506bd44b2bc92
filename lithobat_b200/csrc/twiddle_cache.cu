// Twiddle tables exp(+2 pi i j / n), j < n, for every power-of-two n in
// [2, 8192], built once per device and shared by every transform call.
//
// Each table is evaluated in FP64 (sincospi) and stored as FP32, exactly as
// k_twiddle_table fills a workspace table, so a kernel reads the same values
// either way. The tables live in one static device array (the table of n at
// [n, 2n)); the first call on a device outside a stream capture fills it on a
// private stream and waits for it, so any later call, on any stream, reads a
// finished table. A call that finds the array unbuilt while its stream is
// capturing, or asks for another size, gets nullptr and builds its own table
// in its workspace as before.
#include <mutex>

#include "common.cuh"

namespace litho {
namespace {

constexpr int kTwMax = 8192;
constexpr int kMaxDevices = 64;
__device__ __align__(16) float2 g_twiddles[2 * kTwMax];

std::mutex g_tw_mu;
const float2* g_tw_dev[kMaxDevices] = {nullptr};

__global__ void k_twiddle_all(float2* tab) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x + 2; i < 2 * kTwMax; i += gridDim.x * blockDim.x) {
    const int n = 1 << (31 - __clz(i));  // the table i belongs to: n <= i < 2n
    const int j = i - n;
    double s, c;
    sincospi(2.0 * (double)j / (double)n, &s, &c);
    tab[i] = make_float2((float)c, (float)s);
  }
}

}  // namespace

const float2* shared_twiddles(int n, cudaStream_t s) {
  if (n < 2 || n > kTwMax || (n & (n - 1))) return nullptr;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return nullptr;
  std::lock_guard<std::mutex> lock(g_tw_mu);
  if (!g_tw_dev[dev]) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return nullptr;
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_twiddles) != cudaSuccess || !p) return nullptr;
    cudaStream_t ps = nullptr;
    if (cudaStreamCreateWithFlags(&ps, cudaStreamNonBlocking) != cudaSuccess) return nullptr;
    k_twiddle_all<<<32, 256, 0, ps>>>(static_cast<float2*>(p));
    const bool ok = cudaGetLastError() == cudaSuccess && cudaStreamSynchronize(ps) == cudaSuccess;
    cudaStreamDestroy(ps);
    if (!ok) return nullptr;
    g_tw_dev[dev] = static_cast<const float2*>(p);
  }
  return g_tw_dev[dev] + n;
}

}  // namespace litho
