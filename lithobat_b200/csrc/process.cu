// Process-window helpers on top of the imaging path:
//   dose stacks — analysis/process_window.py:285-290: every dose of a
//       dose-focus sweep is a rescale of the raw Abbe sum of its focus,
//       out[f][d] = raw[f] * normalisation_scale(mode, peak[f], clear[f], dose[d])
//       (expose/aerial_image.py:217-241);
//   clamp — the clip to [0, 1] after PEB diffusion (bake/peb.py:65-66).
#include "common.cuh"

namespace litho {

__global__ void k_dose_stack(const float* __restrict__ raw, const float* __restrict__ peak,
                             const float* __restrict__ clear, int mode, long long npix,
                             const float* __restrict__ doses, int n_doses, float* __restrict__ out) {
  const int f = blockIdx.y / n_doses, d = blockIdx.y % n_doses;
  const float dose = doses[d];
  float s = dose;
  if (mode == 1) s = peak[f] > 0.f ? dose / peak[f] : dose;
  if (mode == 2) s = clear[f] > 0.f ? dose / clear[f] : dose;
  const float* src = raw + (size_t)f * npix;
  float* dst = out + ((size_t)f * n_doses + d) * npix;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < npix;
       i += (long long)gridDim.x * blockDim.x)
    dst[i] = src[i] * s;
}

__global__ void k_clamp(float* __restrict__ x, long long count, float lo, float hi) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count;
       i += (long long)gridDim.x * blockDim.x)
    x[i] = fminf(fmaxf(x[i], lo), hi);
}

}  // namespace litho

using namespace litho;

extern "C" int litho_dose_stack(const float* raw, const float* peak, const float* clear, int mode, int n_planes,
                                long long npix, const float* doses, int n_doses, float* out, cudaStream_t s) {
  if (!raw || !doses || !out || (mode == 1 && !peak) || (mode == 2 && !clear)) return LITHO_E_NULL;
  if (n_planes < 1 || n_doses < 1 || npix < 1 || (long long)n_planes * n_doses > 65535 || mode < 0 || mode > 2)
    return LITHO_E_SIZE;
  long long b = (npix + 255) / 256;
  if (b > 1024) b = 1024;
  k_dose_stack<<<dim3((unsigned)b, n_planes * n_doses), 256, 0, s>>>(raw, peak, clear, mode, npix, doses, n_doses,
                                                                      out);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? LITHO_OK : (int)e;
}

extern "C" int litho_clamp(float* x, long long count, float lo, float hi, cudaStream_t s) {
  if (!x) return LITHO_E_NULL;
  if (count < 0 || !(lo <= hi)) return LITHO_E_SIZE;
  long long b = (count + 255) / 256;
  if (b > 4096) b = 4096;
  if (b < 1) b = 1;
  k_clamp<<<(unsigned)b, 256, 0, s>>>(x, count, lo, hi);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? LITHO_OK : (int)e;
}
