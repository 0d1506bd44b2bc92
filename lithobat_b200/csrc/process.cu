// Process-window helpers on top of the imaging path:
//   dose stacks — analysis/process_window.py:285-290: every dose of a
//       dose-focus sweep is a rescale of the raw Abbe sum of its focus,
//       out[f][d] = raw[f] * normalisation_scale(mode, peak[f], clear[f], dose[d])
//       (expose/aerial_image.py:217-241);
//   clamp — the clip to [0, 1] after PEB diffusion (bake/peb.py:65-66);
//   depth interpolation — develop/resist3d.py:176-183 (exposure_volume):
//       the optical planes through the resist film, linearly interpolated
//       along depth onto the voxel planes (np.interp per pixel), with each
//       voxel plane's interval and weight computed once on the host in FP64.
#include "common.cuh"

namespace litho {

// One (focus, dose) plane per blockIdx.y; VEC: four pixels per thread per
// iteration (npix % 4 == 0 and 16-byte aligned planes).
template <bool VEC>
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
  const long long stride = (long long)gridDim.x * blockDim.x;
  if (VEC) {
    const float4* s4 = reinterpret_cast<const float4*>(src);
    float4* d4 = reinterpret_cast<float4*>(dst);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < (npix >> 2); i += stride) {
      const float4 v = s4[i];
      __stcs(d4 + i, make_float4(v.x * s, v.y * s, v.z * s, v.w * s));
    }
  } else {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < npix; i += stride) dst[i] = src[i] * s;
  }
}

__global__ void k_clamp(float* __restrict__ x, long long count, float lo, float hi) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count;
       i += (long long)gridDim.x * blockDim.x)
    x[i] = fminf(fmaxf(x[i], lo), hi);
}

// out[v][p] = a[p] + w[v] (b[p] - a[p]) with a = planes[k[v].x], b =
// planes[k[v].y]: one voxel plane per blockIdx.y, the pixels grid-strided
// four at a time (VEC: npix % 4 == 0 and 16-byte aligned planes). A plane
// index outside [0, n_planes) leaves its voxel plane unwritten and sets
// LITHO_E_BAND in *status.
template <bool VEC>
__global__ void k_depth_interp(const float* __restrict__ planes, int n_planes, long long npix,
                               const int2* __restrict__ k, const float* __restrict__ w, float* __restrict__ out,
                               int* __restrict__ status) {
  const int v = blockIdx.y;
  const int2 kv = k[v];
  if (kv.x < 0 || kv.y < 0 || kv.x >= n_planes || kv.y >= n_planes) {
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicCAS(status, 0, LITHO_E_BAND);
    return;
  }
  const float wv = w[v];
  const float* a = planes + (size_t)kv.x * npix;
  const float* b = planes + (size_t)kv.y * npix;
  float* dst = out + (size_t)v * npix;
  const long long stride = (long long)gridDim.x * blockDim.x;
  if (VEC) {
    const float4* a4 = reinterpret_cast<const float4*>(a);
    const float4* b4 = reinterpret_cast<const float4*>(b);
    float4* d4 = reinterpret_cast<float4*>(dst);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < (npix >> 2); i += stride) {
      const float4 x = a4[i], y = b4[i];
      __stcs(d4 + i, make_float4(fmaf(wv, y.x - x.x, x.x), fmaf(wv, y.y - x.y, x.y), fmaf(wv, y.z - x.z, x.z),
                                 fmaf(wv, y.w - x.w, x.w)));
    }
  } else {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < npix; i += stride)
      dst[i] = fmaf(wv, b[i] - a[i], a[i]);
  }
}

}  // namespace litho

using namespace litho;

extern "C" int litho_dose_stack(const float* raw, const float* peak, const float* clear, int mode, int n_planes,
                                long long npix, const float* doses, int n_doses, float* out, cudaStream_t s) {
  if (!raw || !doses || !out || (mode == 1 && !peak) || (mode == 2 && !clear)) return LITHO_E_NULL;
  if (n_planes < 1 || n_doses < 1 || npix < 1 || (long long)n_planes * n_doses > 65535 || mode < 0 || mode > 2)
    return LITHO_E_SIZE;
  const bool vec = (npix & 3) == 0 && !((uintptr_t)raw & 15) && !((uintptr_t)out & 15);
  const int planes = n_planes * n_doses;
  long long b = ((vec ? npix >> 2 : npix) + 255) / 256;
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (sms <= 0) sms = 148;
  const long long cap = (8LL * sms + planes - 1) / planes;   // about 8 blocks per SM over all planes
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  if (vec)
    k_dose_stack<true><<<dim3((unsigned)b, planes), 256, 0, s>>>(raw, peak, clear, mode, npix, doses, n_doses, out);
  else
    k_dose_stack<false><<<dim3((unsigned)b, planes), 256, 0, s>>>(raw, peak, clear, mode, npix, doses, n_doses, out);
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

extern "C" int litho_depth_interp(const float* planes, int n_planes, long long npix, const int* k_dev,
                                  const float* w_dev, int n_out, float* out, int* status_dev, cudaStream_t s) {
  if (!planes || !k_dev || !w_dev || !out || !status_dev) return LITHO_E_NULL;
  if (n_planes < 1 || npix < 1 || n_out < 1 || n_out > 65535) return LITHO_E_SIZE;
  if (((uintptr_t)k_dev & 7) || ((uintptr_t)w_dev & 3)) return LITHO_E_ALIGN;
  const bool vec = (npix & 3) == 0 && !((uintptr_t)planes & 15) && !((uintptr_t)out & 15);
  const long long units = vec ? npix >> 2 : npix;
  long long b = (units + 255) / 256;
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (sms <= 0) sms = 148;
  const long long cap = (8LL * sms + n_out - 1) / n_out;   // about 8 blocks per SM over all voxel planes
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  const int2* k2 = reinterpret_cast<const int2*>(k_dev);
  if (vec)
    k_depth_interp<true><<<dim3((unsigned)b, n_out), 256, 0, s>>>(planes, n_planes, npix, k2, w_dev, out, status_dev);
  else
    k_depth_interp<false><<<dim3((unsigned)b, n_out), 256, 0, s>>>(planes, n_planes, npix, k2, w_dev, out,
                                                                    status_dev);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? LITHO_OK : (int)e;
}
