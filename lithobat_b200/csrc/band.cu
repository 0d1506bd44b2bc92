// Band-limited forward DFT of the rows of a batch of N x N fields.
//
// out[clip][k + bm][i] = scale * sum_x in[clip][i][x] * exp(-2 pi i k x / N),
// for k in [-bm, bm]. The output is written transposed (frequency-major), so
// running the kernel twice — on the masks, then on its own output — gives the
// 2-D band spectrum M[ky][kx] of each clip: the thin-mask spectrum of
// expose/m3d/provider.py:ThinMaskSpectra (:177-178), restricted to the
// frequencies any source point's pupil can reach.
//
// Method (N = 32 M): x = b + M a. Each lane runs a 32-point FFT in registers
// over a for one residue b, multiplies by exp(-2 pi i k b / N) and the lanes
// of a row are summed through a per-warp shared-memory transpose:
//   U(k) = sum_b exp(-2 pi i k b / N) X_b(k mod 32).
// A warp covers 32/min(M,32) rows at a time, so every lane is busy for any
// N that is a multiple of 32.
#include "common.cuh"

namespace litho {

constexpr int kBandWarps = 4;

template <bool CPLX>
__global__ void __launch_bounds__(kBandWarps * 32)
k_row_band_dft(const void* __restrict__ in, int n_rows, int rows_per_clip, int n, int bm,
               float2* __restrict__ out, float scale, const float2* __restrict__ tw_inv) {
  extern __shared__ float2 smem[];
  float2* tw = smem;                                   // exp(+2 pi i j / n), j < n
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float2* tb = smem + n + warp * (32 * 33);            // per-warp 32 x 33 transpose buffer
  for (int j = threadIdx.x; j < n; j += blockDim.x) tw[j] = tw_inv[j];
  __syncthreads();

  const int M = n >> 5;
  const int Mp = M < 32 ? M : 32;          // lanes per row
  const int G = 32 / Mp;                   // rows per warp pass
  const int per_lane = M / Mp;             // residues b per lane
  const int Bm = 2 * bm + 1;
  const int r_loc = lane / Mp, bl = lane % Mp;
  const int wmin = -((bm + 31) >> 5), wmax = (bm + 31) >> 5;
  const int total_warps = gridDim.x * kBandWarps;

  for (int rg = blockIdx.x * kBandWarps + warp; rg * G < n_rows; rg += total_warps) {
    const int row = rg * G + r_loc;
    const bool active = row < n_rows;
    float2 v[32];
    int have = -1;  // residue index q whose transform v holds
    // Accumulate sum_b X_b(k') * exp(-2 pi i (k' + 32 w) b / n) per wrap w.
    for (int w = wmin; w <= wmax; ++w) {
      // does any k = k' + 32 w fall in [-bm, bm]?
      if (32 * w + 31 < -bm || 32 * w > bm) continue;
#pragma unroll 1
      for (int c = 0; c < 32; ++c) tb[c * 33 + lane] = make_float2(0.f, 0.f);
      __syncwarp();
      for (int q = 0; q < per_lane; ++q) {
        const int b = bl + q * Mp;
        if (have != q) {
        have = q;
        if (active) {
          if (CPLX) {
            const float2* src = reinterpret_cast<const float2*>(in) + (size_t)row * n + b;
#pragma unroll
            for (int a = 0; a < 32; ++a) v[a] = __ldg(src + (size_t)a * M);
          } else {
            const float* src = reinterpret_cast<const float*>(in) + (size_t)row * n + b;
#pragma unroll
            for (int a = 0; a < 32; ++a) v[a] = make_float2(__ldg(src + (size_t)a * M), 0.f);
          }
        } else {
#pragma unroll
          for (int a = 0; a < 32; ++a) v[a] = make_float2(0.f, 0.f);
        }
        fft_reg<32, -1>(v);
        }
#pragma unroll
        for (int kp = 0; kp < 32; ++kp) {
          const int k = kp + 32 * w;
          int t = (int)(((long long)k * b) % n);
          t = t < 0 ? -t : (t == 0 ? 0 : n - t);       // exponent -k b mod n
          const float2 y = cmul(v[kp], tw[t]);
          float2 acc = tb[kp * 33 + lane];
          tb[kp * 33 + lane] = cadd(acc, y);
        }
      }
      __syncwarp();
      // lane kp sums over the residues of each of the G rows
      for (int r = 0; r < G; ++r) {
        float2 s = make_float2(0.f, 0.f);
        for (int j = 0; j < Mp; ++j) s = cadd(s, tb[lane * 33 + r * Mp + j]);
        const int orow = rg * G + r;
        const int k = lane + 32 * w;
        if (orow < n_rows && k >= -bm && k <= bm) {
          const int clip = orow / rows_per_clip, i = orow % rows_per_clip;
          out[((size_t)clip * Bm + (k + bm)) * rows_per_clip + i] = cscale(s, scale);
        }
      }
      __syncwarp();
    }
  }
}

// Fallback for N not a multiple of 32: one thread per (row, k), direct sum.
template <bool CPLX>
__global__ void k_row_band_direct(const void* __restrict__ in, int n_rows, int rows_per_clip, int n,
                                  int bm, float2* __restrict__ out, float scale,
                                  const float2* __restrict__ tw_inv) {
  const int Bm = 2 * bm + 1;
  const long long total = (long long)n_rows * Bm;
  for (long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x; id < total;
       id += (long long)gridDim.x * blockDim.x) {
    const int row = (int)(id / Bm), k = (int)(id % Bm) - bm;
    float2 s = make_float2(0.f, 0.f);
    for (int x = 0; x < n; ++x) {
      int t = (int)(((long long)k * x) % n);
      t = t < 0 ? -t : (t == 0 ? 0 : n - t);
      float2 v = CPLX ? reinterpret_cast<const float2*>(in)[(size_t)row * n + x]
                      : make_float2(reinterpret_cast<const float*>(in)[(size_t)row * n + x], 0.f);
      s = cadd(s, cmul(v, tw_inv[t]));
    }
    const int clip = row / rows_per_clip, i = row % rows_per_clip;
    out[((size_t)clip * Bm + (k + bm)) * rows_per_clip + i] = cscale(s, scale);
  }
}

__global__ void k_twiddle_table(float2* w, int n, int sign) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    double s, c;
    sincospi(2.0 * (double)j / (double)n, &s, &c);
    w[j] = make_float2((float)c, (float)(sign * s));
  }
}

size_t band_dft_smem(int n) { return (size_t)(n + kBandWarps * 32 * 33) * sizeof(float2); }

// Launch the row-band DFT for n_rows rows (grouped rows_per_clip per clip).
cudaError_t launch_row_band_dft(const void* in, bool cplx, int n_rows, int rows_per_clip, int n,
                                int bm, float2* out, float scale, const float2* tw_inv,
                                int num_sms, cudaStream_t st) {
  if (n % 32 == 0) {
    const int M = n / 32, Mp = M < 32 ? M : 32, G = 32 / Mp;
    const int warps = (n_rows + G - 1) / G;
    int blocks = (warps + kBandWarps - 1) / kBandWarps;
    const int cap = num_sms * 16;
    if (blocks > cap) blocks = cap;
    const size_t sm = band_dft_smem(n);
    if (cplx) {
      cudaFuncSetAttribute(k_row_band_dft<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
      k_row_band_dft<true><<<blocks, kBandWarps * 32, sm, st>>>(in, n_rows, rows_per_clip, n, bm,
                                                                out, scale, tw_inv);
    } else {
      cudaFuncSetAttribute(k_row_band_dft<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
      k_row_band_dft<false><<<blocks, kBandWarps * 32, sm, st>>>(in, n_rows, rows_per_clip, n, bm,
                                                                 out, scale, tw_inv);
    }
  } else {
    const long long total = (long long)n_rows * (2 * bm + 1);
    int blocks = (int)((total + 255) / 256);
    if (blocks > num_sms * 32) blocks = num_sms * 32;
    if (cplx)
      k_row_band_direct<true><<<blocks, 256, 0, st>>>(in, n_rows, rows_per_clip, n, bm, out, scale, tw_inv);
    else
      k_row_band_direct<false><<<blocks, 256, 0, st>>>(in, n_rows, rows_per_clip, n, bm, out, scale, tw_inv);
  }
  return cudaGetLastError();
}

}  // namespace litho
