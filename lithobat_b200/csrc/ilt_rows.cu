// Fused per-pixel passes of one ILT iteration (opc/ilt.py:576-596 with the
// objective of :311-336), for the configuration without blurs or penalties
// (sigma_px = 0, smooth = 0, weight_tv = weight_discrete = 0).
//
// An ILT step touches every pixel in two places: after the SOCS forward
// (image -> relaxed resist -> dJ/dI) and after the adjoint (dJ/dm -> dJ/dtheta
// -> Adam -> the next mask). Each becomes one pass over pixel rows that starts
// from a band box (the image's, or the gradient's) and ends with the band of
// the next spectrum (dJ/dI's, or the next mask's), so no per-pixel image,
// gradient or mask is written to HBM:
//
//   objective rows (MODE 0): I = synthesis of the image box (two rows per
//       complex 32-point FFT per residue, as rows.cu), fld = scale I,
//       s = sign (fld - level), z = sigmoid(a s) (clipped at +-60),
//       r = z - t, cost += r^2, perr += [s > 0] != [t > 0.5],
//       dJ/dI = sign (2 / N^2) r a z (1 - z); then the band-limited row DFT of
//       dJ/dI (band.cu's method) -> band rows [clip][k + bm][y].
//   update rows (MODE 1): g = synthesis of the gradient box (dJ/dm),
//       m = sigmoid(beta theta), q = g beta m (1 - m) (opc/ilt.py:381-389),
//       Adam on theta (:587-591), m' = sigmoid(beta' theta') (:368-378); then
//       the band row DFT of m' -> band rows of the next mask.
//
// N = 32 M with M in {8, 16, 32}; box half-width g0 <= 31; output band
// 2 bm + 1 <= 64. Every reduction is in a fixed order.
#include "common.cuh"

namespace litho {

__device__ __forceinline__ int band_kk(int kp, int p, int bm) { return -bm + ((kp + bm) & 31) + 32 * p; }

struct IltRowsArgs {
  const float2* box;   // [clip][(2 g0 + 1)^2]
  int g0;
  int bm;
  const float2* tw;    // exp(+2 pi i j / N)
  float2* band_out;    // [clip][2 bm + 1][N]
  // objective
  const float* target;
  float scale, level, sign, a, inv2;
  float* signed_out;
  double* cost_part;
  unsigned int* perr_part;
  // update
  float* theta;
  float* m1;
  float* m2;
  float beta, beta_next, step, b1, b2, eps, c1, c2;
  float* mask_out;
};

constexpr int kIrWarps = 8;
constexpr int kIrRows = 64;
constexpr int kIrG0Max = 31;

struct IltRowsSmem {
  int M, Lp, P, gp, G, Bm, npass, LD;
  size_t off_tbs, off_tbb, off_c, off_u, yw, zw, total;
};

__host__ __device__ inline IltRowsSmem ilt_rows_smem(int n, int g0, int bm) {
  IltRowsSmem s{};
  s.M = n >> 5;
  s.Lp = s.M < 32 ? s.M : 32;
  s.P = 32 / s.Lp;
  s.gp = g0 + 1;
  s.G = 2 * g0 + 1;
  s.Bm = 2 * bm + 1;
  s.npass = (s.Bm + 31) >> 5;
  s.LD = s.M + 1;
  s.off_tbs = 0;                                                     // [g][b] synthesis twiddles
  s.off_tbb = s.off_tbs + (size_t)s.gp * s.M * 8;                    // [pass][kp][b] band twiddles
  s.off_c = s.off_tbb + (size_t)s.npass * 32 * s.M * 8;              // [row][gx]
  s.off_u = s.off_c + (size_t)kIrRows * s.gp * 8;                    // box, then per-warp Y and Z
  s.yw = (size_t)s.P * 32 * s.LD;                                    // float2 per warp
  s.zw = (size_t)s.P * s.npass * 32;                                 // float2 per warp
  const size_t u_box = (size_t)s.G * s.G * 8, u_yz = (size_t)kIrWarps * (s.yw + s.zw) * 8;
  s.total = s.off_u + (u_box > u_yz ? u_box : u_yz);
  return s;
}

bool ilt_rows_ok(int n, int g0, int bm) {
  if (n != 256 && n != 512 && n != 1024) return false;
  if (g0 < 0 || g0 > kIrG0Max || bm < 0 || 2 * bm + 1 > 64) return false;
  return ilt_rows_smem(n, g0, bm).total <= 112 * 1024;
}

__device__ __forceinline__ float sigmoid60(float s) {
  s = fminf(fmaxf(s, -60.f), 60.f);
  return 1.0f / (1.0f + expf(-s));
}

template <int MODE, int M>
__global__ void __launch_bounds__(kIrWarps * 32, 2) k_ilt_rows(IltRowsArgs A) {
  constexpr int n = 32 * M, Lp = M < 32 ? M : 32, P = 32 / Lp, LD = M + 1;
  extern __shared__ __align__(16) unsigned char ir_raw[];
  const IltRowsSmem L = ilt_rows_smem(n, A.g0, A.bm);
  const int g0 = A.g0, gp = L.gp, G = L.G, bm = A.bm, Bm = L.Bm, npass = L.npass;
  const int clip = blockIdx.y, y0 = blockIdx.x * kIrRows;
  float2* TBS = reinterpret_cast<float2*>(ir_raw + L.off_tbs);
  float2* TBB = reinterpret_cast<float2*>(ir_raw + L.off_tbb);
  float2* C = reinterpret_cast<float2*>(ir_raw + L.off_c);
  float2* B = reinterpret_cast<float2*>(ir_raw + L.off_u);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float2* Y = reinterpret_cast<float2*>(ir_raw + L.off_u) + warp * (L.yw + L.zw);
  float2* Z = Y + L.yw;
  __shared__ double red_c[kIrWarps];
  __shared__ unsigned int red_p[kIrWarps];

  const float2* Bo = A.box + (size_t)clip * G * G;
  for (int j = threadIdx.x; j < G * G; j += blockDim.x) B[j] = Bo[j];
  for (int j = threadIdx.x; j < gp * M; j += blockDim.x) {
    const int g = j / M, b = j % M;
    TBS[j] = __ldg(A.tw + ((g * b) & (n - 1)));
  }
  for (int j = threadIdx.x; j < npass * 32 * M; j += blockDim.x) {
    const int p = j / (32 * M), kp = (j / M) & 31, b = j % M;
    const int k = band_kk(kp, p, bm);
    const float2 w = __ldg(A.tw + ((k * b) & (n - 1)));
    TBB[j] = k <= bm ? make_float2(w.x, -w.y) : make_float2(0.f, 0.f);   // exp(-2 pi i k b / N)
  }
  __syncthreads();
  for (int id = threadIdx.x; id < kIrRows * gp; id += blockDim.x) {
    const int r = id / gp, gx = id % gp, y = y0 + r;
    float2 acc = make_float2(0.f, 0.f);
    const float2* bc = B + gx + g0;
    for (int gy = -g0; gy <= g0; ++gy) acc = cadd(acc, cmul(bc[(gy + g0) * G], __ldg(A.tw + ((gy * y) & (n - 1)))));
    C[id] = acc;
  }
  __syncthreads();  // B is dead from here: its space holds Y and Z

  const int pg = lane / Lp, b = lane % Lp;
  double cost = 0.0;
  unsigned int perr = 0;
  constexpr int iters = kIrRows / (2 * kIrWarps * P);
  const float hs = 0.5f;
  for (int it = 0; it < iters; ++it) {
    const int pair = (it * kIrWarps + warp) * P + pg;
    const int ya = y0 + 2 * pair;
    const float2* c1 = C + (2 * pair) * gp;
    const float2* c2 = c1 + gp;
    float2 v[32];
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = make_float2(0.f, 0.f);
    {
      const float2 a1 = c1[0], a2 = c2[0];
      v[0] = make_float2(a1.x - a2.y, a1.y + a2.x);
    }
#pragma unroll
    for (int g = 1; g <= kIrG0Max; ++g) {
      if (g <= g0) {
        const float2 a1 = c1[g], a2 = c2[g];
        const float2 t = TBS[g * M + b];
        const float2 dp = make_float2(a1.x - a2.y, a1.y + a2.x);
        const float2 dm = make_float2(a1.x + a2.y, a2.x - a1.y);
        v[g & 31] = cadd(v[g & 31], cmul(dp, t));
        v[(-g) & 31] = cadd(v[(-g) & 31], cmulc(dm, t));
      }
    }
    fft_reg<32, +1>(v);   // v[a] = I(b + M a, ya) + i I(b + M a, ya + 1)
    const size_t row1 = ((size_t)clip * n + ya) * n, row2 = row1 + n;
    if (MODE == 0) {
      const float* __restrict__ tg = A.target;
      float* __restrict__ so = A.signed_out;
#pragma unroll
      for (int a0 = 0; a0 < 32; a0 += 8) {
        float t[8][2];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          t[j][0] = __ldg(tg + row1 + b + M * (a0 + j));
          t[j][1] = __ldg(tg + row2 + b + M * (a0 + j));
        }
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const int a = a0 + j;
          float d[2];
#pragma unroll
          for (int q = 0; q < 2; ++q) {
            const float I = q ? v[a].y : v[a].x;
            const float s = A.sign * (I * A.scale - A.level);
            const float z = sigmoid60(A.a * s);
            const float r = z - t[j][q];
            cost += (double)r * (double)r;
            perr += ((s > 0.f) != (t[j][q] > 0.5f)) ? 1u : 0u;
            d[q] = A.sign * (A.inv2 * r * (A.a * z * (1.0f - z)));
            if (so) so[(q ? row2 : row1) + b + M * a] = s;
          }
          v[a] = make_float2(d[0], d[1]);
        }
      }
    } else {
      float* __restrict__ tht = A.theta;
      float* __restrict__ mo1 = A.m1;
      float* __restrict__ mo2 = A.m2;
      float* __restrict__ mko = A.mask_out;
#pragma unroll
      for (int a0 = 0; a0 < 32; a0 += 4) {
        float th[4][2], u1[4][2], u2[4][2];
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
          for (int q = 0; q < 2; ++q) {
            const size_t i = (q ? row2 : row1) + b + M * (a0 + j);
            th[j][q] = tht[i];
            u1[j][q] = mo1[i];
            u2[j][q] = mo2[i];
          }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int a = a0 + j;
          float mo[2];
#pragma unroll
          for (int q = 0; q < 2; ++q) {
            const size_t i = (q ? row2 : row1) + b + M * a;
            const float gm = q ? v[a].y : v[a].x;
            float x = th[j][q];
            const float m = sigmoid60(A.beta * x);
            const float gi = gm * (A.beta * m * (1.f - m));
            const float am = A.b1 * u1[j][q] + (1.f - A.b1) * gi;
            const float av = A.b2 * u2[j][q] + (1.f - A.b2) * gi * gi;
            mo1[i] = am;
            mo2[i] = av;
            x -= A.step * (am / A.c1) / (sqrtf(av / A.c2) + A.eps);
            tht[i] = x;
            mo[q] = sigmoid60(A.beta_next * x);
            if (mko) mko[i] = mo[q];
          }
          v[a] = make_float2(mo[0], mo[1]);
        }
      }
    }
    // band row DFT of the two real rows held as one complex row
    fft_reg<32, -1>(v);
    for (int p = 0; p < npass; ++p) {
      const float2* tb = TBB + p * 32 * M + b;
      float2* yr = Y + pg * 32 * LD + b;
#pragma unroll
      for (int kp = 0; kp < 32; ++kp) yr[kp * LD] = cmul(v[kp], tb[kp * M]);
      __syncwarp();
      const int k = band_kk(lane, p, bm);
#pragma unroll
      for (int r = 0; r < P; ++r) {
        const float2* ys = Y + (r * 32 + lane) * LD;
        float2 s0 = make_float2(0.f, 0.f), s1 = make_float2(0.f, 0.f);
#pragma unroll
        for (int j = 0; j + 1 < M; j += 2) {
          s0 = cadd(s0, ys[j]);
          s1 = cadd(s1, ys[j + 1]);
        }
        if (k <= bm) Z[r * npass * 32 + (k + bm)] = cadd(s0, s1);
      }
      __syncwarp();
    }
#pragma unroll
    for (int r = 0; r < P; ++r) {
      const int yr0 = y0 + 2 * ((it * kIrWarps + warp) * P + r);
      const float2* zr = Z + r * npass * 32;
      for (int kk = lane; kk < Bm; kk += 32) {
        const float2 z = zr[kk], zm = zr[Bm - 1 - kk];   // Z(k), Z(-k)
        float2* dst = A.band_out + ((size_t)clip * Bm + kk) * n + yr0;
        dst[0] = make_float2((z.x + zm.x) * hs, (z.y - zm.y) * hs);
        dst[1] = make_float2((z.y + zm.y) * hs, (zm.x - z.x) * hs);
      }
    }
    __syncwarp();
  }
  if (MODE == 0) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      cost += __shfl_xor_sync(0xffffffffu, cost, o);
      perr += __shfl_xor_sync(0xffffffffu, perr, o);
    }
    if (lane == 0) {
      red_c[warp] = cost;
      red_p[warp] = perr;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double c = 0.0;
      unsigned int pe = 0;
      for (int w = 0; w < kIrWarps; ++w) {
        c += red_c[w];
        pe += red_p[w];
      }
      A.cost_part[(size_t)clip * gridDim.x + blockIdx.x] = c;
      A.perr_part[(size_t)clip * gridDim.x + blockIdx.x] = pe;
    }
  }
}

template <int MODE>
static cudaError_t launch_ilt_rows(const IltRowsArgs& A, int n, int n_fields, cudaStream_t s) {
  const IltRowsSmem L = ilt_rows_smem(n, A.g0, A.bm);
  const dim3 grid(n / kIrRows, n_fields);
  switch (n) {
    case 256:
      cudaFuncSetAttribute(k_ilt_rows<MODE, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.total);
      k_ilt_rows<MODE, 8><<<grid, kIrWarps * 32, L.total, s>>>(A);
      break;
    case 512:
      cudaFuncSetAttribute(k_ilt_rows<MODE, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.total);
      k_ilt_rows<MODE, 16><<<grid, kIrWarps * 32, L.total, s>>>(A);
      break;
    case 1024:
      cudaFuncSetAttribute(k_ilt_rows<MODE, 32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.total);
      k_ilt_rows<MODE, 32><<<grid, kIrWarps * 32, L.total, s>>>(A);
      break;
    default:
      return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_row_band_dft(const void* in, bool cplx, int n_rows, int rows_per_clip, int n, int bm,
                                float2* out, float scale, const float2* tw_inv, int num_sms, cudaStream_t st,
                                int* status);

static int sms_ir() {
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (sms <= 0) sms = 148;
  }
  return sms;
}

}  // namespace litho

using namespace litho;

// Workspace: status word + twiddle table.
static int64_t ilt_rows_ws(int n) { return align16(16) + align16((int64_t)n * 8); }

extern "C" int litho_ilt_rows_workspace(int n, size_t* bytes) {
  if (!bytes) return LITHO_E_NULL;
  if (n < 32) return LITHO_E_SIZE;
  *bytes = (size_t)ilt_rows_ws(n);
  return LITHO_OK;
}

extern "C" int litho_ilt_rows_supported(int n, int g0, int bm) { return ilt_rows_ok(n, g0, bm) ? 1 : 0; }

extern "C" int litho_ilt_objective_rows(const void* image_box, int g0, int n_fields, int n, const float* target,
                                        float scale, float level, float sign, float steepness_a, float* signed_out,
                                        double* cost_part, unsigned int* perr_part, int bm, void* band_rows_out,
                                        void* ws, size_t ws_bytes, cudaStream_t s) {
  if (!image_box || !target || !cost_part || !perr_part || !band_rows_out || !ws) return LITHO_E_NULL;
  if (n_fields < 1 || n_fields > 65535) return LITHO_E_SIZE;
  if (!ilt_rows_ok(n, g0, bm)) return LITHO_E_UNSUPPORTED;
  if ((int64_t)ws_bytes < ilt_rows_ws(n)) return LITHO_E_WORKSPACE;
  float2* tw = reinterpret_cast<float2*>(static_cast<char*>(ws) + align16(16));
  k_twiddle_table<<<(n + 255) / 256, 256, 0, s>>>(tw, n, +1);
  IltRowsArgs A{};
  A.box = static_cast<const float2*>(image_box);
  A.g0 = g0;
  A.bm = bm;
  A.tw = tw;
  A.band_out = static_cast<float2*>(band_rows_out);
  A.target = target;
  A.scale = scale;
  A.level = level;
  A.sign = sign;
  A.a = steepness_a;
  A.inv2 = (float)(2.0 / ((double)n * n));
  A.signed_out = signed_out;
  A.cost_part = cost_part;
  A.perr_part = perr_part;
  const cudaError_t e = launch_ilt_rows<0>(A, n, n_fields, s);
  return e == cudaSuccess ? LITHO_OK : (int)e;
}

extern "C" int litho_ilt_update_rows(const void* grad_box, int g0, int n_fields, int n, float* theta, float* m1,
                                     float* m2, float beta, float beta_next, float step, float b1, float b2,
                                     float eps, int it, float* mask_out, int bm, void* band_rows_out, void* ws,
                                     size_t ws_bytes, cudaStream_t s) {
  if (!grad_box || !theta || !m1 || !m2 || !band_rows_out || !ws) return LITHO_E_NULL;
  if (n_fields < 1 || n_fields > 65535 || it < 1) return LITHO_E_SIZE;
  if (!ilt_rows_ok(n, g0, bm)) return LITHO_E_UNSUPPORTED;
  if ((int64_t)ws_bytes < ilt_rows_ws(n)) return LITHO_E_WORKSPACE;
  float2* tw = reinterpret_cast<float2*>(static_cast<char*>(ws) + align16(16));
  k_twiddle_table<<<(n + 255) / 256, 256, 0, s>>>(tw, n, +1);
  IltRowsArgs A{};
  A.box = static_cast<const float2*>(grad_box);
  A.g0 = g0;
  A.bm = bm;
  A.tw = tw;
  A.band_out = static_cast<float2*>(band_rows_out);
  A.theta = theta;
  A.m1 = m1;
  A.m2 = m2;
  A.beta = beta;
  A.beta_next = beta_next;
  A.step = step;
  A.b1 = b1;
  A.b2 = b2;
  A.eps = eps;
  A.c1 = (float)(1.0 - pow((double)b1, it));
  A.c2 = (float)(1.0 - pow((double)b2, it));
  A.mask_out = mask_out;
  const cudaError_t e = launch_ilt_rows<1>(A, n, n_fields, s);
  return e == cudaSuccess ? LITHO_OK : (int)e;
}

// The column pass of a band spectrum whose row pass is done: rows [field][2bm+1][n]
// -> box [field][(2bm+1)^2] (times scale).
extern "C" int litho_band_columns(const void* band_rows, int n_fields, int n, int bm, float scale, void* box_out,
                                  void* ws, size_t ws_bytes, cudaStream_t s) {
  if (!band_rows || !box_out || !ws) return LITHO_E_NULL;
  if (n_fields < 1 || n < 32 || bm < 0) return LITHO_E_SIZE;
  if ((int64_t)ws_bytes < ilt_rows_ws(n)) return LITHO_E_WORKSPACE;
  int* status = static_cast<int*>(ws);
  float2* tw = reinterpret_cast<float2*>(static_cast<char*>(ws) + align16(16));
  cudaError_t e = cudaMemsetAsync(status, 0, sizeof(int), s);
  if (e != cudaSuccess) return (int)e;
  k_twiddle_table<<<(n + 255) / 256, 256, 0, s>>>(tw, n, +1);
  const int Bm = 2 * bm + 1;
  e = launch_row_band_dft(band_rows, true, n_fields * Bm, Bm, n, bm, static_cast<float2*>(box_out), scale, tw,
                          sms_ir(), s, status);
  return e == cudaSuccess ? LITHO_OK : (int)e;
}
