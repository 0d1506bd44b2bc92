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
#include "fftwarp.cuh"

namespace litho {


// Pass p handles, for each residue k' = k mod 32, the p-th frequency of
// [-bm, bm] congruent to k' (in increasing order from -bm).
__device__ __forceinline__ int band_k(int kp, int p, int bm) {
  return -bm + ((kp + bm) & 31) + 32 * p;
}

// Shared-memory plan of one block of k_row_band_tma.
struct BandSmem {
  int warps, G, ld, tile_rows;
  size_t tile_bytes, off_stage1, off_tw, off_y, total;
};

__host__ __device__ inline BandSmem band_smem(int n, int esz, int warps) {
  BandSmem b{};
  const int M = n >> 5, Mp = M < 32 ? M : 32, per = M / Mp;
  b.warps = warps;
  b.G = 32 / Mp;
  b.ld = Mp * per + 1;
  b.tile_rows = warps * b.G;
  b.tile_bytes = (size_t)b.tile_rows * n * esz;
  b.off_stage1 = 16 + b.tile_bytes;
  b.off_tw = 16 + 2 * b.tile_bytes;
  b.off_y = b.off_tw + (size_t)n * sizeof(float2);
  b.total = b.off_y + (size_t)warps * b.G * 32 * b.ld * sizeof(float2);
  return b;
}

// Rows arrive in tiles of `tile_rows` contiguous rows through a two-stage
// TMA pipeline (one elected thread issues cp.async.bulk; consumers wait on
// the stage's mbarrier); every warp owns G rows of a tile.
template <bool CPLX>
__global__ void __launch_bounds__(128)
k_row_band_tma(const void* __restrict__ in, int n_rows, int rows_per_clip, int n, int bm,
               float2* __restrict__ out, float scale, const float2* __restrict__ tw_inv,
               int* __restrict__ status) {
  extern __shared__ __align__(128) unsigned char smraw[];
  const int esz = CPLX ? 8 : 4;
  const BandSmem L = band_smem(n, esz, blockDim.x >> 5);
  const int M = n >> 5;
  const int Mp = M < 32 ? M : 32;
  const int per_lane = M / Mp;
  const int G = L.G, ld = L.ld;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint64_t* mbar = reinterpret_cast<uint64_t*>(smraw);
  unsigned char* stage[2] = {smraw + 16, smraw + L.off_stage1};
  float2* tw = reinterpret_cast<float2*>(smraw + L.off_tw);
  float2* Y = reinterpret_cast<float2*>(smraw + L.off_y) + warp * (G * 32 * ld);
  __shared__ int s_fail;

  const int n_tiles = (n_rows + L.tile_rows - 1) / L.tile_rows;
  int n_issued[2] = {0, 0};   // copies thread 0 has issued into each stage
  auto issue = [&](int t, int st) {
    ++n_issued[st];
    const int r0 = t * L.tile_rows;
    const int rows = (n_rows - r0) < L.tile_rows ? (n_rows - r0) : L.tile_rows;
    const uint32_t bytes = (uint32_t)((size_t)rows * n * esz);
    mbar_expect_tx(&mbar[st], bytes);
    bulk_g2s(stage[st], static_cast<const unsigned char*>(in) + (size_t)r0 * n * esz, bytes, &mbar[st]);
  };
  if (threadIdx.x == 0) {
    s_fail = 0;
    mbar_init(&mbar[0], 1);
    mbar_init(&mbar[1], 1);
    fence_mbar_init();
  }
  for (int j = threadIdx.x; j < n; j += blockDim.x) tw[j] = tw_inv[j];
  __syncthreads();
  if (threadIdx.x == 0) {
    if ((int)blockIdx.x < n_tiles) issue(blockIdx.x, 0);
    if ((int)(blockIdx.x + gridDim.x) < n_tiles) issue(blockIdx.x + gridDim.x, 1);
  }

  const int Bm = 2 * bm + 1;
  const int npass = (Bm + 31) >> 5;
  const int r_loc = lane / Mp, bl = lane % Mp;
  const bool pow2 = (n & (n - 1)) == 0;
  int it = 0;
  for (int t = blockIdx.x; t < n_tiles; t += gridDim.x, ++it) {
    const int st = it & 1;
    if (!mbar_wait(&mbar[st], (it >> 1) & 1)) atomicExch(&s_fail, 1);
    __syncthreads();
    if (s_fail) break;  // uniform: every thread saw the same flag
    const unsigned char* tile = stage[st];
    const int row_in_tile = warp * G + r_loc;
    const int row = t * L.tile_rows + row_in_tile;
    const bool active = row < n_rows;
    for (int p = 0; p < npass; ++p) {
      for (int q = 0; q < per_lane; ++q) {
        const int b = bl + q * Mp;
        float2 v[32];
        if (active) {
          if (CPLX) {
            const float2* src = reinterpret_cast<const float2*>(tile) + (size_t)row_in_tile * n + b;
#pragma unroll
            for (int a = 0; a < 32; ++a) v[a] = src[a * M];
          } else {
            const float* src = reinterpret_cast<const float*>(tile) + (size_t)row_in_tile * n + b;
#pragma unroll
            for (int a = 0; a < 32; ++a) v[a] = make_float2(src[a * M], 0.f);
          }
        } else {
#pragma unroll
          for (int a = 0; a < 32; ++a) v[a] = make_float2(0.f, 0.f);
        }
        fft_reg<32, -1>(v);
        float2* yr = Y + (r_loc * 32) * ld + b;
#pragma unroll
        for (int kp = 0; kp < 32; ++kp) {
          const int k = band_k(kp, p, bm);
          const int e = -k * b;  // |e| < 2^24
          const int tt = pow2 ? (e & (n - 1)) : ((e % n) + n) % n;
          yr[kp * ld] = k <= bm ? cmul(v[kp], tw[tt]) : make_float2(0.f, 0.f);
        }
      }
      __syncwarp();
      const int k = band_k(lane, p, bm);
      for (int r = 0; r < G; ++r) {
        const float2* yr = Y + (r * 32 + lane) * ld;
        float2 s0 = make_float2(0.f, 0.f), s1 = make_float2(0.f, 0.f);
        int j = 0;
        for (; j + 1 < M; j += 2) {
          s0 = cadd(s0, yr[j]);
          s1 = cadd(s1, yr[j + 1]);
        }
        if (j < M) s0 = cadd(s0, yr[j]);
        const int orow = t * L.tile_rows + warp * G + r;
        if (orow < n_rows && k <= bm) {
          const int clip = orow / rows_per_clip, i = orow % rows_per_clip;
          out[((size_t)clip * Bm + (k + bm)) * rows_per_clip + i] = cscale(cadd(s0, s1), scale);
        }
      }
      __syncwarp();
    }
    __syncthreads();  // stage st fully consumed
    if (threadIdx.x == 0 && t + 2 * (int)gridDim.x < n_tiles) {
      fence_proxy_async();
      issue(t + 2 * gridDim.x, st);
    }
  }
  if (s_fail) {
    // drain: the latest copy into each stage (parity of its last phase; a
    // stage is refilled only after its previous copy was consumed) lands
    // before the block exits, then report
    if (threadIdx.x == 0) {
      for (int sg = 0; sg < 2; ++sg)
        if (n_issued[sg] > 0) mbar_wait_drain(&mbar[sg], (uint32_t)((n_issued[sg] - 1) & 1));
      atomicExch(status, LITHO_E_TIMEOUT);
    }
  }
}

// ---------------------------------------------------------------------------
// Register-direct variant for power-of-two N in [32, 2048] (the common case).
// Each lane loads the 32 samples of its residue b with coalesced loads
// straight into registers (a warp reads 32 consecutive elements per load), so
// no staging buffer limits the number of resident warps; the 32-point FFT
// result stays in registers across the passes over the band. Real rows go two
// at a time as one complex row z = r1 + i r2 and are separated on the band:
// R1(k) = (Z(k) + conj Z(-k)) / 2, R2(k) = (Z(k) - conj Z(-k)) / 2i.
// ---------------------------------------------------------------------------
struct BandGeo {
  int M, Lp, P, q, ld, gp, Bm, npass, warps;
  bool tb_smem;                                    // per-pass twiddle table in shared memory
  size_t y_per_warp, z_per_warp, off_y, off_z, total;
};

__host__ __device__ inline BandGeo band_geo(int n, int bm, int warps) {
  BandGeo g{};
  g.M = n >> 5;
  g.Lp = g.M < 32 ? g.M : 32;
  g.P = 32 / g.Lp;
  g.q = g.M / g.Lp;
  g.ld = g.M + 1;
  g.gp = band_group_pitch(g.M);
  g.Bm = 2 * bm + 1;
  g.npass = (g.Bm + 31) >> 5;
  g.warps = warps;
  g.y_per_warp = (size_t)g.P * g.gp;               // float2
  g.z_per_warp = (size_t)g.P * g.npass * 32;       // float2
  g.tb_smem = (size_t)g.npass * 32 * g.M * 8 <= 64 * 1024;
  g.off_y = g.tb_smem ? (size_t)g.npass * 32 * g.M * 8 : 0;   // after the twiddle table
  g.off_z = g.off_y + (size_t)warps * g.y_per_warp * 8;
  g.total = g.off_z + (size_t)warps * g.z_per_warp * 8;
  return g;
}

// M = N / 32 is a template constant, so every shared-memory offset below is
// an immediate; the twiddle table is laid out per (pass, register kp, residue
// b) with zeros where band_k(kp, pass) falls outside the band.
// LEV (with CPLX): the input is a level map, one byte per pixel indexing the
// row's clip's levels[clip][0 .. n_levels), complex; an index past the table
// takes the last level.
// LEV2 (real path): a two-level map, m = L0 + (L1 - L0) b with b = [index >=
// 1] real, so two rows of b go through one complex transform (as real rows
// do) and each band value is (L1 - L0) B(k) + L0 N [k = 0]: half the
// transforms of the complex level path, the same spectrum to rounding.
template <bool CPLX, int M, bool TBS, bool LEV = false, bool LEV2 = false>
__global__ void __launch_bounds__(256, 2)
k_band_rows(const void* __restrict__ in, int n_rows, int rows_per_clip, int bm, float2* __restrict__ out,
            float scale, const float2* __restrict__ tw_inv, const float2* __restrict__ levels = nullptr,
            int n_levels = 0) {
  static_assert(!LEV || CPLX, "level maps are complex inputs");
  static_assert(!LEV2 || !CPLX, "two-level maps take the real path");
  constexpr int n = 32 * M, Lp = M < 32 ? M : 32, P = 32 / Lp, Q = M / Lp, LD = M + 1;
  extern __shared__ __align__(16) float2 bsm[];
  const BandGeo g = band_geo(n, bm, blockDim.x >> 5);
  const int Bm = g.Bm, npass = g.npass;
  float2* TB = bsm;                                        // [pass][kp][b] = w^(-k b) or 0
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  constexpr int GP = band_group_pitch(M);
  float2* Y = bsm + g.off_y / 8 + warp * g.y_per_warp;   // [group (pitch GP)][kp (pitch LD)][b]
  float2* Z = bsm + g.off_z / 8 + warp * g.z_per_warp;   // [group][k + bm] (real pairs)
  if (TBS) {
    for (int j = threadIdx.x; j < npass * 32 * M; j += blockDim.x) {
      const int p = j / (32 * M), kp = (j / M) & 31, b = j % M;
      const int k = band_k(kp, p, bm);
      TB[j] = k <= bm ? tw_inv[(-k * b) & (n - 1)] : make_float2(0.f, 0.f);
    }
  }
  __syncthreads();
  const int pg = lane / Lp, bl = lane % Lp;
  constexpr int rows_per_iter = CPLX ? P : 2 * P;
  const int n_iter = (n_rows + rows_per_iter - 1) / rows_per_iter;
  for (int wi = blockIdx.x * g.warps + warp; wi < n_iter; wi += gridDim.x * g.warps) {
    const int row0 = wi * rows_per_iter;
    const int r1 = CPLX ? row0 + pg : row0 + 2 * pg;
    const bool live = r1 < n_rows;
    float2 v[32];
    for (int p = 0; p < npass; ++p) {
#pragma unroll
      for (int qq = 0; qq < Q; ++qq) {
        const int b = bl + qq * Lp;
        if (p == 0 || Q > 1) {
          if (live) {
            if (LEV) {
              const uint8_t* src = static_cast<const uint8_t*>(in) + (size_t)r1 * n + b;
              const float2* lv = levels + (size_t)(r1 / rows_per_clip) * n_levels;
              uint32_t q[32];
#pragma unroll
              for (int a = 0; a < 32; ++a) q[a] = __ldcs(src + M * a);
              if (n_levels <= 4) {   // the row's levels in registers: selects, no dependent loads
                const float2 l0 = __ldg(lv), l1 = n_levels > 1 ? __ldg(lv + 1) : l0;
                const float2 l2 = n_levels > 2 ? __ldg(lv + 2) : l1, l3 = n_levels > 3 ? __ldg(lv + 3) : l2;
#pragma unroll
                for (int a = 0; a < 32; ++a) {
                  const uint32_t k = q[a];
                  const float2 lo = k == 0u ? l0 : l1, hi = k == 2u ? l2 : l3;
                  v[a] = k < 2u ? lo : hi;
                }
              } else {
#pragma unroll
                for (int a = 0; a < 32; ++a)
                  v[a] = __ldg(lv + (q[a] < (uint32_t)n_levels ? q[a] : n_levels - 1));
              }
            } else if (CPLX) {
              const float2* src = static_cast<const float2*>(in) + (size_t)r1 * n + b;
#pragma unroll
              for (int a = 0; a < 32; ++a) v[a] = __ldcs(src + M * a);
            } else if (LEV2) {
              const uint8_t* s1 = static_cast<const uint8_t*>(in) + (size_t)r1 * n + b;
#pragma unroll
              for (int a = 0; a < 32; ++a)
                v[a] = make_float2(__ldcs(s1 + M * a) ? 1.f : 0.f, __ldcs(s1 + n + M * a) ? 1.f : 0.f);
            } else {
              const float* s1 = static_cast<const float*>(in) + (size_t)r1 * n + b;
#pragma unroll
              for (int a = 0; a < 32; ++a) v[a] = make_float2(__ldcs(s1 + M * a), __ldcs(s1 + n + M * a));
            }
          } else {
#pragma unroll
            for (int a = 0; a < 32; ++a) v[a] = make_float2(0.f, 0.f);
          }
          fft_reg<32, -1>(v);
        }
        float2* yr = Y + pg * GP + b;
        if (TBS) {
          const float2* tb = TB + p * 32 * M + b;
#pragma unroll
          for (int kp = 0; kp < 32; ++kp) yr[kp * LD] = cmul(v[kp], tb[kp * M]);
        } else {  // wide bands: twiddles from the global table (L1-resident)
#pragma unroll
          for (int kp = 0; kp < 32; ++kp) {
            const int k = band_k(kp, p, bm);
            yr[kp * LD] = k <= bm ? cmul(v[kp], __ldg(tw_inv + ((-k * b) & (n - 1)))) : make_float2(0.f, 0.f);
          }
        }
      }
      __syncwarp();
      const int k = band_k(lane, p, bm);
#pragma unroll
      for (int r = 0; r < P; ++r) {
        const float2* yr = Y + r * GP + lane * LD;
        float2 s0 = make_float2(0.f, 0.f), s1 = make_float2(0.f, 0.f);
#pragma unroll
        for (int j = 0; j + 1 < M; j += 2) {
          s0 = cadd(s0, yr[j]);
          s1 = cadd(s1, yr[j + 1]);
        }
        if (M & 1) s0 = cadd(s0, yr[M - 1]);
        const float2 sum = cadd(s0, s1);
        if (k <= bm) {
          if (CPLX) {
            const int row = row0 + r;
            if (row < n_rows) {
              const int clip = row / rows_per_clip, i = row % rows_per_clip;
              out[((size_t)clip * Bm + (k + bm)) * rows_per_clip + i] = cscale(sum, scale);
            }
          } else {
            Z[r * npass * 32 + (k + bm)] = sum;
          }
        }
      }
      __syncwarp();
    }
    if (!CPLX) {
      const float hs = 0.5f * scale;
#pragma unroll
      for (int r = 0; r < P; ++r) {
        const int ra = row0 + 2 * r;
        if (ra < n_rows) {
          const int clip = ra / rows_per_clip, i = ra % rows_per_clip;
          const float2* zr = Z + r * npass * 32;
          float2 dl = make_float2(0.f, 0.f), l0n = make_float2(0.f, 0.f);
          if (LEV2) {   // this clip's L1 - L0 and L0 N scale (the DC term of the constant L0)
            const float2 a0 = __ldg(levels + (size_t)clip * 2), a1 = __ldg(levels + (size_t)clip * 2 + 1);
            dl = make_float2(a1.x - a0.x, a1.y - a0.y);
            l0n = make_float2(a0.x * (float)n * scale, a0.y * (float)n * scale);
          }
          for (int kk = lane; kk < Bm; kk += 32) {
            const float2 z = zr[kk], zm = zr[Bm - 1 - kk];       // Z(k), Z(-k)
            float2 o1 = make_float2((z.x + zm.x) * hs, (z.y - zm.y) * hs);
            float2 o2 = make_float2((z.y + zm.y) * hs, (zm.x - z.x) * hs);
            if (LEV2) {
              o1 = cmul(dl, o1);
              o2 = cmul(dl, o2);
              if (kk == bm) {
                o1 = cadd(o1, l0n);
                o2 = cadd(o2, l0n);
              }
            }
            float2* dst = out + ((size_t)clip * Bm + kk) * rows_per_clip + i;
            dst[0] = o1;
            dst[1] = o2;
          }
        }
      }
      __syncwarp();
    }
  }
}

template <bool CPLX, int M, bool LEV = false, bool LEV2 = false>
static cudaError_t launch_band_rows_m(const void* in, int n_rows, int rows_per_clip, int bm, float2* out,
                                      float scale, const float2* tw_inv, int num_sms, cudaStream_t st,
                                      const float2* levels = nullptr, int n_levels = 0) {
  const int n = 32 * M;
  const int warps = n <= 1024 ? 8 : 4;
  const BandGeo g = band_geo(n, bm, warps);
  if (g.total > 200 * 1024) return cudaErrorInvalidValue;
  const int rows_per_iter = CPLX ? g.P : 2 * g.P;
  const long long n_iter = ((long long)n_rows + rows_per_iter - 1) / rows_per_iter;
  const int per_sm = (int)((227 * 1024) / g.total) >= 2 ? 2 : 1;
  long long blocks = (n_iter + warps - 1) / warps;
  if (blocks > (long long)num_sms * per_sm) blocks = (long long)num_sms * per_sm;
  if (LEV2) {   // two-level maps: the real path, table in shared memory
    if (!g.tb_smem) return cudaErrorInvalidValue;
    cudaFuncSetAttribute(k_band_rows<false, M, true, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)g.total);
    k_band_rows<false, M, true, false, true><<<(int)blocks, warps * 32, g.total, st>>>(
        in, n_rows, rows_per_clip, bm, out, scale, tw_inv, levels, n_levels);
  } else if (LEV) {   // level maps: the common (table in shared memory) form only
    if (!g.tb_smem) return cudaErrorInvalidValue;
    cudaFuncSetAttribute(k_band_rows<true, M, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)g.total);
    k_band_rows<true, M, true, true><<<(int)blocks, warps * 32, g.total, st>>>(in, n_rows, rows_per_clip, bm, out,
                                                                               scale, tw_inv, levels, n_levels);
  } else if (g.tb_smem) {
    cudaFuncSetAttribute(k_band_rows<CPLX, M, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)g.total);
    k_band_rows<CPLX, M, true><<<(int)blocks, warps * 32, g.total, st>>>(in, n_rows, rows_per_clip, bm, out, scale,
                                                                         tw_inv);
  } else {  // wide bands: a separate instantiation, so the common path keeps its registers
    cudaFuncSetAttribute(k_band_rows<CPLX, M, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)g.total);
    k_band_rows<CPLX, M, false><<<(int)blocks, warps * 32, g.total, st>>>(in, n_rows, rows_per_clip, bm, out, scale,
                                                                          tw_inv);
  }
  return cudaGetLastError();
}

template <bool CPLX>
static cudaError_t launch_band_rows(const void* in, int n_rows, int rows_per_clip, int n, int bm, float2* out,
                                    float scale, const float2* tw_inv, int num_sms, cudaStream_t st) {
  switch (n) {
    case 32: return launch_band_rows_m<CPLX, 1>(in, n_rows, rows_per_clip, bm, out, scale, tw_inv, num_sms, st);
    case 64: return launch_band_rows_m<CPLX, 2>(in, n_rows, rows_per_clip, bm, out, scale, tw_inv, num_sms, st);
    case 128: return launch_band_rows_m<CPLX, 4>(in, n_rows, rows_per_clip, bm, out, scale, tw_inv, num_sms, st);
    case 256: return launch_band_rows_m<CPLX, 8>(in, n_rows, rows_per_clip, bm, out, scale, tw_inv, num_sms, st);
    case 512: return launch_band_rows_m<CPLX, 16>(in, n_rows, rows_per_clip, bm, out, scale, tw_inv, num_sms, st);
    case 1024: return launch_band_rows_m<CPLX, 32>(in, n_rows, rows_per_clip, bm, out, scale, tw_inv, num_sms, st);
    case 2048: return launch_band_rows_m<CPLX, 64>(in, n_rows, rows_per_clip, bm, out, scale, tw_inv, num_sms, st);
    default: return cudaErrorInvalidValue;
  }
}

// Wide bands (the residue method's twiddle table outgrows shared memory):
// full transforms of each row with the warp-per-line register FFT. With
// SPLIT = N / L sub-sequences x_j(i) = x(j + SPLIT i) (L <= 1024 points each),
//     U(k) = sum_j exp(-2 pi i j k / N) F_j(k mod L),
// so a row costs SPLIT L-point FFTs; the band [-bm, bm] (2 bm + 1 <= L) meets
// each residue k mod L at most once. The partial sums live in a per-warp
// shared-memory array while the sub-transforms run.
constexpr int kBfWarps = 4;

__host__ __device__ inline size_t bandfft_smem(int L) {
  return (size_t)L * 8 + (size_t)kBfWarps * 32 * kTbLd * 8 + (size_t)kBfWarps * 32 * 32 * 8;
}

template <bool CPLX, int L, int SPLIT>
__global__ void __launch_bounds__(kBfWarps * 32)
k_band_rows_fft(const void* __restrict__ in, int n_rows, int rows_per_clip, int bm, float2* __restrict__ out,
                float scale, const float2* __restrict__ tw_inv) {
  constexpr int R = L / 32, LPW = 32 / R, N = L * SPLIT;
  extern __shared__ float2 bf_sm[];
  float2* tw = bf_sm;  // exp(+2 pi i j / L)
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float2* tb = bf_sm + L + warp * 32 * kTbLd;
  float2* acc = bf_sm + L + kBfWarps * 32 * kTbLd + warp * 32 * 32;  // [s][lane]
  fill_lane_twiddles(tw, L, tw_inv, SPLIT);
  __syncthreads();
  const int Bm = 2 * bm + 1;
  const int lp = lane / R, rp = lane % R;
  for (long long r0 = ((long long)blockIdx.x * kBfWarps + warp) * LPW; r0 < n_rows;
       r0 += (long long)gridDim.x * kBfWarps * LPW) {
#pragma unroll 1
    for (int j = 0; j < SPLIT; ++j) {
      float2 x[32];
#pragma unroll
      for (int l = 0; l < LPW; ++l) {
        const long long row = r0 + l;
#pragma unroll
        for (int q = 0; q < R; ++q) {
          const size_t e = (size_t)row * N + j + SPLIT * (lane + 32 * q);
          float2 v = make_float2(0.f, 0.f);
          if (row < n_rows) {
            if (CPLX) v = __ldg(reinterpret_cast<const float2*>(in) + e);
            else v.x = __ldg(reinterpret_cast<const float*>(in) + e);
          }
          x[l * R + q] = v;
        }
      }
      warp_fft_lines<L, -1>(x, tb, tw);  // lane: row r0 + lp, k' = rp + R s
#pragma unroll
      for (int sidx = 0; sidx < 32; ++sidx) {
        const int kp = rp + R * sidx;
        const int k = kp <= bm ? kp : kp - L;  // the band value with residue kp, if any
        float2 v = x[sidx];
        if (SPLIT > 1 && j > 0) {
          const float2 w = __ldg(tw_inv + ((j * k) & (N - 1)));
          v = cmulc(v, w);  // times exp(-2 pi i j k / N)
          v = cadd(v, acc[sidx * 32 + lane]);
        }
        acc[sidx * 32 + lane] = v;
      }
    }
    const long long row = r0 + lp;
    if (row >= n_rows) continue;
    const long long clip = row / rows_per_clip, i = row % rows_per_clip;
#pragma unroll
    for (int sidx = 0; sidx < 32; ++sidx) {
      const int kp = rp + R * sidx;
      if (kp <= bm || kp >= L - bm) {
        const int k = kp <= bm ? kp : kp - L;
        out[((size_t)clip * Bm + (k + bm)) * rows_per_clip + i] = cscale(acc[sidx * 32 + lane], scale);
      }
    }
  }
}

template <bool CPLX, int L, int SPLIT>
static cudaError_t launch_band_fft_l(const void* in, int n_rows, int rows_per_clip, int bm, float2* out,
                                     float scale, const float2* tw_inv, int num_sms, cudaStream_t st) {
  constexpr int R = L / 32, LPW = 32 / R;
  const size_t sm = bandfft_smem(L);
  cudaFuncSetAttribute(k_band_rows_fft<CPLX, L, SPLIT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  long long blocks = ((long long)n_rows + kBfWarps * LPW - 1) / (kBfWarps * LPW);
  const long long cap = (long long)num_sms * 3;
  if (blocks > cap) blocks = cap;
  k_band_rows_fft<CPLX, L, SPLIT><<<(int)blocks, kBfWarps * 32, sm, st>>>(in, n_rows, rows_per_clip, bm, out, scale,
                                                                          tw_inv);
  return cudaGetLastError();
}

// N in {256 .. 4096} (power of two), 2 bm + 1 <= min(N, 1024).
template <bool CPLX>
static cudaError_t launch_band_fft(const void* in, int n_rows, int rows_per_clip, int n, int bm, float2* out,
                                   float scale, const float2* tw_inv, int num_sms, cudaStream_t st) {
  switch (n) {
    case 256: return launch_band_fft_l<CPLX, 256, 1>(in, n_rows, rows_per_clip, bm, out, scale, tw_inv, num_sms, st);
    case 512: return launch_band_fft_l<CPLX, 512, 1>(in, n_rows, rows_per_clip, bm, out, scale, tw_inv, num_sms, st);
    case 1024: return launch_band_fft_l<CPLX, 1024, 1>(in, n_rows, rows_per_clip, bm, out, scale, tw_inv, num_sms, st);
    case 2048: return launch_band_fft_l<CPLX, 1024, 2>(in, n_rows, rows_per_clip, bm, out, scale, tw_inv, num_sms, st);
    case 4096: return launch_band_fft_l<CPLX, 1024, 4>(in, n_rows, rows_per_clip, bm, out, scale, tw_inv, num_sms, st);
    default: return cudaErrorInvalidValue;
  }
}

static bool band_fft_ok(int n, int bm) {
  const int L = n < 1024 ? n : 1024;
  return n >= 256 && n <= 4096 && (n & (n - 1)) == 0 && 2 * bm + 1 <= L;
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
      const int t = ((-k * x) % n + n) % n;
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

// Launch the row-band DFT for n_rows rows (grouped rows_per_clip per clip).
// The first band pass of a level map (uint8 [clip][n][n] indexing levels
// [clip][n_levels]): powers of two n in [32, 2048] whose band twiddles fit
// shared memory; cudaErrorInvalidValue otherwise.
cudaError_t launch_row_band_dft_levels(const uint8_t* in, const float2* levels, int n_levels, int n_rows,
                                       int rows_per_clip, int n, int bm, float2* out, float scale,
                                       const float2* tw_inv, int num_sms, cudaStream_t st) {
  if (!levels || n_levels < 1) return cudaErrorInvalidValue;
  if (n_levels == 2 && rows_per_clip % 2 == 0 && n_rows % 2 == 0) {
    switch (n) {
      case 32: return launch_band_rows_m<false, 1, false, true>(in, n_rows, rows_per_clip, bm, out, scale, tw_inv,
                                                                num_sms, st, levels, 2);
      case 64: return launch_band_rows_m<false, 2, false, true>(in, n_rows, rows_per_clip, bm, out, scale, tw_inv,
                                                                num_sms, st, levels, 2);
      case 128: return launch_band_rows_m<false, 4, false, true>(in, n_rows, rows_per_clip, bm, out, scale, tw_inv,
                                                                 num_sms, st, levels, 2);
      case 256: return launch_band_rows_m<false, 8, false, true>(in, n_rows, rows_per_clip, bm, out, scale, tw_inv,
                                                                 num_sms, st, levels, 2);
      case 512: return launch_band_rows_m<false, 16, false, true>(in, n_rows, rows_per_clip, bm, out, scale, tw_inv,
                                                                  num_sms, st, levels, 2);
      case 1024: return launch_band_rows_m<false, 32, false, true>(in, n_rows, rows_per_clip, bm, out, scale,
                                                                   tw_inv, num_sms, st, levels, 2);
      case 2048: return launch_band_rows_m<false, 64, false, true>(in, n_rows, rows_per_clip, bm, out, scale,
                                                                   tw_inv, num_sms, st, levels, 2);
      default: return cudaErrorInvalidValue;
    }
  }
  switch (n) {
    case 32: return launch_band_rows_m<true, 1, true>(in, n_rows, rows_per_clip, bm, out, scale, tw_inv, num_sms, st,
                                                      levels, n_levels);
    case 64: return launch_band_rows_m<true, 2, true>(in, n_rows, rows_per_clip, bm, out, scale, tw_inv, num_sms, st,
                                                      levels, n_levels);
    case 128: return launch_band_rows_m<true, 4, true>(in, n_rows, rows_per_clip, bm, out, scale, tw_inv, num_sms,
                                                       st, levels, n_levels);
    case 256: return launch_band_rows_m<true, 8, true>(in, n_rows, rows_per_clip, bm, out, scale, tw_inv, num_sms,
                                                       st, levels, n_levels);
    case 512: return launch_band_rows_m<true, 16, true>(in, n_rows, rows_per_clip, bm, out, scale, tw_inv, num_sms,
                                                        st, levels, n_levels);
    case 1024: return launch_band_rows_m<true, 32, true>(in, n_rows, rows_per_clip, bm, out, scale, tw_inv, num_sms,
                                                         st, levels, n_levels);
    case 2048: return launch_band_rows_m<true, 64, true>(in, n_rows, rows_per_clip, bm, out, scale, tw_inv, num_sms,
                                                         st, levels, n_levels);
    default: return cudaErrorInvalidValue;
  }
}

bool row_band_levels_ok(int n, int bm) {
  const bool pow2 = n >= 32 && n <= 2048 && (n & (n - 1)) == 0;
  return pow2 && band_geo(n, bm, n <= 1024 ? 8 : 4).tb_smem && band_geo(n, bm, n <= 1024 ? 8 : 4).total <= 200 * 1024;
}

cudaError_t launch_row_band_dft(const void* in, bool cplx, int n_rows, int rows_per_clip, int n,
                                int bm, float2* out, float scale, const float2* tw_inv,
                                int num_sms, cudaStream_t st, int* status) {
  const int esz = cplx ? 8 : 4;
  const int M = n >> 5;
  const bool pow2 = n >= 32 && (n & (n - 1)) == 0;
  const bool wide = pow2 && n >= 256 && (n > 2048 || !band_geo(n, bm, n <= 1024 ? 8 : 4).tb_smem);
  if (wide && band_fft_ok(n, bm)) {
    // wide bands: full row transforms (the residue method's twiddle table would not fit)
    const cudaError_t e = cplx ? launch_band_fft<true>(in, n_rows, rows_per_clip, n, bm, out, scale, tw_inv, num_sms, st)
                               : launch_band_fft<false>(in, n_rows, rows_per_clip, n, bm, out, scale, tw_inv, num_sms,
                                                        st);
    if (e != cudaSuccess) return e;
  } else if (n >= 32 && n <= 2048 && (n & (n - 1)) == 0 && (cplx || (rows_per_clip % 2 == 0 && n_rows % 2 == 0))) {
    const cudaError_t e = cplx ? launch_band_rows<true>(in, n_rows, rows_per_clip, n, bm, out, scale, tw_inv, num_sms, st)
                               : launch_band_rows<false>(in, n_rows, rows_per_clip, n, bm, out, scale, tw_inv, num_sms,
                                                         st);
    if (e != cudaSuccess) return e;
  } else if (n % 32 == 0 && (32 % M == 0 || M % 32 == 0) && ((uintptr_t)in & 15) == 0) {
    // TMA-staged variant: the residue layout needs M to divide 32 or 32 to divide M
    int warps = 4;
    while (warps > 1 && band_smem(n, esz, warps).total > 200 * 1024) warps >>= 1;
    const BandSmem L = band_smem(n, esz, warps);
    if (L.total > 227 * 1024) return cudaErrorInvalidValue;
    const int tiles = (n_rows + L.tile_rows - 1) / L.tile_rows;
    const int per_sm = (int)((227 * 1024) / L.total) > 0 ? (int)((227 * 1024) / L.total) : 1;
    int blocks = num_sms * per_sm;
    if (blocks > tiles) blocks = tiles;
    if (cplx) {
      cudaFuncSetAttribute(k_row_band_tma<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.total);
      k_row_band_tma<true><<<blocks, warps * 32, L.total, st>>>(in, n_rows, rows_per_clip, n, bm, out, scale,
                                                                 tw_inv, status);
    } else {
      cudaFuncSetAttribute(k_row_band_tma<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.total);
      k_row_band_tma<false><<<blocks, warps * 32, L.total, st>>>(in, n_rows, rows_per_clip, n, bm, out, scale,
                                                                  tw_inv, status);
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

namespace litho {
// This module's progress-wait budget on the current device (litho_set_wait_limit).
cudaError_t set_wait_limit_band(long long cycles) { return set_wait_limit_here(cycles); }
}  // namespace litho
