// Band-limited synthesis of real images on the tcgen05 tensor cores.
//
// The last stage of the Abbe sum (expose/aerial_image.py:488-494) and of the
// SOCS image and gradient (opc/ilt.py:227-232, 263-266) evaluates
//     I(x, y) = sum_{|gx|,|gy| <= g0} B(gx, gy) w^(gx x + gy y),  w = exp(2 pi i / N),
// for a Hermitian box B, so I is real. With the column stage
//     C(gx, y) = sum_gy B(gx, gy) w^(gy y)   (gx = 0..g0),
// the row stage is one real product per image:
//     I(x, y) = sum_k Q[x][k] P[y][k],  K = 2 g0 + 1 terms,
//     Q[x] = [1, cos(2 pi x / N), sin(2 pi x / N), cos(4 pi x / N), ...],
//     P[y] = [Re C(0, y), 2 Re C(1, y), -2 Im C(1, y), 2 Re C(2, y), ...],
// i.e. a GEMM with M = N = image side and K = 2 g0 + 1 (padded to Kp, a
// multiple of 16). It runs as tcgen05.mma kind::f16 with every operand split
// into FP16 hi + lo planes and three products per K step (hi hi + hi lo +
// lo hi), FP32 accumulation in TMEM: about 2^-22 of the largest term, the
// accuracy of FP32 operands. P is scaled per output by a power of two so that
// its bound 2 max_gx sum_gy |B(gx, gy)| stays below 2^14; the drain undoes it
// exactly. FP16 runs the tensor cores at twice the TF32 rate with half the
// operand bytes.
//
// Kernels:
//   k_synth_pplanes(_blk) : P for every output and row (column sums by
//                     32-point FFTs over residues), written in the MMA's
//                     shared-memory layout so each 256 x Kp tile is one bulk
//                     copy, and the output's scale;
//   k_synth_qplanes : Q for every x (the same for all outputs);
//   k_synth_mma     : persistent, one CTA per SM; a CTA takes (output, row
//                     tile, x range) units: one thread loads operand tiles
//                     (cp.async.bulk, double-buffered), one thread issues the
//                     MMAs into two TMEM accumulators, four warps drain the
//                     accumulators (tcgen05.ld), scale, stage 32 x 32 image
//                     blocks in shared memory for 2-D tensor stores
//                     (cp.async.bulk.tensor; coalesced row stores when no
//                     tensor map can be made) and keep the maxima.
// Peak normalisation needs the peak before the scaled image is written:
// pass 0 computes only the maxima, pass 1 writes. Every wait is bounded and a
// wait that gives up reports LITHO_E_TIMEOUT through the status word.
#include <cuda.h>  // CUtensorMap (the encoder is fetched through the runtime)
#include <cuda_fp16.h>

#include <type_traits>

#include "common.cuh"
#include "rows.cuh"
#include "tcgen05.cuh"

namespace litho {

constexpr int kSmMT = 128;        // x rows per tile (MMA M)
constexpr int kSmNT = 256;        // image rows per tile (MMA N)
constexpr int kSmG0Max = 31;      // box half-width limit (K = 2 g0 + 1 <= 63)
constexpr int kSmDrainWarps = 4;  // warp w drains TMEM lanes 32 w .. 32 w + 31
constexpr int kSmThreads = (kSmDrainWarps + 2) * 32;  // + one loading warp and one MMA warp

__host__ __device__ inline int smma_kp(int g0) { return (2 * g0 + 1 + 15) & ~15; }
// bytes of one operand tile (hi and lo planes, FP16)
__host__ __device__ inline uint32_t smma_a_bytes(int kp) { return (uint32_t)kSmMT * kp * 4; }
__host__ __device__ inline uint32_t smma_b_bytes(int kp) { return (uint32_t)kSmNT * kp * 4; }
// byte offset of element (row, k) in one plane of a tile of R rows: K-major
// core matrices (8 rows x 16 bytes = 8 FP16), 16-byte K chunks R * 16 bytes apart
__host__ __device__ inline uint32_t smma_off(int R, int row, int k) {
  return (uint32_t)((k >> 3) * (R * 16) + row * 16 + (k & 7) * 2);
}

bool synth_mma_ok(int n, int g0) {
  return g0 >= 0 && g0 <= kSmG0Max && n >= kSmNT && n <= 4096 && (n & (n - 1)) == 0;
}

// Worth it when there are enough 128 x 256 output tiles to keep every SM's
// MMA and drain pipeline busy (about 8 per SM: 1024 images of 256^2 gain
// 9 % over the pair synthesis; 64 of 512^2, 3.5 tiles per SM, do not);
// smaller batches use the pair synthesis, whose fixed costs are lower.
bool synth_mma_pick(int n_out, int n, int g0) {
  return synth_mma_ok(n, g0) && (int64_t)n_out * (n / kSmNT) * (n / kSmMT) >= 8 * 148;
}

// P planes, then Q planes, then the per-output inverse scales.
static int64_t pplanes_bytes(int n_out, int n, int kp) { return align16((int64_t)n_out * n * kp * 4); }
static int64_t qplanes_bytes(int n, int kp) { return align16((int64_t)n * kp * 4); }

int64_t synth_mma_bytes(int n_out, int n, int g0) {
  const int kp = smma_kp(g0);
  return pplanes_bytes(n_out, n, kp) + qplanes_bytes(n, kp) + align16((int64_t)n_out * 4);
}

__device__ __forceinline__ void split_f16(float v, __half& hi, __half& lo) {
  hi = __float2half_rn(v);
  lo = __float2half_rn(v - __half2float(hi));
}

// Power-of-two scale for output o's P values, from the bound
// |P_k(y)| <= 2 max_gx sum_gy |B(gx, gy)|, computed the same way in every
// block. bs: the output's box staged in shared memory, complete before the
// call; element (gy, gx) at bs[(gy + g0) * rs + (gx + g0) * cs]. Contains a
// __syncthreads.
__device__ float p_scale(const float2* bs, int g0, int rs, int cs, float* red) {
  const int G = 2 * g0 + 1;
  if (threadIdx.x <= g0) {
    float sum = 0.f;
    for (int i = 0; i < G; ++i) {
      const float2 b = bs[i * rs + (threadIdx.x + g0) * cs];
      sum += sqrtf(b.x * b.x + b.y * b.y);
    }
    red[threadIdx.x] = sum;
  }
  __syncthreads();
  float m = 0.f;
  for (int i = 0; i <= g0; ++i) m = fmaxf(m, red[i]);
  m *= 2.f;
  if (!(m > 0.f) || !isfinite(m)) return 1.f;
  int e;
  frexpf(m, &e);               // m < 2^e
  return ldexpf(1.f, 14 - e);  // scaled bound < 2^14
}

// P planes: [output][row tile][hi | lo][chunk][row][8] (row tile of 256 rows).
// The column sums C(gx, y) come from 32-point FFTs over residues: with
// N = 32 M and y = b + M a, C(gx, b + M a) = sum_r w32^(r a) S_b(r),
// S_b(r) = sum_{gy = r mod 32} B(gx, gy) w^(gy b), one FFT per residue b held
// in a lane's registers.
__device__ __forceinline__ void column_fft(const float2* cw, const float2* TB, int g0, int M, int b,
                                           float2 (&Q)[32]) {
#pragma unroll
  for (int i = 0; i < 32; ++i) Q[i] = make_float2(0.f, 0.f);
  Q[0] = cw[0];
#pragma unroll
  for (int g = 1; g <= kSmG0Max; ++g) {
    if (g <= g0) {
      const float2 t = TB[g * M + b];
      Q[g & 31] = cadd(Q[g & 31], cmul(cw[g], t));
      Q[(-g) & 31] = cadd(Q[(-g) & 31], cmulc(cw[-g], t));
    }
  }
  fft_reg<32, +1>(Q);
}

// One warp per (output, gx), scattered 2-byte stores; the gx = 0 warp also
// writes the zero padding K <= k < Kp. For grids whose column sums do not fit
// in shared memory.
constexpr int kPpWarps = 8;

__device__ __forceinline__ void p_put(__half* tile, int kp, int row, int k, float v) {
  __half h, l;
  split_f16(v, h, l);
  const uint32_t o = smma_off(kSmNT, row, k) >> 1;
  tile[o] = h;
  tile[(size_t)kSmNT * kp + o] = l;
}

__global__ void __launch_bounds__(kPpWarps * 32)
k_synth_pplanes(const float2* __restrict__ Bbox, int g0, int n, const float2* __restrict__ tw_inv, int kp,
                __half* __restrict__ planes, float* __restrict__ inv_scale) {
  extern __shared__ float2 pp_tb[];                     // [g][b] = w^(g b), g = 0..g0, then the box
  __shared__ float2 col[kPpWarps][2 * kSmG0Max + 2];    // B(gx, gy + g0) of each warp's column
  __shared__ float red[kSmG0Max + 1];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int o = blockIdx.y, gx = blockIdx.x * kPpWarps + warp;
  const int gp = g0 + 1, G = 2 * g0 + 1, M = n >> 5, nmask = n - 1;
  const float2* Bo = Bbox + (size_t)o * G * G;
  float2* bs = pp_tb + (size_t)gp * M;                  // [gy + g0][gx + g0]
  for (int j = threadIdx.x; j < gp * M; j += blockDim.x) {
    const int g = j / M, b = j % M;
    pp_tb[j] = __ldg(tw_inv + ((g * b) & nmask));
  }
  for (int j = threadIdx.x; j < G * G; j += blockDim.x) bs[j] = Bo[j];
  __syncthreads();
  if (gx < gp)
    for (int i = lane; i < G; i += 32) col[warp][i] = bs[i * G + gx + g0];
  const float sc = p_scale(bs, g0, G, 1, red);
  if (blockIdx.x == 0 && threadIdx.x == 0) inv_scale[o] = 1.f / sc;
  if (gx >= gp) return;
  const float2* cw = col[warp] + g0;
  __half* base = planes + (size_t)o * (n / kSmNT) * ((size_t)kSmNT * kp * 2);
  for (int b = lane; b < M; b += 32) {
    float2 Q[32];
    column_fft(cw, pp_tb, g0, M, b, Q);
#pragma unroll
    for (int a = 0; a < 32; ++a) {
      const int y = b + M * a, row = y % kSmNT;
      __half* tile = base + (size_t)(y / kSmNT) * ((size_t)kSmNT * kp * 2);
      if (gx == 0) {
        p_put(tile, kp, row, 0, Q[a].x * sc);
        for (int k = G; k < kp; ++k) p_put(tile, kp, row, k, 0.f);
      } else {
        p_put(tile, kp, row, 2 * gx - 1, 2.f * Q[a].x * sc);
        p_put(tile, kp, row, 2 * gx, -2.f * Q[a].y * sc);
      }
    }
  }
}

// The same planes with the column sums gathered per output in shared memory
// first (C[gx][y] for all y), so each thread then writes whole 16-byte K
// chunks of one row: one block per output, used when C fits in shared memory.
constexpr int kPbWarps = 16;

__host__ __device__ inline size_t pblk_smem(int n, int g0) {
  const int gp = g0 + 1;
  return (size_t)gp * n * 8 + (size_t)gp * (n >> 5) * 8 + (size_t)(2 * g0 + 1) * (2 * g0 + 1) * 8;
}

__global__ void __launch_bounds__(kPbWarps * 32)
k_synth_pplanes_blk(const float2* __restrict__ Bbox, int g0, int n, const float2* __restrict__ tw_inv, int kp,
                    __half* __restrict__ planes, float* __restrict__ inv_scale) {
  extern __shared__ float2 pb_sm[];
  __shared__ float red[kSmG0Max + 1];
  const int gp = g0 + 1, G = 2 * g0 + 1, M = n >> 5, nmask = n - 1;
  float2* Cs = pb_sm;                      // [gx][y]
  float2* TB = Cs + (size_t)gp * n;        // [g][b] = w^(g b)
  float2* bs = TB + (size_t)gp * M;        // the box, transposed: [gx + g0][gy + g0]
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, o = blockIdx.x;
  const float2* Bo = Bbox + (size_t)o * G * G;
  for (int j = threadIdx.x; j < gp * M; j += blockDim.x) {
    const int g = j / M, b = j % M;
    TB[j] = __ldg(tw_inv + ((g * b) & nmask));
  }
  for (int j = threadIdx.x; j < G * G; j += blockDim.x) bs[(j % G) * G + j / G] = Bo[j];
  __syncthreads();
  const float sc = p_scale(bs, g0, 1, G, red);
  if (threadIdx.x == 0) inv_scale[o] = 1.f / sc;
  for (int gx = warp; gx < gp; gx += kPbWarps) {
    const float2* cw = bs + (gx + g0) * G + g0;  // B(gx, gy) at cw[gy]
    for (int b = lane; b < M; b += 32) {
      float2 Q[32];
      column_fft(cw, TB, g0, M, b, Q);
#pragma unroll
      for (int a = 0; a < 32; ++a) Cs[(size_t)gx * n + b + M * a] = Q[a];
    }
  }
  __syncthreads();
  const int K = G, nck = kp >> 3;
  __half* base = planes + (size_t)o * (n / kSmNT) * ((size_t)kSmNT * kp * 2);
  for (int id = threadIdx.x; id < nck * n; id += blockDim.x) {
    const int y = id % n, c = id / n;
    __align__(16) __half hv[8];
    __align__(16) __half lv[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int k = 8 * c + q;
      float f = 0.f;
      if (k == 0) f = Cs[y].x;
      else if (k < K) f = (k & 1) ? 2.f * Cs[(size_t)((k + 1) >> 1) * n + y].x : -2.f * Cs[(size_t)(k >> 1) * n + y].y;
      split_f16(f * sc, hv[q], lv[q]);
    }
    __half* tile = base + (size_t)(y / kSmNT) * ((size_t)kSmNT * kp * 2);
    const uint32_t off = smma_off(kSmNT, y % kSmNT, 8 * c) >> 1;
    *reinterpret_cast<uint4*>(tile + off) = *reinterpret_cast<const uint4*>(hv);
    *reinterpret_cast<uint4*>(tile + (size_t)kSmNT * kp + off) = *reinterpret_cast<const uint4*>(lv);
  }
}

// Q planes: [x tile][hi | lo][chunk][row][8], identical for every output.
__global__ void __launch_bounds__(kSmMT)
k_synth_qplanes(const float2* __restrict__ tw, int g0, int n, int kp, __half* __restrict__ planes) {
  const int x = blockIdx.x * kSmMT + threadIdx.x;
  const int K = 2 * g0 + 1, nmask = n - 1;
  __half* hi = planes + (size_t)blockIdx.x * kSmMT * kp * 2;
  __half* lo = hi + (size_t)kSmMT * kp;
  for (int c = 0; c < kp / 8; ++c) {
    __align__(16) __half h[8];
    __align__(16) __half l[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int k = 8 * c + q;
      float f = 0.f;
      if (k == 0) {
        f = 1.f;
      } else if (k < K) {
        const int g = (k + 1) >> 1;
        const float2 w = tw[(g * x) & nmask];
        f = (k & 1) ? w.x : w.y;
      }
      split_f16(f, h[q], l[q]);
    }
    const uint32_t o = smma_off(kSmMT, threadIdx.x, 8 * c) >> 1;
    *reinterpret_cast<uint4*>(hi + o) = *reinterpret_cast<const uint4*>(h);
    *reinterpret_cast<uint4*>(lo + o) = *reinterpret_cast<const uint4*>(l);
  }
}

__device__ __forceinline__ void umma_f16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
}

// PASS 0: maxima of peak-normalised outputs only (others skipped).
// PASS 1: every output: image = raw * scale (scale / peak for peak-normalised
//         outputs) and the maxima of the raw image.
// blockmax[o][row tile][x range][warp]: the maximum over each drain warp's part.
// N: the image side as a compile-time constant (the drain's store offsets
// become immediates).
// One 32 x 32 FP32 block (shared, row-major, 128-byte rows) to the image
// tensor at element (x, y); x a multiple of 32.
__device__ __forceinline__ void tma_store_block(const CUtensorMap* m, const void* src, int x, int y) {
  asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%2, %3}], [%1];" ::"l"(m),
               "r"(smem_u32(src)), "r"(x), "r"(y)
               : "memory");
}

template <int PASS, int N>
__global__ void __launch_bounds__(kSmThreads, 1)
k_synth_mma(const __half* __restrict__ pplanes, const __half* __restrict__ qplanes,
            const float* __restrict__ inv_scale, int n_out, int kp, int xsplit, const LithoNorm* __restrict__ norm,
            const float* __restrict__ peak, float* __restrict__ image, float* __restrict__ blockmax,
            int* __restrict__ status, const __grid_constant__ CUtensorMap tmap, int use_tmap) {
  extern __shared__ __align__(1024) unsigned char sm_raw[];
  __shared__ uint64_t bar_bfull[2], bar_bempty[2], bar_afull[2], bar_aempty[2], bar_accfull[2], bar_accempty[2];
  __shared__ uint64_t bar_drain;
  __shared__ uint32_t s_tmem;
  __shared__ volatile int s_fail;
  constexpr int nt = kSmNT;
  const uint32_t abytes = smma_a_bytes(kp), bbytes = smma_b_bytes(kp);
  unsigned char* bufB0 = sm_raw;
  unsigned char* bufA0 = sm_raw + 2 * bbytes;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  constexpr int n = N;
  const int yt_per = n / nt, xt_per = n / kSmMT, xper = xt_per / xsplit;
  const int n_units = n_out * yt_per * xsplit;  // unit: (output, row tile, x range of xper tiles)
  const uint32_t tcols = 2u * (uint32_t)nt;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                 "r"(tcols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (threadIdx.x == 0) {
    s_fail = 0;
    for (int b = 0; b < 2; ++b) {
      mbar_init(&bar_bfull[b], 1);
      mbar_init(&bar_bempty[b], 1);
      mbar_init(&bar_afull[b], 1);
      mbar_init(&bar_aempty[b], 1);
      mbar_init(&bar_accfull[b], 1);
      mbar_init(&bar_accempty[b], kSmDrainWarps * 32);
    }
    mbar_init(&bar_drain, 1);
    fence_mbar_init();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s_tmem;

  auto live = [&](int u) -> bool {
    if (PASS == 1) return true;
    return norm != nullptr && norm[u / (yt_per * xsplit)].mode == 1;
  };

  if (warp == kSmDrainWarps) {
    // ---- operand loads ----------------------------------------------------
    if (lane == 0) {
      int i = 0, a = 0;
      bool ok = true;
      for (int u = blockIdx.x; u < n_units && ok; u += gridDim.x) {
        if (!live(u)) continue;
        const int ib = i & 1;
        if (i >= 2 && !mbar_wait(&bar_bempty[ib], ((i >> 1) - 1) & 1)) { ok = false; break; }
        mbar_expect_tx(&bar_bfull[ib], bbytes);
        bulk_g2s(bufB0 + ib * bbytes, pplanes + (size_t)(u / xsplit) * (bbytes >> 1), bbytes, &bar_bfull[ib]);
        ++i;
        for (int j = (u % xsplit) * xper; j < (u % xsplit + 1) * xper; ++j) {
          const int ab = a & 1;
          if (s_fail || (a >= 2 && !mbar_wait(&bar_aempty[ab], ((a >> 1) - 1) & 1))) { ok = false; break; }
          mbar_expect_tx(&bar_afull[ab], abytes);
          bulk_g2s(bufA0 + ab * abytes, qplanes + (size_t)j * (abytes >> 1), abytes, &bar_afull[ab]);
          ++a;
        }
      }
      if (!ok) s_fail = 1;
      // let the last copy into each buffer land before the block can exit
      // (the latest phase of a buffer's barrier; earlier phases completed
      // before it was refilled)
      for (int k = 1; k <= 2; ++k) {
        if (i - k >= 0 && !mbar_wait_drain(&bar_bfull[(i - k) & 1], ((i - k) >> 1) & 1)) s_fail = 1;
        if (a - k >= 0 && !mbar_wait_drain(&bar_afull[(a - k) & 1], ((a - k) >> 1) & 1)) s_fail = 1;
      }
    }
  } else if (warp == kSmDrainWarps + 1) {
    // ---- MMA issue --------------------------------------------------------
    if (lane == 0) {
      // D f32, A and B f16, both K-major, N = 256, M = 128
      const uint32_t idesc = (1u << 4) | ((uint32_t)(nt >> 3) << 17) | ((uint32_t)(kSmMT >> 4) << 24);
      int i = 0, a = 0, c = 0;
      bool ok = true;
      for (int u = blockIdx.x; u < n_units && ok; u += gridDim.x) {
        if (!live(u)) continue;
        const int ib = i & 1;
        if (!mbar_wait(&bar_bfull[ib], (i >> 1) & 1)) { ok = false; break; }
        const uint32_t bh0 = smem_u32(bufB0 + ib * bbytes), bl0 = bh0 + (bbytes >> 1);
        for (int j = 0; j < xper; ++j) {
          const int ab = a & 1, cb = c & 1;
          if (s_fail || !mbar_wait(&bar_afull[ab], (a >> 1) & 1) ||
              (c >= 2 && !mbar_wait(&bar_accempty[cb], ((c >> 1) - 1) & 1))) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t ah0 = smem_u32(bufA0 + ab * abytes), al0 = ah0 + (abytes >> 1);
          const uint32_t d = tmem + (uint32_t)(cb * nt);
          for (int s = 0; s < kp / 16; ++s) {
            const uint32_t ao = (uint32_t)s * 2 * (kSmMT * 16), bo = (uint32_t)s * 2 * (nt * 16);
            const uint64_t ah = umma_desc(ah0 + ao, kSmMT * 16, 128), al = umma_desc(al0 + ao, kSmMT * 16, 128);
            const uint64_t bh = umma_desc(bh0 + bo, nt * 16, 128), bl = umma_desc(bl0 + bo, nt * 16, 128);
            umma_f16(d, ah, bh, idesc, s > 0 ? 1u : 0u);
            umma_f16(d, ah, bl, idesc, 1u);
            umma_f16(d, al, bh, idesc, 1u);
          }
          umma_commit(&bar_accfull[cb]);
          umma_commit(&bar_aempty[ab]);
          if (j == xper - 1) umma_commit(&bar_bempty[ib]);
          ++a;
          ++c;
        }
        ++i;
      }
      if (!ok) s_fail = 1;
      if (c > 0) {  // every MMA this thread issued has completed before TMEM is released
        umma_commit(&bar_drain);
        if (!mbar_wait_drain(&bar_drain, 0)) s_fail = 1;
      }
    }
  } else {
    // ---- accumulator drain (warps 0-3: TMEM lanes 32 w .. 32 w + 31) -------
    // A chunk of 32 image rows x 32 x goes through this warp's shared-memory
    // stage (two buffers) and out as one 2-D tensor store issued by lane 0,
    // so the copy engine carries the image stores. Without a tensor map each
    // store instruction writes 32 consecutive x of one row (128 bytes).
    float* stage = reinterpret_cast<float*>(sm_raw + 2 * (abytes + bbytes)) + warp * 2 * 1024;
    int sb = 0;
    int c = 0;
    bool ok = true;
    for (int u = blockIdx.x; u < n_units && ok; u += gridDim.x) {
      if (!live(u)) continue;
      const int tile = u / xsplit, xs = u % xsplit;
      const int o = tile / yt_per, y0 = (tile % yt_per) * nt;
      const float inv = inv_scale[o];  // a power of two: exact
      float sc = inv;
      bool want_max = true;  // the writing pass of a peak-normalised output has its peak already
      if (PASS == 1) {
        const LithoNorm nm = norm ? norm[o] : LithoNorm{0, 1.0f};
        sc = nm.scale * inv;
        if (nm.mode == 1) {
          const float pk = peak[o];
          sc = (pk > 0.f ? nm.scale / pk : nm.scale) * inv;
          want_max = false;
        }
      }
      float mx = 0.f;
      float* img = image + (size_t)o * n * n;
      for (int j = xs * xper; j < (xs + 1) * xper; ++j) {
        const int cb = c & 1;
        if (s_fail || !mbar_wait(&bar_accfull[cb], (c >> 1) & 1)) { ok = false; break; }
        tc_fence_after();
        const int x = j * kSmMT + warp * 32 + lane;
        const uint32_t ta = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(cb * nt);
        for (int c0 = 0; c0 < nt; c0 += 32) {
          uint32_t r[32];
          tmem_ld32(ta + (uint32_t)c0, r);
          tmem_ld_wait();
          if (PASS == 0 || want_max) {
#pragma unroll
            for (int q = 0; q < 32; ++q) mx = fmaxf(mx, __uint_as_float(r[q]));
          }
          if (PASS == 1 && use_tmap) {
            float* sbuf = stage + sb * 1024;   // [row q][x]
            if (lane == 0) bulk_wait_read<1>();  // the store out of sbuf (two chunks ago) has read it
            __syncwarp();
#pragma unroll
            for (int q = 0; q < 32; ++q) sbuf[q * 32 + lane] = __uint_as_float(r[q]) * sc;
            fence_proxy_async_smem();
            __syncwarp();
            if (lane == 0) {
              tma_store_block(&tmap, sbuf, x - lane, o * N + y0 + c0);
              bulk_commit();
            }
            sb ^= 1;
          } else if (PASS == 1) {
            float* dst = img + (size_t)(y0 + c0) * N + x;
#pragma unroll
            for (int q = 0; q < 32; ++q) __stcs(dst + q * N, __uint_as_float(r[q]) * sc);
          }
        }
        tc_fence_before();
        mbar_arrive(&bar_accempty[cb]);
        ++c;
      }
      if (!ok) break;
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, off));
      if (lane == 0) blockmax[(size_t)u * kSmDrainWarps + warp] = mx * inv;
    }
    if (PASS == 1 && use_tmap && lane == 0) bulk_wait<0>();  // every store out of the stage is done
    if (!ok) s_fail = 1;
  }

  tc_fence_before();
  __syncthreads();
  if (s_fail && threadIdx.x == 0) atomicExch(status, LITHO_E_TIMEOUT);
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(tcols));
}

__global__ void k_peak(const float* __restrict__ blockmax, int nblk, const LithoNorm* __restrict__ norm, int n_out,
                       int which, float* __restrict__ peak);

// The n_out x n x n FP32 images as a 2-D tensor (n columns, n_out n rows)
// stored in 32 x 32 blocks. False when the driver's encoder is unavailable or
// refuses the layout (the drain then stores rows itself).
static bool image_tmap(CUtensorMap* m, float* image, int n, int n_out) {
  using Encode = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                              const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                              CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
  static const Encode enc = []() -> Encode {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &f, 12000, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return nullptr;
    return reinterpret_cast<Encode>(f);
  }();
  if (!enc || ((uintptr_t)image & 15) || (int64_t)n_out * n >= ((int64_t)1 << 31)) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)n, (cuuint64_t)n_out * (cuuint64_t)n};
  const cuuint64_t strides[1] = {(cuuint64_t)n * 4};
  const cuuint32_t box[2] = {32, 32}, estride[2] = {1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, image, dims, strides, box, estride, CU_TENSOR_MAP_INTERLEAVE_NONE,
             CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
         CUDA_SUCCESS;
}

// Synthesis of n_out Hermitian boxes of side 2 g0 + 1 into n x n images, with
// the normalisation of `norm` (nullptr: scale 1), the raw peaks into `peak`
// (may be nullptr when norm is) and `mid` (optional) recorded between the
// peak pass and the writing pass. planes: synth_mma_bytes(n_out, n, g0) of
// workspace. Requires synth_mma_ok(n, g0).
cudaError_t launch_synth_mma(const float2* box, int g0, int n, int n_out, const float2* tw, const LithoNorm* norm,
                             float* image, float* peak, float* blockmax, cudaStream_t s, cudaEvent_t mid,
                             void* planes, int* status, int num_sms) {
  const int kp = smma_kp(g0);
  char* pb = static_cast<char*>(planes);
  __half* pp = reinterpret_cast<__half*>(pb);
  __half* qp = reinterpret_cast<__half*>(pb + pplanes_bytes(n_out, n, kp));
  float* inv = reinterpret_cast<float*>(pb + pplanes_bytes(n_out, n, kp) + qplanes_bytes(n, kp));
  cudaError_t e;
  const size_t smb = pblk_smem(n, g0);
  if (smb <= 200 * 1024) {
    cudaFuncSetAttribute(k_synth_pplanes_blk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smb);
    k_synth_pplanes_blk<<<n_out, kPbWarps * 32, smb, s>>>(box, g0, n, tw, kp, pp, inv);
  } else {
    const size_t smp = (size_t)(g0 + 1) * (n >> 5) * 8 + (size_t)(2 * g0 + 1) * (2 * g0 + 1) * 8;
    cudaFuncSetAttribute(k_synth_pplanes, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smp);
    k_synth_pplanes<<<dim3((g0 + 1 + kPpWarps - 1) / kPpWarps, n_out), kPpWarps * 32, smp, s>>>(box, g0, n, tw,
                                                                                               kp, pp, inv);
  }
  k_synth_qplanes<<<n / kSmMT, kSmMT, 0, s>>>(tw, g0, n, kp, qp);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  // operand buffers, then the drain warps' image stages (2 x 32 x 32 floats each)
  const size_t smm = 2 * (size_t)(smma_a_bytes(kp) + smma_b_bytes(kp)) + (size_t)kSmDrainWarps * 2 * 1024 * 4;
  // split the x tiles of a (output, row tile) over blocks when there are
  // fewer of those than SMs (at most 8 ways, so the block maxima fit in
  // n / 8 floats per output)
  int xsplit = 1;
  const int tiles = n_out * (n / kSmNT);
  while (tiles * xsplit < num_sms && xsplit * 2 <= n / kSmMT && xsplit * 2 <= kSmNT / 32) xsplit *= 2;
  const int units = tiles * xsplit;
  const int grid = units < num_sms ? units : num_sms;
  const int nblk = (n / kSmNT) * xsplit * kSmDrainWarps;
  const int pk_blocks = (n_out + 7) / 8;
  CUtensorMap tmap{};
  const int use_tmap = image_tmap(&tmap, image, n, n_out) ? 1 : 0;
  auto pass = [&](auto pass_c) -> cudaError_t {
    constexpr int P = decltype(pass_c)::value;
    switch (n) {
#define LITHO_SMMA(NN)                                                                                           \
  case NN:                                                                                                       \
    cudaFuncSetAttribute(k_synth_mma<P, NN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smm);             \
    k_synth_mma<P, NN><<<grid, kSmThreads, smm, s>>>(pp, qp, inv, n_out, kp, xsplit, norm, peak, image,          \
                                                      blockmax, status, tmap, P == 1 ? use_tmap : 0);           \
    break;
      LITHO_SMMA(256) LITHO_SMMA(512) LITHO_SMMA(1024) LITHO_SMMA(2048) LITHO_SMMA(4096)
#undef LITHO_SMMA
      default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
  };
  if (norm) {
    if (!peak) return cudaErrorInvalidValue;
    if ((e = pass(std::integral_constant<int, 0>{})) != cudaSuccess) return e;
    k_peak<<<pk_blocks, 256, 0, s>>>(blockmax, nblk, norm, n_out, 1, peak);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  if (mid) cudaEventRecord(mid, s);
  if ((e = pass(std::integral_constant<int, 1>{})) != cudaSuccess) return e;
  if (peak) k_peak<<<pk_blocks, 256, 0, s>>>(blockmax, nblk, norm, n_out, norm ? 0 : -1, peak);
  return cudaGetLastError();
}

}  // namespace litho

namespace litho {
// This module's progress-wait budget on the current device (litho_set_wait_limit).
cudaError_t set_wait_limit_synth(long long cycles) { return set_wait_limit_here(cycles); }
}  // namespace litho
