// Row engines: band-limited synthesis of real images by 32-point FFTs over
// pairs of rows, and the per-output peak.
//
// Synthesis (the last stage of the Abbe sum, expose/aerial_image.py:488-494,
// and of the SOCS image and gradient, opc/ilt.py:227-232, 263-266):
//     I(x, y) = sum_{|gx|,|gy| <= g0} B(gx, gy) w^(gx x + gy y),  w = exp(2 pi i / N),
// with B Hermitian (B(-g) = conj B(g)), so I is real.
//   column stage: C(gx, y) = sum_gy B(gx, gy) w^(gy y), for gx >= 0 (C(-gx) = conj C(gx));
//   row stage   : two real rows at once, Z(x) = sum_g (C(g, y1) + i C(g, y2)) w^(g x)
//                 = I(x, y1) + i I(x, y2). With N = 32 M and x = b + M a,
//                 Z(b + M a) = sum_r w32^(r a) Q_b(r),  Q_b(r) = sum_{g = r mod 32} D(g) w^(g b),
//                 a 32-point inverse FFT per residue b held in one lane's registers.
// About 10 FP32 operations per pixel instead of the ~60 of a direct sum, so
// the pass is bound by its HBM writes.
//
// Peak normalisation needs the peak before the scaled image is written, so
// peak-normalised outputs run the synthesis twice: pass 0 computes only the
// block maxima (no HBM traffic), pass 1 recomputes and writes
// raw * scale / peak. Every reduction is in a fixed order.
#include "common.cuh"
#include "ilt_math.cuh"
#include "rows.cuh"

namespace litho {

constexpr int kSyWarps = 8;
constexpr int kSyRows = 64;      // rows per block
constexpr int kSyG0Max = 31;     // box half-width limit: G = 2 g0 + 1 <= 63
constexpr int kSyObjStage = 2048;  // target values staged per warp (2 P rows of n <= 1024)

// Shared-memory plan of one synthesis block.
struct SynthSmem {
  int M, Lp, P, q, G, gp;
  size_t off_tw, off_tb, off_c, off_b, total;
};

// cols_ahead: the column stage was done ahead (k_synth_cols), so the block
// needs only the row-stage twiddles TB and its rows' C; the full table tw and
// the box B (the direct column stage's operands) are left out.
__host__ __device__ inline SynthSmem synth_smem(int n, int g0, bool cols_ahead = false) {
  SynthSmem s{};
  s.M = n >> 5;
  s.Lp = s.M < 32 ? s.M : 32;
  s.P = 32 / s.Lp;
  s.q = s.M / s.Lp;
  s.G = 2 * g0 + 1;
  s.gp = g0 + 1;
  s.off_tw = 0;
  s.off_tb = cols_ahead ? 0 : s.off_tw + (size_t)n * 8;
  s.off_c = s.off_tb + (size_t)s.gp * s.M * 8;
  s.off_b = s.off_c + (size_t)kSyRows * s.gp * 8;
  s.total = cols_ahead ? s.off_b : s.off_b + (size_t)s.G * s.G * 8;
  return s;
}

// Offset of the objective's target stage: after the synthesis operands,
// rounded up to 128 bytes (its 16-byte copies need aligned destinations; the
// operands end with the G x G box, an odd multiple of 8 bytes for odd G).
__host__ __device__ inline size_t obj_stage_off(const SynthSmem& s) { return (s.total + 127) & ~(size_t)127; }
// Floats of one warp's stage in the band form: the 2 P target rows, or the
// band DFT's transpose of P row pairs (P groups of band_group_pitch(M)
// complex), whichever is larger, in 128-byte units.
__host__ __device__ inline int band_stage_floats(int M, int P) {
  const int y = P * band_group_pitch(M) * 2;
  const int f = y > kSyObjStage ? y : kSyObjStage;
  return (f + 31) & ~31;
}

// Is the pair-FFT synthesis available for this grid and box?
bool synth_pairs_ok(int n, int g0) {
  return n >= 256 && n <= 2048 && (n & (n - 1)) == 0 && g0 >= 0 && g0 <= kSyG0Max &&
         synth_smem(n, g0).total <= 200 * 1024;
}

// PASS 0: block maxima only, for peak-normalised outputs (others return).
// PASS 1: write raw * scale (scale / peak for peak-normalised outputs) and
//         the block maxima of the raw image.
// Column stage for whole images, done once ahead of both synthesis passes:
// C[o][gx][y] = sum_gy B(gx, gy) w^(gy y) for gx = 0..g0 and every row y,
// by the same residue method as the row stage (y = b + M a, a 32-point FFT
// per residue). One warp per (output, gx).
constexpr int kColWarps = 8;

__global__ void __launch_bounds__(kColWarps * 32, 2)
k_synth_cols(const float2* __restrict__ Bbox, int g0, int n, const float2* __restrict__ tw_inv,
             float2* __restrict__ Cg) {
  extern __shared__ float2 cols_tb[];                   // [g][b] = w^(g b), g = 0..g0
  __shared__ float2 col[kColWarps][2 * kSyG0Max + 2];   // B(gx, gy + g0) of each warp's column
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int o = blockIdx.y, gx = blockIdx.x * kColWarps + warp;
  const int gp = g0 + 1, G = 2 * g0 + 1, M = n >> 5, nmask = n - 1;
  for (int j = threadIdx.x; j < gp * M; j += blockDim.x) {
    const int g = j / M, b = j % M;
    cols_tb[j] = __ldg(tw_inv + ((g * b) & nmask));
  }
  if (gx < gp) {
    const float2* bc = Bbox + (size_t)o * G * G + gx + g0;
    for (int i = lane; i < G; i += 32) col[warp][i] = bc[(size_t)i * G];
  }
  __syncthreads();
  if (gx >= gp) return;
  const float2* cw = col[warp] + g0;
  float2* dst = Cg + ((size_t)o * gp + gx) * n;
  for (int b = lane; b < M; b += 32) {
    float2 Q[32];
#pragma unroll
    for (int i = 0; i < 32; ++i) Q[i] = make_float2(0.f, 0.f);
    Q[0] = cw[0];
#pragma unroll
    for (int g = 1; g <= kSyG0Max; ++g) {
      if (g <= g0) {
        const float2 t = cols_tb[g * M + b];
        Q[g & 31] = cadd(Q[g & 31], cmul(cw[g], t));
        Q[(-g) & 31] = cadd(Q[(-g) & 31], cmulc(cw[-g], t));
      }
    }
    fft_reg<32, +1>(Q);
#pragma unroll
    for (int a = 0; a < 32; ++a) dst[b + M * a] = Q[a];
  }
}

// OBJ (PASS 1 only): the image is not stored; each pixel goes through the ILT
// objective (ilt_objective_pixel against obj.target, whose rows are copied to
// shared memory while the row pair's transform runs), dJ/dfield is stored in
// obj.dfield, and the block's cost and pattern-error sums go to the partial
// arrays, which the last block of each output totals (as k_ilt_objective).
// BAND (with OBJ): dJ/dfield is not stored either; the row pair's values go
// through the forward band DFT of its rows (the first pass of
// litho_band_spectrum, same arithmetic: a 32-point FFT per residue, the
// per-pass twiddle table and the transpose-sum in the warp's stage buffer)
// and only the band rows obj.band_rows[o][k + kb][row], |k| <= kb, are written.
template <int PASS, bool OBJ = false, bool BAND = false>
__global__ void __launch_bounds__(kSyWarps * 32, 2)
k_synth_pairs(const float2* __restrict__ Bbox, int g0, int n, const float2* __restrict__ tw_inv,
              const LithoNorm* __restrict__ norm, const float* __restrict__ peak, float* __restrict__ image,
              float* __restrict__ blockmax, const float2* __restrict__ Cg, SynthObj obj = SynthObj{}) {
  static_assert(!OBJ || PASS == 1, "the objective runs in the writing pass");
  static_assert(!BAND || OBJ, "the band form is a form of the objective pass");
  extern __shared__ __align__(16) unsigned char sy_raw[];
  const SynthSmem L = synth_smem(n, g0, Cg != nullptr);
  const int o = blockIdx.y, y0 = blockIdx.x * kSyRows;
  const LithoNorm nm = norm ? norm[o] : LithoNorm{0, 1.0f};
  if (PASS == 0 && nm.mode != 1) return;
  float2* tw = reinterpret_cast<float2*>(sy_raw + L.off_tw);
  float2* TB = reinterpret_cast<float2*>(sy_raw + L.off_tb);   // [g][b] = w^(g b), g = 0..g0
  float2* C = reinterpret_cast<float2*>(sy_raw + L.off_c);     // [row][gx], gx = 0..g0
  float2* B = reinterpret_cast<float2*>(sy_raw + L.off_b);     // [gy + g0][gx + g0]
  __shared__ float red[kSyWarps];
  const int M = L.M, G = L.G, gp = L.gp, nmask = n - 1;
  if (Cg) {
    // column stage done ahead (k_synth_cols): C[o][gx][y] -> C[row][gx]
    for (int j = threadIdx.x; j < gp * M; j += blockDim.x) {
      const int g = j / M, b = j % M;
      TB[j] = __ldg(tw_inv + ((g * b) & nmask));
    }
    const float2* cs = Cg + (size_t)o * gp * n + y0;
    for (int id = threadIdx.x; id < kSyRows * gp; id += blockDim.x) {
      const int gx = id / kSyRows, r = id % kSyRows;
      C[r * gp + gx] = __ldg(cs + (size_t)gx * n + r);
    }
  } else {
    for (int j = threadIdx.x; j < n; j += blockDim.x) tw[j] = tw_inv[j];
    const float2* Bo = Bbox + (size_t)o * G * G;
    for (int j = threadIdx.x; j < G * G; j += blockDim.x) B[j] = Bo[j];
    __syncthreads();
    for (int j = threadIdx.x; j < gp * M; j += blockDim.x) {
      const int g = j / M, b = j % M;
      TB[j] = tw[(g * b) & nmask];
    }
    // column stage for the block's rows
    for (int id = threadIdx.x; id < kSyRows * gp; id += blockDim.x) {
      const int r = id / gp, gx = id % gp, y = y0 + r;
      float2 acc = make_float2(0.f, 0.f);
      const float2* bc = B + gx + g0;
      for (int gy = -g0; gy <= g0; ++gy) acc = cadd(acc, cmul(bc[(gy + g0) * G], tw[(gy * y) & nmask]));
      C[id] = acc;
    }
  }
  __syncthreads();

  float sc = nm.scale;
  if (PASS == 1 && nm.mode == 1) {
    const float pk = peak[o];
    sc = pk > 0.f ? nm.scale / pk : nm.scale;
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int pg = lane / L.Lp, bl = lane % L.Lp;
  const int iters = kSyRows / (2 * kSyWarps * L.P);
  float mx = 0.f;
  double ocost = 0.0;
  unsigned int operr = 0;
  // OBJ: this warp's 2 P target rows (2048 contiguous values for n <= 1024);
  // BAND: the same buffer then holds the band DFT's transpose
  const int stage_f = BAND ? band_stage_floats(M, L.P) : kSyObjStage;
  float* tg = reinterpret_cast<float*>(sy_raw + obj_stage_off(L)) + warp * stage_f;
  const int kb = obj.band_half, Bmb = 2 * kb + 1, npass = (Bmb + 31) >> 5;
  float2* BTB = reinterpret_cast<float2*>(sy_raw + obj_stage_off(L) + (size_t)kSyWarps * stage_f * 4);
  float2* Zw = BTB + (size_t)npass * 32 * M + (size_t)warp * L.P * npass * 32;   // [pair group][k + kb]
  if (BAND) {   // the forward band twiddles w^(-k b) per (pass, register kp, residue b), 0 off the band
    for (int j = threadIdx.x; j < npass * 32 * M; j += blockDim.x) {
      const int p = j / (32 * M), kp = (j / M) & 31, b = j % M;
      const int k = -kb + ((kp + kb) & 31) + 32 * p;
      BTB[j] = k <= kb ? tw_inv[(-k * b) & nmask] : make_float2(0.f, 0.f);
    }
    __syncthreads();
  }
  for (int it = 0; it < iters; ++it) {
    const int pair = (it * kSyWarps + warp) * L.P + pg;
    if (OBJ) {
      const float* src = obj.target + ((size_t)o * n + y0 + 2 * (it * kSyWarps + warp) * L.P) * n;
      for (int e = lane * 4; e < kSyObjStage; e += 128) cp_async16(tg + e, src + e);
      cp_async_commit();
    }
    const float2* c1 = C + (2 * pair) * gp;
    const float2* c2 = c1 + gp;
    float* row1 = image + ((size_t)o * n + y0 + 2 * pair) * n;
    float* row2 = row1 + n;
    for (int qq = 0; qq < L.q; ++qq) {
      const int b = bl + qq * L.Lp;
      float2 Q[32];
#pragma unroll
      for (int i = 0; i < 32; ++i) Q[i] = make_float2(0.f, 0.f);
      {  // g = 0, then +g and -g together: D(-g) = conj C(g, y1) + i conj C(g, y2), w^(-g b) = conj w^(g b)
        const float2 a1 = c1[0], a2 = c2[0];
        Q[0] = make_float2(a1.x - a2.y, a1.y + a2.x);
      }
#pragma unroll
      for (int g = 1; g <= kSyG0Max; ++g) {
        if (g <= g0) {
          const float2 a1 = c1[g], a2 = c2[g];
          const float2 t = TB[g * M + b];
          const float2 dp = make_float2(a1.x - a2.y, a1.y + a2.x);
          const float2 dm = make_float2(a1.x + a2.y, a2.x - a1.y);
          Q[g & 31] = cadd(Q[g & 31], cmul(dp, t));
          Q[(-g) & 31] = cadd(Q[(-g) & 31], cmulc(dm, t));
        }
      }
      fft_reg<32, +1>(Q);
#pragma unroll
      for (int a = 0; a < 32; ++a) mx = fmaxf(mx, fmaxf(Q[a].x, Q[a].y));
      if (PASS == 1 && OBJ) {
        const size_t i1 = ((size_t)o * n + y0 + 2 * pair) * n + b;
        const float* t1 = tg + 2 * pg * n + b;
        float* __restrict__ d1 = obj.dfield + i1;
        float cc = 0.f, sg;
        cp_async_wait_all();
        __syncwarp();
#pragma unroll
        for (int a = 0; a < 32; ++a) {
          const float ta = t1[M * a], tb = t1[n + M * a];
          const float da = ilt_objective_pixel(Q[a].x * sc, ta, obj.scale, obj.level, obj.sign, obj.a,
                                               obj.inv_npix2, cc, operr, &sg);
          const float db = ilt_objective_pixel(Q[a].y * sc, tb, obj.scale, obj.level, obj.sign, obj.a,
                                               obj.inv_npix2, cc, operr, &sg);
          if (BAND) {
            Q[a] = make_float2(da, db);
          } else {
            __stcs(d1 + M * a, da);
            __stcs(d1 + n + M * a, db);
          }
        }
        ocost += (double)cc;
        __syncwarp();  // every lane is done with the stage before the next copy into it
        if (BAND) {
          // rows y1 + i y2 of this pair group: X_b(kp) over a, then per pass
          // the transpose-sum U(k) = sum_b w^(-k b) X_b(k mod 32)
          fft_reg<32, -1>(Q);
          float2* Y = reinterpret_cast<float2*>(tg);     // [pair group (pitch GP)][kp (pitch M + 1)][b]
          const int LD = M + 1, GP = band_group_pitch(M);
          for (int p = 0; p < npass; ++p) {
            float2* yr = Y + pg * GP + b;
            const float2* tb = BTB + p * 32 * M + b;
#pragma unroll
            for (int kp = 0; kp < 32; ++kp) yr[kp * LD] = cmul(Q[kp], tb[kp * M]);
            __syncwarp();
            const int k = -kb + ((lane + kb) & 31) + 32 * p;
            for (int r = 0; r < L.P; ++r) {
              const float2* yq = Y + r * GP + lane * LD;
              float2 s0 = make_float2(0.f, 0.f), s1 = make_float2(0.f, 0.f);
              for (int j = 0; j + 1 < M; j += 2) {
                s0 = cadd(s0, yq[j]);
                s1 = cadd(s1, yq[j + 1]);
              }
              if (M & 1) s0 = cadd(s0, yq[M - 1]);
              if (k <= kb) Zw[r * npass * 32 + (k + kb)] = cadd(s0, s1);
            }
            __syncwarp();
          }
          for (int r = 0; r < L.P; ++r) {   // separate the two real rows of each pair: R1 = (Z + Z*(-k)) / 2, ...
            const int ra = y0 + 2 * ((it * kSyWarps + warp) * L.P + r);
            const float2* zr = Zw + r * npass * 32;
            for (int kk = lane; kk < Bmb; kk += 32) {
              const float2 z = zr[kk], zm = zr[Bmb - 1 - kk];
              float2* dst = obj.band_rows + ((size_t)o * Bmb + kk) * n + ra;
              dst[0] = make_float2((z.x + zm.x) * 0.5f, (z.y - zm.y) * 0.5f);
              dst[1] = make_float2((z.y + zm.y) * 0.5f, (zm.x - z.x) * 0.5f);
            }
          }
          __syncwarp();  // the stage and Z are free before the next copy into them
        }
      } else if (PASS == 1) {
#pragma unroll
        for (int a = 0; a < 32; ++a) {
          __stcs(row1 + b + M * a, Q[a].x * sc);
          __stcs(row2 + b + M * a, Q[a].y * sc);
        }
      }
    }
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, off));
  if (lane == 0) red[warp] = mx;
  __syncthreads();
  if (threadIdx.x == 0) {
    float m = red[0];
    for (int i = 1; i < kSyWarps; ++i) m = fmaxf(m, red[i]);
    blockmax[(size_t)o * gridDim.x + blockIdx.x] = m;
  }
  if (OBJ) {
    __shared__ double rc[kSyWarps];
    __shared__ unsigned int rp[kSyWarps];
    __shared__ bool last;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      ocost += __shfl_xor_sync(0xffffffffu, ocost, off);
      operr += __shfl_xor_sync(0xffffffffu, operr, off);
    }
    if (lane == 0) {
      rc[warp] = ocost;
      rp[warp] = operr;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double c = 0.0;
      unsigned int p = 0;
      for (int i = 0; i < kSyWarps; ++i) {
        c += rc[i];
        p += rp[i];
      }
      obj.cost_part[(size_t)o * gridDim.x + blockIdx.x] = c;
      obj.perr_part[(size_t)o * gridDim.x + blockIdx.x] = p;
      __threadfence();  // the partials are visible before this block is counted
      last = atomicAdd(&obj.counters[o], 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
      __threadfence();
      double c = 0.0;
      long long p = 0;
      for (unsigned int i = 0; i < gridDim.x; ++i) {
        c += __ldcg(obj.cost_part + (size_t)o * gridDim.x + i);
        p += __ldcg(obj.perr_part + (size_t)o * gridDim.x + i);
      }
      obj.cost_out[o] = c / ((double)n * (double)n);
      obj.perr_out[o] = p;
      obj.counters[o] = 0u;
    }
  }
}

// peak[o] = max of its block maxima, for outputs whose mode matches `which`
// (1: peak-normalised only, 0: all others, -1: every output). One warp each.
__global__ void k_peak(const float* __restrict__ blockmax, int nblk, const LithoNorm* __restrict__ norm, int n_out,
                       int which, float* __restrict__ peak) {
  const int o = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (o >= n_out) return;
  if (which >= 0) {
    const int mode = norm ? norm[o].mode : 0;
    if ((which == 1) != (mode == 1)) return;
  }
  float m = 0.f;
  for (int i = lane; i < nblk; i += 32) m = fmaxf(m, blockmax[(size_t)o * nblk + i]);
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, off));
  if (lane == 0) peak[o] = m;
}

int synth_pairs_blocks(int n) { return n / kSyRows; }

// Synthesis of n_out Hermitian boxes of side 2 g0 + 1 into n x n images with
// the normalisation of `norm` (nullptr: scale 1), the raw peaks into `peak`
// (may be nullptr when norm is) and `mid` (optional) recorded between the
// peak pass and the writing pass. cbuf (optional, n_out x (g0 + 1) x n
// complex): the column stage then runs once for whole images ahead of both
// passes. Requires synth_pairs_ok(n, g0).
cudaError_t launch_synth_pairs(const float2* box, int g0, int n, int n_out, const float2* tw, const LithoNorm* norm,
                               float* image, float* peak, float* blockmax, cudaStream_t s, cudaEvent_t mid,
                               float2* cbuf) {
  const SynthSmem L = synth_smem(n, g0, cbuf != nullptr);
  const dim3 grid(n / kSyRows, n_out);
  const int pk_blocks = (n_out + 7) / 8;
  cudaError_t e;
  if (cbuf) {
    const size_t smc = (size_t)(g0 + 1) * (n >> 5) * 8;
    k_synth_cols<<<dim3((g0 + 1 + kColWarps - 1) / kColWarps, n_out), kColWarps * 32, smc, s>>>(box, g0, n, tw,
                                                                                               cbuf);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  if (norm) {
    if (!peak) return cudaErrorInvalidValue;
    cudaFuncSetAttribute(k_synth_pairs<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.total);
    k_synth_pairs<0><<<grid, kSyWarps * 32, L.total, s>>>(box, g0, n, tw, norm, peak, image, blockmax, cbuf);
    k_peak<<<pk_blocks, 256, 0, s>>>(blockmax, grid.x, norm, n_out, 1, peak);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  if (mid) cudaEventRecord(mid, s);
  cudaFuncSetAttribute(k_synth_pairs<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.total);
  k_synth_pairs<1><<<grid, kSyWarps * 32, L.total, s>>>(box, g0, n, tw, norm, peak, image, blockmax, cbuf);
  if (peak) k_peak<<<pk_blocks, 256, 0, s>>>(blockmax, grid.x, norm, n_out, norm ? 0 : -1, peak);
  return cudaGetLastError();
}

int64_t synth_cols_bytes(int n_out, int n, int g0) { return (int64_t)n_out * (g0 + 1) * n * 8; }

// The objective synthesis stages each warp's 2 P target rows (2 P n = 2048
// values) in shared memory next to the synthesis operands.
bool synth_objective_ok(int n, int g0) {
  return synth_pairs_ok(n, g0) && n <= 1024 &&
         obj_stage_off(synth_smem(n, g0, true)) + (size_t)kSyWarps * kSyObjStage * 4 <= 110 * 1024;
}

// The image synthesis of launch_synth_pairs (no normalisation) with the ILT
// objective applied to every pixel instead of storing the image; the column
// stage runs ahead into cbuf. Partials: [n_out][n / kSyRows] in obj.
cudaError_t launch_synth_objective(const float2* box, int g0, int n, int n_out, const float2* tw, float* blockmax,
                                   float2* cbuf, const SynthObj& obj, cudaStream_t s) {
  const SynthSmem L = synth_smem(n, g0, true);
  const dim3 grid(n / kSyRows, n_out);
  const size_t smc = (size_t)(g0 + 1) * (n >> 5) * 8;
  k_synth_cols<<<dim3((g0 + 1 + kColWarps - 1) / kColWarps, n_out), kColWarps * 32, smc, s>>>(box, g0, n, tw, cbuf);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  const size_t sm = obj_stage_off(L) + (size_t)kSyWarps * kSyObjStage * 4;
  cudaFuncSetAttribute(k_synth_pairs<1, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  k_synth_pairs<1, true><<<grid, kSyWarps * 32, sm, s>>>(box, g0, n, tw, nullptr, nullptr, nullptr, blockmax, cbuf,
                                                         obj);
  return cudaGetLastError();
}

// Shared memory of the band form: the objective's (with the larger stage),
// the forward band twiddles and each warp's band values.
size_t synth_objective_band_smem(int n, int g0, int kb) {
  const SynthSmem L = synth_smem(n, g0, true);
  const int npass = (2 * kb + 1 + 31) >> 5;
  return obj_stage_off(L) + (size_t)kSyWarps * band_stage_floats(L.M, L.P) * 4 + (size_t)npass * 32 * L.M * 8 +
         (size_t)kSyWarps * L.P * npass * 32 * 8;
}

bool synth_objective_band_ok(int n, int g0, int kb) {
  return synth_objective_ok(n, g0) && kb >= 0 && 2 * kb + 1 <= n && synth_objective_band_smem(n, g0, kb) <= 110 * 1024;
}

// launch_synth_objective with the band rows of dJ/dfield (obj.band_rows,
// obj.band_half) written instead of dJ/dfield.
cudaError_t launch_synth_objective_band(const float2* box, int g0, int n, int n_out, const float2* tw,
                                        float* blockmax, float2* cbuf, const SynthObj& obj, cudaStream_t s) {
  const dim3 grid(n / kSyRows, n_out);
  const size_t smc = (size_t)(g0 + 1) * (n >> 5) * 8;
  k_synth_cols<<<dim3((g0 + 1 + kColWarps - 1) / kColWarps, n_out), kColWarps * 32, smc, s>>>(box, g0, n, tw, cbuf);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  const size_t sm = synth_objective_band_smem(n, g0, obj.band_half);
  cudaFuncSetAttribute(k_synth_pairs<1, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  k_synth_pairs<1, true, true><<<grid, kSyWarps * 32, sm, s>>>(box, g0, n, tw, nullptr, nullptr, nullptr, blockmax,
                                                               cbuf, obj);
  return cudaGetLastError();
}

}  // namespace litho
