// Abbe imaging for wide pupils: the band-limited engine on coarse grids of
// L = 128 .. 1024 points (pupil half-width h >= 16 bins, e.g. EUV clips at
// 512^2 and above), where one coherent system's L x L transform no longer
// fits a warp's registers.
//
// Same mathematics as abbe.cu (expose/aerial_image.py:421-494 restated on
// the smallest grid that holds |E|^2 exactly, L >= 4h + 1), with the two
// passes of each coherent transform split across thread blocks:
//   pass A (k_wide_cols_w): per transform and chunk of spectral columns kx,
//       the inverse L-point FFT over ky of P M on the (2h+1)-row band ->
//       T[kx][v] in global memory (L2-resident for a chunk of jobs);
//   pass B (k_wide_rows_w): per work item and chunk of rows v, the inverse
//       L-point FFT over kx of T[.][v] for every transform of the item and
//       J(u, v) += w |e|^2 in shared memory -> the item's partial J;
//   reduce (k_wide_reduce) in item order, F = FFT_L(J) / L^2 and the image
//       band box B(g), |g| <= 2h (k_wide_box);
//   synthesis: two outputs per complex transform (B is Hermitian, so each
//       image is real): a column stage over gy, then a row stage over gx that
//       writes both images (k_wsyn_cols, k_wsyn_rows), then the
//       normalisation of aerial_image.py:217-241.
// Passes A and B, the adjoint passes, the synthesis and the L x L transforms
// of J and g_L (rows straight from global memory, columns through a padded
// shared tile: k_wfft_rows, k_wfft_cols) run warp-per-line register FFTs
// (fftwarp.cuh). Every reduction has a fixed order, so results are
// deterministic.
#include <algorithm>

#include "common.cuh"
#include "fftsmem.cuh"
#include "fftwarp.cuh"
#include "wide.cuh"

namespace litho {

cudaError_t plain_fft2(const void* in, bool in_real, float2* buf, long long planes, int n, int sign, float scale_rows,
                       float scale_cols, const float2* tw, cudaStream_t st);
cudaError_t launch_row_band_dft(const void* in, bool cplx, int n_rows, int rows_per_clip, int n, int bm,
                                float2* out, float scale, const float2* tw_inv, int num_sms, cudaStream_t st,
                                int* status);
cudaError_t launch_pupil_table(const LithoAbbePlan& p, const void* blob, float2* table, cudaStream_t s);
__global__ void k_normalise(const float* __restrict__ blockmax, int nblk, const LithoNorm* __restrict__ norm,
                            int n, float* __restrict__ image, float* __restrict__ peak, int apply_mode0);

constexpr int kWideMaxBlk = 256;    // block maxima per output
constexpr int64_t kWideTBudget = 512ll << 20;   // bytes of pass-A output per job chunk
constexpr int kWideSpecPairs = 4;   // output pairs per synthesis chunk

// Register-FFT forms of passes A and B (fftwarp.cuh): a warp transforms
// 32 / R lines of L = 32 R points at once; kWfWarps warps per block.
constexpr int kWfWarps = 8;

// twiddles and the warps' transpose buffers
__host__ __device__ inline size_t wf_smem(int L) { return (size_t)L * 8 + (size_t)kWfWarps * 32 * kTbLd * 8; }
// pass B keeps J in registers up to L = 256; longer lines leave no registers
// for it and keep the warps' J rows in shared memory after the buffers above
__host__ __device__ constexpr bool wf_j_regs(int L) { return L <= 256; }
__host__ __device__ inline size_t wf_rows_smem(int L) {
  return wf_smem(L) + (wf_j_regs(L) ? 0 : (size_t)kWfWarps * 32 * 32 * 4);
}

// Pass A. Grid (transform t of the chunk, chunk of kWfWarps * LPW columns).
template <int L>
__global__ void __launch_bounds__(kWfWarps * 32, 2)
k_wide_cols_w(const LithoJob* __restrict__ jobs, int j0, int ncomp_max, const float2* __restrict__ table, int h,
              const float2* __restrict__ Mb, int bm, const float2* __restrict__ twL, float2* __restrict__ T) {
  constexpr int R = L / 32, LPW = 32 / R;
  extern __shared__ float2 wsm[];
  float2* tw = wsm;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float2* tb = wsm + L + warp * 32 * kTbLd;
  const int t = blockIdx.x;
  const int side = 2 * h + 1, npts = side * side, Bm = 2 * bm + 1;
  const int tj = div_ncomp(t, ncomp_max), j = j0 + tj, c = t - tj * ncomp_max;
  const LithoJob job = jobs[j];
  if (c >= job.ncomp) return;
  fill_lane_twiddles(tw, L, twL, 1);
  __syncthreads();
  const int col0 = (blockIdx.y * kWfWarps + warp) * LPW;
  if (col0 >= side) return;
  const float2* tp = table + ((size_t)job.tab * ncomp_max + c) * npts;
  const float2* m = Mb + (size_t)job.clip * Bm * Bm;
  float2 x[32];
#pragma unroll
  for (int l = 0; l < LPW; ++l) {
    const int kxi = col0 + l;
    const int mx = job.cx + (kxi - h) + bm;
    const bool col_ok = kxi < side && mx >= 0 && mx < Bm;
#pragma unroll
    for (int q = 0; q < R; ++q) {
      const int i = lane + 32 * q;
      const int ky = i <= h ? i : i - L;  // in [-h, h] when i <= h or i >= L - h
      float2 v = make_float2(0.f, 0.f);
      const int my = job.cy + ky + bm;
      if (col_ok && (i <= h || i >= L - h) && my >= 0 && my < Bm)
        v = cmul(__ldg(tp + (ky + h) * side + kxi), __ldg(m + (size_t)my * Bm + mx));
      x[l * R + q] = v;
    }
  }
  warp_fft_lines<L, +1>(x, tb, tw);
  const int kxi = col0 + lane / R;
  if (kxi < side) {
    float2* dst = T + ((size_t)t * side + kxi) * L + lane % R;
#pragma unroll
    for (int s = 0; s < 32; ++s) dst[R * s] = x[s];
  }
}

// Pass B. Grid (item, chunk of kWfWarps * LPW rows v). Adds the item's
// transforms whose jobs lie in [j0, j0 + nj) to partial[item][v][u]; each
// lane keeps its J values in registers (L <= 256) or in its warp's rows in
// shared memory across the transforms.
template <int L>
__global__ void __launch_bounds__(kWfWarps * 32, 2)
k_wide_rows_w(const LithoItem* __restrict__ items, const LithoJob* __restrict__ jobs, int j0, int nj,
              int ncomp_max, int h, const float2* __restrict__ twL, const float2* __restrict__ T,
              float* __restrict__ partial) {
  constexpr int R = L / 32, LPW = 32 / R;
  extern __shared__ float2 wsm[];
  float2* tw = wsm;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float2* tb = wsm + L + warp * 32 * kTbLd;
  const LithoItem it = items[blockIdx.x];
  const int jb = it.job_begin > j0 ? it.job_begin : j0;
  const int je = it.job_end < j0 + nj ? it.job_end : j0 + nj;
  if (jb >= je) return;
  fill_lane_twiddles(tw, L, twL, 1);
  __syncthreads();
  const int side = 2 * h + 1;
  const int v0 = (blockIdx.y * kWfWarps + warp) * LPW;
  float* pj = partial + ((size_t)blockIdx.x * L + v0 + lane / R) * L + lane % R;
  float Jr[wf_j_regs(L) ? 32 : 1];
  float* Js = reinterpret_cast<float*>(wsm + L + kWfWarps * 32 * kTbLd) + warp * 32 * 32 + lane;  // [s][lane]
#pragma unroll
  for (int s = 0; s < 32; ++s) {
    if constexpr (wf_j_regs(L)) Jr[s] = pj[R * s];
    else Js[s * 32] = pj[R * s];
  }
  for (int jj = jb; jj < je; ++jj) {
    const LithoJob job = jobs[jj];
    const float w = (float)job.weight;
    for (int c = 0; c < job.ncomp; ++c) {
      const float2* Tt = T + (size_t)((jj - j0) * ncomp_max + c) * side * L + v0;
      float2 x[32];
#pragma unroll
      for (int l = 0; l < LPW; ++l) {
#pragma unroll
        for (int q = 0; q < R; ++q) {
          const int i = lane + 32 * q;
          const int kx = i <= h ? i : i - L;
          x[l * R + q] = (i <= h || i >= L - h) ? Tt[(size_t)(kx + h) * L + l] : make_float2(0.f, 0.f);
        }
      }
      warp_fft_lines<L, +1>(x, tb, tw);
#pragma unroll
      for (int s = 0; s < 32; ++s) {
        if constexpr (wf_j_regs(L)) Jr[s] = fmaf(w, cabs2(x[s]), Jr[s]);
        else Js[s * 32] = fmaf(w, cabs2(x[s]), Js[s * 32]);
      }
    }
  }
#pragma unroll
  for (int s = 0; s < 32; ++s) pj[R * s] = wf_j_regs(L) ? Jr[s] : Js[s * 32];
}

template <int L>
static cudaError_t launch_wide_passes_l(const LithoAbbePlan& p, int j0, int nj, const LithoItem* items,
                                        const LithoJob* jobs, const float2* table, const float2* mb,
                                        const float2* twL, float2* T, float* partial, cudaStream_t s) {
  constexpr int R = L / 32, LPW = 32 / R;
  const int side = 2 * p.h + 1;
  const size_t sm = wf_smem(L), smr = wf_rows_smem(L);
  cudaFuncSetAttribute(k_wide_cols_w<L>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  cudaFuncSetAttribute(k_wide_rows_w<L>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smr);
  dim3 ga(nj * p.ncomp_max, (side + kWfWarps * LPW - 1) / (kWfWarps * LPW));
  k_wide_cols_w<L><<<ga, kWfWarps * 32, sm, s>>>(jobs, j0, p.ncomp_max, table, p.h, mb, p.bm, twL, T);
  dim3 gb(p.n_items, L / (kWfWarps * LPW));
  k_wide_rows_w<L><<<gb, kWfWarps * 32, smr, s>>>(items, jobs, j0, nj, p.ncomp_max, p.h, twL, T, partial);
  return cudaGetLastError();
}

static cudaError_t launch_wide_passes(const LithoAbbePlan& p, int j0, int nj, const LithoItem* items,
                                      const LithoJob* jobs, const float2* table, const float2* mb,
                                      const float2* twL, float2* T, float* partial, cudaStream_t s) {
  switch (p.L) {
    case 128: return launch_wide_passes_l<128>(p, j0, nj, items, jobs, table, mb, twL, T, partial, s);
    case 256: return launch_wide_passes_l<256>(p, j0, nj, items, jobs, table, mb, twL, T, partial, s);
    case 512: return launch_wide_passes_l<512>(p, j0, nj, items, jobs, table, mb, twL, T, partial, s);
    case 1024: return launch_wide_passes_l<1024>(p, j0, nj, items, jobs, table, mb, twL, T, partial, s);
    default: return cudaErrorInvalidValue;
  }
}

// ---------------------------------------------------------------------------
// 2-D transforms of L x L planes (the coarse-grid J and g_L) with the warp
// register FFT: rows straight from global memory (a warp takes 1024 / L rows,
// coalesced both ways), then columns through a padded shared-memory tile of
// 8 x 1024 / L columns (coalesced row segments in and out). Same sums as
// plain_fft2: out = scale_cols * FFT_cols(scale_rows * FFT_rows(in)),
// SIGN = +1 unnormalised inverse, -1 forward.
// ---------------------------------------------------------------------------
template <int L, int SIGN, bool REAL>
__global__ void __launch_bounds__(kWfWarps * 32, 2)
k_wfft_rows(const void* __restrict__ in, float2* __restrict__ out, long long n_rows, float scale,
            const float2* __restrict__ twL) {
  constexpr int R = L / 32, LPW = 32 / R;
  extern __shared__ float2 wsm[];
  float2* tw = wsm;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float2* tb = wsm + L + warp * 32 * kTbLd;
  fill_lane_twiddles(tw, L, twL, 1);
  __syncthreads();
  const long long groups = n_rows / LPW;
  for (long long gi = (long long)blockIdx.x * kWfWarps + warp; gi < groups; gi += (long long)gridDim.x * kWfWarps) {
    const long long r0 = gi * LPW;
    float2 x[32];
#pragma unroll
    for (int l = 0; l < LPW; ++l) {
#pragma unroll
      for (int q = 0; q < R; ++q) {
        const size_t g = (size_t)(r0 + l) * L + lane + 32 * q;
        x[l * R + q] = REAL ? make_float2(reinterpret_cast<const float*>(in)[g], 0.f)
                            : reinterpret_cast<const float2*>(in)[g];
      }
    }
    warp_fft_lines<L, SIGN>(x, tb, tw);   // lane: row r0 + lane / R, index lane % R + R s
    float2* dst = out + (size_t)(r0 + lane / R) * L + lane % R;
#pragma unroll
    for (int s = 0; s < 32; ++s) dst[R * s] = cscale(x[s], scale);
  }
}

template <int L, int SIGN>
__global__ void __launch_bounds__(kWfWarps * 32, 1)
k_wfft_cols(float2* __restrict__ buf, long long planes, float scale, const float2* __restrict__ twL) {
  constexpr int R = L / 32, LPW = 32 / R, TC = kWfWarps * LPW, PT = TC + 1;
  extern __shared__ float2 wsm[];
  float2* tw = wsm;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float2* tb = wsm + L + warp * 32 * kTbLd;
  float2* tile = wsm + L + kWfWarps * 32 * kTbLd;   // [row][TC + 1]
  fill_lane_twiddles(tw, L, twL, 1);
  __syncthreads();
  const long long tiles = planes * (L / TC);
  for (long long t = blockIdx.x; t < tiles; t += gridDim.x) {
    float2* base = buf + (size_t)(t / (L / TC)) * L * L + (size_t)(t % (L / TC)) * TC;
    for (int id = threadIdx.x; id < L * TC; id += blockDim.x) {
      const int r = id / TC, c = id - r * TC;
      tile[r * PT + c] = base[(size_t)r * L + c];
    }
    __syncthreads();
    float2 x[32];
#pragma unroll
    for (int l = 0; l < LPW; ++l) {
#pragma unroll
      for (int q = 0; q < R; ++q) x[l * R + q] = tile[(lane + 32 * q) * PT + warp * LPW + l];
    }
    warp_fft_lines<L, SIGN>(x, tb, tw);   // lane: column warp LPW + lane / R, row lane % R + R s
    __syncthreads();                      // every warp has read the tile
#pragma unroll
    for (int s = 0; s < 32; ++s) tile[(lane % R + R * s) * PT + warp * LPW + lane / R] = cscale(x[s], scale);
    __syncthreads();
    for (int id = threadIdx.x; id < L * TC; id += blockDim.x) {
      const int r = id / TC, c = id - r * TC;
      base[(size_t)r * L + c] = tile[r * PT + c];
    }
    __syncthreads();
  }
}

template <int L>
static cudaError_t wfft2_l(const void* in, bool in_real, float2* buf, long long planes, int sign, float scale_rows,
                           float scale_cols, const float2* twL, cudaStream_t s) {
  constexpr int R = L / 32, LPW = 32 / R, TC = kWfWarps * LPW;
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (sms <= 0) sms = 148;
  const size_t smr = wf_smem(L), smc = wf_smem(L) + (size_t)L * (TC + 1) * 8;
  const long long rows = planes * L, groups = rows / LPW;
  const int gr = (int)std::min<long long>((groups + kWfWarps - 1) / kWfWarps, 2LL * sms);
  const int gc = (int)std::min<long long>(planes * (L / TC), (long long)sms);
  const void* src = in ? in : buf;
  if (sign > 0) {
    cudaFuncSetAttribute(k_wfft_rows<L, 1, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smr);
    k_wfft_rows<L, 1, false><<<gr, kWfWarps * 32, smr, s>>>(src, buf, rows, scale_rows, twL);
    cudaFuncSetAttribute(k_wfft_cols<L, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smc);
    k_wfft_cols<L, 1><<<gc, kWfWarps * 32, smc, s>>>(buf, planes, scale_cols, twL);
  } else {
    if (in_real) {
      cudaFuncSetAttribute(k_wfft_rows<L, -1, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smr);
      k_wfft_rows<L, -1, true><<<gr, kWfWarps * 32, smr, s>>>(src, buf, rows, scale_rows, twL);
    } else {
      cudaFuncSetAttribute(k_wfft_rows<L, -1, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smr);
      k_wfft_rows<L, -1, false><<<gr, kWfWarps * 32, smr, s>>>(src, buf, rows, scale_rows, twL);
    }
    cudaFuncSetAttribute(k_wfft_cols<L, -1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smc);
    k_wfft_cols<L, -1><<<gc, kWfWarps * 32, smc, s>>>(buf, planes, scale_cols, twL);
  }
  return cudaGetLastError();
}

// plain_fft2 for the wide engine's coarse grids: L in {128 .. 1024} on the
// warp register FFT, other sizes through plain_fft2.
static cudaError_t wide_fft2(const void* in, bool in_real, float2* buf, long long planes, int L, int sign,
                             float scale_rows, float scale_cols, const float2* twL, cudaStream_t s) {
  switch (L) {
    case 128: return wfft2_l<128>(in, in_real, buf, planes, sign, scale_rows, scale_cols, twL, s);
    case 256: return wfft2_l<256>(in, in_real, buf, planes, sign, scale_rows, scale_cols, twL, s);
    case 512: return wfft2_l<512>(in, in_real, buf, planes, sign, scale_rows, scale_cols, twL, s);
    case 1024: return wfft2_l<1024>(in, in_real, buf, planes, sign, scale_rows, scale_cols, twL, s);
    default: return plain_fft2(in, in_real, buf, planes, L, sign, scale_rows, scale_cols, twL, s);
  }
}

// J[o] = sum of its items' partials, in item order.
__global__ void k_wide_reduce(const int32_t* __restrict__ out_items, const float* __restrict__ partial, int LL,
                              float* __restrict__ J) {
  const int o = blockIdx.y;
  const int i0 = out_items[o], i1 = out_items[o + 1];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < LL; i += gridDim.x * blockDim.x) {
    float acc = 0.f;
    for (int it = i0; it < i1; ++it) acc += partial[(size_t)it * LL + i];
    J[(size_t)o * LL + i] = acc;
  }
}

// Image band box B(g) = F(g mod L), |g| <= 2h (F already scaled by 1/L^2).
// transposed: F is the transform of J^T (the work queue's pass B stores the
// partials column by column), so B(gx, gy) = F(gy, gx).
__global__ void k_wide_box(const float2* __restrict__ F, int L, int h, float2* __restrict__ bbox,
                           int transposed) {
  const int o = blockIdx.y, G = 4 * h + 1, g0 = 2 * h;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < G * G; i += gridDim.x * blockDim.x) {
    int gy = (i / G - g0) & (L - 1), gx = (i % G - g0) & (L - 1);
    if (transposed) {
      const int t = gx;
      gx = gy;
      gy = t;
    }
    bbox[(size_t)o * G * G + i] = F[((size_t)o * L + gy) * L + gx];
  }
}

// Synthesis of two outputs per complex transform with the warp register FFT:
// Z = I_a + i I_b from the boxes' sum D = B_a + i B_b (B Hermitian, so each
// image is real). Column stage: for every gx in [-g0, g0] the inverse N-point
// transform over gy of D(gx, .) -> Cw[pair][gx + g0][y]; row stage: for every
// y the inverse transform over gx of Cw[pair][.][y] -> the two images' rows.
// N = SPLIT L (L <= 1024) by decimation in frequency: output x = SPLIT m + e
// comes from the L-point transform of y_e(x') = w_N^(e x')
// sum_t d(x' + t L) w_SPLIT^(e t).
template <int L, int SPLIT, class Load>
__device__ __forceinline__ void band_ifft_e(int e, int g0, const Load& ld, float2 (&x)[32], float2* tb,
                                            const float2* tw, const float2* __restrict__ twN) {
  constexpr int R = L / 32, LPW = 32 / R, N = L * SPLIT;
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int l = 0; l < LPW; ++l) {
#pragma unroll
    for (int q = 0; q < R; ++q) {
      const int xp = lane + 32 * q;
      float2 acc = make_float2(0.f, 0.f);
#pragma unroll
      for (int t = 0; t < SPLIT; ++t) {
        const int idx = xp + t * L;
        if (idx <= g0 || idx >= N - g0) {
          float2 v = ld(l, idx <= g0 ? idx : idx - N);
          if (SPLIT > 1 && t > 0 && e > 0) v = cmul(v, __ldg(twN + ((e * t * L) & (N - 1))));
          acc = cadd(acc, v);
        }
      }
      if (SPLIT > 1 && e > 0) acc = cmul(acc, __ldg(twN + ((e * xp) & (N - 1))));
      x[l * R + q] = acc;
    }
  }
  warp_fft_lines<L, +1>(x, tb, tw);  // lane: line lane / R, output SPLIT (lane % R + R s) + e
}

template <int L, int SPLIT>
__global__ void __launch_bounds__(kWfWarps * 32, 2)
k_wsyn_cols(const float2* __restrict__ bbox, int o0, int n_out, int g0, const float2* __restrict__ twN,
            float2* __restrict__ Cw) {
  constexpr int R = L / 32, LPW = 32 / R, N = L * SPLIT;
  extern __shared__ float2 wsm[];
  float2* tw = wsm;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float2* tb = wsm + L + warp * 32 * kTbLd;
  fill_lane_twiddles(tw, L, twN, SPLIT);
  __syncthreads();
  const int pr = blockIdx.y, G = 2 * g0 + 1;
  const int c0 = (blockIdx.x * kWfWarps + warp) * LPW;
  if (c0 >= G) return;
  const int oa = o0 + 2 * pr, ob = oa + 1;
  const float2* Ba = bbox + (size_t)oa * G * G;
  const float2* Bb = bbox + (size_t)ob * G * G;
  const bool has_b = ob < n_out;
  auto ld = [&](int l, int gy) -> float2 {
    const int gxi = c0 + l;
    if (gxi >= G) return make_float2(0.f, 0.f);
    const float2 a = __ldg(Ba + (gy + g0) * G + gxi);
    const float2 b = has_b ? __ldg(Bb + (gy + g0) * G + gxi) : make_float2(0.f, 0.f);
    return make_float2(a.x - b.y, a.y + b.x);
  };
  const int gxi = c0 + lane / R;
  float2* dst = Cw + ((size_t)pr * G + gxi) * N;
  for (int e = 0; e < SPLIT; ++e) {
    float2 x[32];
    band_ifft_e<L, SPLIT>(e, g0, ld, x, tb, tw, twN);
    if (gxi < G) {
#pragma unroll
      for (int sidx = 0; sidx < 32; ++sidx) dst[SPLIT * (lane % R + R * sidx) + e] = x[sidx];
    }
  }
}

// Row stage, writing the images (times the mode-0 scale) and kWideMaxBlk block
// maxima of each raw image (block b of the grid takes rows b, b + kWideMaxBlk,
// ... in units of the block's kWfWarps * LPW rows).
template <int L, int SPLIT>
__global__ void __launch_bounds__(kWfWarps * 32, 2)
k_wsyn_rows(const float2* __restrict__ Cw, int o0, int n_out, int g0, const float2* __restrict__ twN,
            const LithoNorm* __restrict__ norm, float* __restrict__ image, float* __restrict__ blockmax) {
  constexpr int R = L / 32, LPW = 32 / R, N = L * SPLIT;
  extern __shared__ float2 wsm[];
  __shared__ float red[2][kWfWarps];
  float2* tw = wsm;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float2* tb = wsm + L + warp * 32 * kTbLd;
  fill_lane_twiddles(tw, L, twN, SPLIT);
  __syncthreads();
  const int pr = blockIdx.y, G = 2 * g0 + 1;
  const int oa = o0 + 2 * pr, ob = oa + 1;
  const bool has_b = ob < n_out;
  const LithoNorm na = norm ? norm[oa] : LithoNorm{0, 1.0f};
  const LithoNorm nb = (norm && has_b) ? norm[ob] : LithoNorm{0, 1.0f};
  const float sa = na.mode == 1 ? 1.0f : na.scale, sb = nb.mode == 1 ? 1.0f : nb.scale;
  const float2* Cp = Cw + (size_t)pr * G * N;
  float* ia = image + (size_t)oa * N * N;
  float* ib = image + (size_t)ob * N * N;
  float mxa = 0.f, mxb = 0.f;
  for (int y0 = (blockIdx.x * kWfWarps + warp) * LPW; y0 < N; y0 += kWideMaxBlk * kWfWarps * LPW) {
    auto ld = [&](int l, int gx) -> float2 { return Cp[(size_t)(gx + g0) * N + y0 + l]; };
    const int y = y0 + lane / R;
    for (int e = 0; e < SPLIT; ++e) {
      float2 x[32];
      band_ifft_e<L, SPLIT>(e, g0, ld, x, tb, tw, twN);
#pragma unroll
      for (int sidx = 0; sidx < 32; ++sidx) {
        const size_t off = (size_t)y * N + SPLIT * (lane % R + R * sidx) + e;
        mxa = fmaxf(mxa, x[sidx].x);
        ia[off] = x[sidx].x * sa;
        if (has_b) {
          mxb = fmaxf(mxb, x[sidx].y);
          ib[off] = x[sidx].y * sb;
        }
      }
    }
  }
  if (!blockmax) return;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    mxa = fmaxf(mxa, __shfl_xor_sync(0xffffffffu, mxa, off));
    mxb = fmaxf(mxb, __shfl_xor_sync(0xffffffffu, mxb, off));
  }
  if (lane == 0) {
    red[0][warp] = mxa;
    red[1][warp] = mxb;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    float a = red[0][0], b = red[1][0];
    for (int i = 1; i < kWfWarps; ++i) {
      a = fmaxf(a, red[0][i]);
      b = fmaxf(b, red[1][i]);
    }
    blockmax[(size_t)oa * kWideMaxBlk + blockIdx.x] = a;
    if (has_b) blockmax[(size_t)ob * kWideMaxBlk + blockIdx.x] = b;
  }
}

template <int L, int SPLIT>
static cudaError_t launch_wsyn_l(const float2* bbox, int o0, int n_out, int g0, int pairs, const float2* twN,
                                 const LithoNorm* norm, float* image, float* blockmax, float2* Cw, cudaStream_t s) {
  constexpr int R = L / 32, LPW = 32 / R;
  const int G = 2 * g0 + 1;
  const size_t sm = wf_smem(L);
  cudaFuncSetAttribute(k_wsyn_cols<L, SPLIT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  cudaFuncSetAttribute(k_wsyn_rows<L, SPLIT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  k_wsyn_cols<L, SPLIT><<<dim3((G + kWfWarps * LPW - 1) / (kWfWarps * LPW), pairs), kWfWarps * 32, sm, s>>>(
      bbox, o0, n_out, g0, twN, Cw);
  k_wsyn_rows<L, SPLIT><<<dim3(kWideMaxBlk, pairs), kWfWarps * 32, sm, s>>>(Cw, o0, n_out, g0, twN, norm, image,
                                                                            blockmax);
  return cudaGetLastError();
}

// Images o0 .. o0 + 2 pairs - 1 (clipped to n_out) from their boxes of
// half-width g0 (2 g0 + 1 <= n); Cw: pairs x (2 g0 + 1) x n complex.
static cudaError_t wide_synth_pairs_w(const float2* bbox, int o0, int n_out, int g0, int n, int pairs,
                                      const float2* twN, const LithoNorm* norm, float* image, float* blockmax,
                                      float2* Cw, cudaStream_t s) {
  switch (n) {
    case 128: return launch_wsyn_l<128, 1>(bbox, o0, n_out, g0, pairs, twN, norm, image, blockmax, Cw, s);
    case 256: return launch_wsyn_l<256, 1>(bbox, o0, n_out, g0, pairs, twN, norm, image, blockmax, Cw, s);
    case 512: return launch_wsyn_l<512, 1>(bbox, o0, n_out, g0, pairs, twN, norm, image, blockmax, Cw, s);
    case 1024: return launch_wsyn_l<1024, 1>(bbox, o0, n_out, g0, pairs, twN, norm, image, blockmax, Cw, s);
    case 2048: return launch_wsyn_l<1024, 2>(bbox, o0, n_out, g0, pairs, twN, norm, image, blockmax, Cw, s);
    case 4096: return launch_wsyn_l<1024, 4>(bbox, o0, n_out, g0, pairs, twN, norm, image, blockmax, Cw, s);
    default: return cudaErrorInvalidValue;
  }
}

// ---------------------------------------------------------------------------
// SOCS adjoint on wide coarse grids (the ILT gradient for kernel bands wider
// than 15 bins; opc/ilt.py:262-266 restated as in ilt.cu's file comment):
//   e_k = IFFT_L(phi_k M)  (pass A, k_wide_cols, then the row inverse below)
//   Y_k = FFT_L(e_k g_L) / L^2 on |f| <= h,  g_L = IFFT_L(sens band box)
//   A(f) = sum_k lambda_k conj(phi_k(f)) Y_k(f),  H(f) = A(f) + conj A(-f).
// ---------------------------------------------------------------------------

// g_L: the (4h+1)^2 sensitivity box scattered onto the L x L grid.
__global__ void k_wide_scatter_box(const float2* __restrict__ box, int g0, int L, float2* __restrict__ grid) {
  const int c = blockIdx.y, G = 2 * g0 + 1;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < G * G; i += gridDim.x * blockDim.x) {
    const int gy = i / G - g0, gx = i % G - g0;
    grid[((size_t)c * L + (gy & (L - 1))) * L + (gx & (L - 1))] = box[(size_t)c * G * G + i];
  }
}

// Register-FFT forms of the adjoint passes. Pass B of the adjoint, per warp
// LPW rows v of one transform: the row inverse of T (as in pass B), times
// g_L(., v), the forward transform of that product, the band fx in [-h, h]
// -> T2[t][fx + h][v]. Between the two transforms the product goes through the
// warp's buffer as LPW rows of pitch L + R, from the output layout of one
// transform into the input layout of the next.
template <int L>
__global__ void __launch_bounds__(kWfWarps * 32, 2)
k_wide_adj_rows_w(const LithoJob* __restrict__ jobs, int j0, int h, const float2* __restrict__ twL,
                  const float2* __restrict__ T, const float2* __restrict__ gL, float2* __restrict__ T2) {
  constexpr int R = L / 32, LPW = 32 / R, PITCH = L + R;
  static_assert(LPW * PITCH <= 32 * kTbLd, "row buffer fits the transpose buffer");
  extern __shared__ float2 wsm[];
  float2* tw = wsm;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float2* tb = wsm + L + warp * 32 * kTbLd;
  fill_lane_twiddles(tw, L, twL, 1);
  __syncthreads();
  const int t = blockIdx.x, side = 2 * h + 1;
  const int v0 = (blockIdx.y * kWfWarps + warp) * LPW;
  const LithoJob job = jobs[j0 + t];
  const float2* Tt = T + (size_t)t * side * L + v0;
  float2 x[32];
#pragma unroll
  for (int l = 0; l < LPW; ++l) {
#pragma unroll
    for (int q = 0; q < R; ++q) {
      const int i = lane + 32 * q;
      const int kx = i <= h ? i : i - L;
      x[l * R + q] = (i <= h || i >= L - h) ? Tt[(size_t)(kx + h) * L + l] : make_float2(0.f, 0.f);
    }
  }
  warp_fft_lines<L, +1>(x, tb, tw);  // lane: row v0 + lane / R, u = lane % R + R s
  {
    const int lp = lane / R, rp = lane % R;
    const float2* g = gL + ((size_t)job.clip * L + v0 + lp) * L + rp;
#pragma unroll
    for (int sidx = 0; sidx < 32; ++sidx) tb[lp * PITCH + rp + R * sidx] = cmul(x[sidx], __ldg(g + R * sidx));
  }
  __syncwarp();
#pragma unroll
  for (int l = 0; l < LPW; ++l) {
#pragma unroll
    for (int q = 0; q < R; ++q) x[l * R + q] = tb[l * PITCH + lane + 32 * q];
  }
  __syncwarp();
  warp_fft_lines<L, -1>(x, tb, tw);  // lane: row v0 + lane / R, fx = lane % R + R s (mod L)
  const int lp = lane / R, rp = lane % R;
  float2* dst = T2 + (size_t)t * side * L + v0 + lp;
#pragma unroll
  for (int sidx = 0; sidx < 32; ++sidx) {
    const int f = rp + R * sidx;
    const int fx = f <= h ? f : f - L;
    if (f <= h || f >= L - h) dst[(size_t)(fx + h) * L] = x[sidx];
  }
}

// Pass C of the adjoint, per warp LPW columns fx of one transform: forward
// over v of T2[t][fx][.], the band fy in [-h, h], weighted:
// Yt[t][fy + h][fx + h] = lambda conj(phi(fx, fy)) Y / L^2.
template <int L>
__global__ void __launch_bounds__(kWfWarps * 32, 2)
k_wide_adj_cols_w(const LithoJob* __restrict__ jobs, int j0, const float2* __restrict__ table, int h,
                  const float2* __restrict__ twL, const float2* __restrict__ T2, float2* __restrict__ Yt) {
  constexpr int R = L / 32, LPW = 32 / R;
  extern __shared__ float2 wsm[];
  float2* tw = wsm;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float2* tb = wsm + L + warp * 32 * kTbLd;
  fill_lane_twiddles(tw, L, twL, 1);
  __syncthreads();
  const int t = blockIdx.x, side = 2 * h + 1, npts = side * side;
  const int c0 = (blockIdx.y * kWfWarps + warp) * LPW;
  if (c0 >= side) return;
  const LithoJob job = jobs[j0 + t];
  const float2* src = T2 + (size_t)t * side * L;
  float2 x[32];
#pragma unroll
  for (int l = 0; l < LPW; ++l) {
    const int fxi = c0 + l;
#pragma unroll
    for (int q = 0; q < R; ++q)
      x[l * R + q] = fxi < side ? src[(size_t)fxi * L + lane + 32 * q] : make_float2(0.f, 0.f);
  }
  warp_fft_lines<L, -1>(x, tb, tw);  // lane: column c0 + lane / R, fy = lane % R + R s (mod L)
  const int fxi = c0 + lane / R, rp = lane % R;
  if (fxi >= side) return;
  const float2* ph = table + (size_t)job.tab * npts;
  const float sc = (float)job.weight / ((float)L * (float)L);
  float2* dst = Yt + (size_t)t * npts;
#pragma unroll
  for (int sidx = 0; sidx < 32; ++sidx) {
    const int f = rp + R * sidx;
    const int fy = f <= h ? f : f - L;
    if (f <= h || f >= L - h) {
      const int fyi = fy + h;
      dst[fyi * side + fxi] = cscale(cmulc(x[sidx], __ldg(ph + fyi * side + fxi)), sc);
    }
  }
}

template <int L>
static cudaError_t launch_wide_adjoint_l(int j0, int nj, const LithoJob* jobs, const float2* table, int h,
                                         const float2* mask_box, const float2* twL, float2* T, const float2* gL,
                                         float2* T2, float2* Yt, cudaStream_t s) {
  constexpr int R = L / 32, LPW = 32 / R;
  const int side = 2 * h + 1;
  const size_t sm = wf_smem(L);
  cudaFuncSetAttribute(k_wide_cols_w<L>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  cudaFuncSetAttribute(k_wide_adj_rows_w<L>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  cudaFuncSetAttribute(k_wide_adj_cols_w<L>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  const dim3 gc(nj, (side + kWfWarps * LPW - 1) / (kWfWarps * LPW));
  k_wide_cols_w<L><<<gc, kWfWarps * 32, sm, s>>>(jobs, j0, 1, table, h, mask_box, h, twL, T);
  k_wide_adj_rows_w<L><<<dim3(nj, L / (kWfWarps * LPW)), kWfWarps * 32, sm, s>>>(jobs, j0, h, twL, T, gL, T2);
  k_wide_adj_cols_w<L><<<gc, kWfWarps * 32, sm, s>>>(jobs, j0, table, h, twL, T2, Yt);
  return cudaGetLastError();
}

static cudaError_t launch_wide_adjoint(int L, int j0, int nj, const LithoJob* jobs, const float2* table, int h,
                                       const float2* mask_box, const float2* twL, float2* T, const float2* gL,
                                       float2* T2, float2* Yt, cudaStream_t s) {
  switch (L) {
    case 128: return launch_wide_adjoint_l<128>(j0, nj, jobs, table, h, mask_box, twL, T, gL, T2, Yt, s);
    case 256: return launch_wide_adjoint_l<256>(j0, nj, jobs, table, h, mask_box, twL, T, gL, T2, Yt, s);
    case 512: return launch_wide_adjoint_l<512>(j0, nj, jobs, table, h, mask_box, twL, T, gL, T2, Yt, s);
    case 1024: return launch_wide_adjoint_l<1024>(j0, nj, jobs, table, h, mask_box, twL, T, gL, T2, Yt, s);
    default: return cudaErrorInvalidValue;
  }
}

// A[clip] += Yt[t] for the chunk's transforms, in job order; each run of
// consecutive jobs of one clip is summed in registers and stored once.
__global__ void k_wide_adj_acc(const LithoJob* __restrict__ jobs, int j0, int nj, int npts,
                               const float2* __restrict__ Yt, float2* __restrict__ A) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npts; i += gridDim.x * blockDim.x) {
    int t = 0;
    while (t < nj) {
      const int c = jobs[j0 + t].clip;
      float2 acc = A[(size_t)c * npts + i];
#pragma unroll 4
      for (; t < nj && jobs[j0 + t].clip == c; ++t) acc = cadd(acc, __ldcs(Yt + (size_t)t * npts + i));
      A[(size_t)c * npts + i] = acc;
    }
  }
}

// H(f) = A(f) + conj A(-f).
__global__ void k_wide_adj_final(const float2* __restrict__ A, int h, float2* __restrict__ H) {
  const int c = blockIdx.y, side = 2 * h + 1, npts = side * side;
  for (int id = blockIdx.x * blockDim.x + threadIdx.x; id < npts; id += gridDim.x * blockDim.x) {
    const int fy = id / side, fx = id % side;
    const int mid = (2 * h - fy) * side + (2 * h - fx);
    H[(size_t)c * npts + id] = cadd(A[(size_t)c * npts + id], cconj(A[(size_t)c * npts + mid]));
  }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
// t_bytes >= 0: the pass-A buffer T is that many bytes (the work queue's
// ring of slots); < 0: chunks of jobs within kWideTBudget.
WideLayout wide_layout(const LithoAbbePlan& p, int64_t t_bytes) {
  WideLayout l{};
  const int64_t Bm = 2 * p.bm + 1, side = 2 * p.h + 1, G = 4 * p.h + 1, L = p.L, NN = (int64_t)p.n * p.n;
  const int64_t per_job = (int64_t)p.ncomp_max * side * L * 8;
  int64_t jc = (t_bytes >= 0 ? t_bytes : kWideTBudget) / per_job;
  if (jc < 1) jc = 1;
  if (jc > p.n_jobs) jc = p.n_jobs;
  l.jobs_per_chunk = (int)jc;
  const int64_t pairs = (p.n_out + 1) / 2 < kWideSpecPairs ? (p.n_out + 1) / 2 : kWideSpecPairs;
  int64_t off = 0;
  l.status = off;   off = align16(off + 16);
  l.twN = off;      off = align16(off + (int64_t)p.n * 8);
  l.twL = off;      off = align16(off + L * 8);
  l.u1 = off;       off = align16(off + (int64_t)p.n_clips * Bm * p.n * 8);
  l.mb = off;       off = align16(off + (int64_t)p.n_clips * Bm * Bm * 8);
  l.table = off;    off = align16(off + (int64_t)p.n_tab * p.ncomp_max * side * side * 8);
  l.T = off;        off = align16(off + (t_bytes >= 0 ? t_bytes : jc * per_job));
  l.partial = off;  off = align16(off + (int64_t)p.n_items * L * L * 4);
  l.J = off;        off = align16(off + (int64_t)p.n_out * L * L * 4);
  l.F = off;        off = align16(off + (int64_t)p.n_out * L * L * 8);
  l.bbox = off;     off = align16(off + (int64_t)p.n_out * G * G * 8);
  l.spec = off;     off = align16(off + pairs * NN * 8);
  l.blockmax = off; off = align16(off + (int64_t)p.n_out * kWideMaxBlk * 4);
  l.total = off;
  return l;
}

// Is this plan one for the wide engine (valid L above 64)?
bool wide_plan_ok(const LithoAbbePlan& p) {
  return p.L >= 128 && p.L <= 1024 && (p.L & (p.L - 1)) == 0 && 4 * p.h + 1 <= p.L && p.L <= p.n &&
         p.n <= 4096 && (p.n & (p.n - 1)) == 0 && p.bm >= p.h;
}

int64_t wide_workspace_bytes(const LithoAbbePlan& p) { return wide_layout(p).total; }

int wide_prepare(const LithoAbbePlan& p, const void* mask, void* ws, const WideLayout& l, cudaStream_t s,
                 int num_sms) {
  char* w = static_cast<char*>(ws);
  int* status = reinterpret_cast<int*>(w + l.status);
  float2* u1 = reinterpret_cast<float2*>(w + l.u1);
  float2* mb = reinterpret_cast<float2*>(w + l.mb);
  const int n = p.n, Bm = 2 * p.bm + 1;
  cudaError_t e;
  if ((e = cudaMemsetAsync(status, 0, sizeof(int), s)) != cudaSuccess) return (int)e;
  const float2* twN = twiddles_for(n, reinterpret_cast<float2*>(w + l.twN), s);
  e = launch_row_band_dft(mask, p.mask_complex != 0, p.n_clips * n, n, n, p.bm, u1, 1.0f, twN, num_sms, s, status);
  if (e != cudaSuccess) return (int)e;
  e = launch_row_band_dft(u1, true, p.n_clips * Bm, Bm, n, p.bm, mb, 1.0f / ((float)n * (float)n), twN, num_sms, s,
                          status);
  return e == cudaSuccess ? LITHO_OK : (int)e;
}

// ev (optional): events recorded after the band box and after the synthesis
static int wide_finish_ev(const LithoAbbePlan& p, const void* blob, float* image, float* peak, void* ws,
                          const WideLayout& l, bool transposed, cudaStream_t s, cudaEvent_t* ev) {
  const char* b = static_cast<const char*>(blob);
  const int32_t* out_items = reinterpret_cast<const int32_t*>(b + p.off_out_items);
  const LithoNorm* norm = reinterpret_cast<const LithoNorm*>(b + p.off_norm);
  char* w = static_cast<char*>(ws);
  float* partial = reinterpret_cast<float*>(w + l.partial);
  float* J = reinterpret_cast<float*>(w + l.J);
  float2* F = reinterpret_cast<float2*>(w + l.F);
  float2* bbox = reinterpret_cast<float2*>(w + l.bbox);
  float2* spec = reinterpret_cast<float2*>(w + l.spec);
  float* blockmax = reinterpret_cast<float*>(w + l.blockmax);
  const int n = p.n, L = p.L, G = 4 * p.h + 1;
  const size_t NN = (size_t)n * n;
  const float2* twN = twiddles_for(n, reinterpret_cast<float2*>(w + l.twN), s);
  const float2* twL = twiddles_for(L, reinterpret_cast<float2*>(w + l.twL), s);
  cudaError_t e;
  const int LL = L * L;
  dim3 gr((LL + 255) / 256 < 1024 ? (LL + 255) / 256 : 1024, p.n_out);
  k_wide_reduce<<<gr, 256, 0, s>>>(out_items, partial, LL, J);
  e = wide_fft2(J, true, F, p.n_out, L, -1, 1.0f, 1.0f / ((float)L * (float)L), twL, s);
  if (e != cudaSuccess) return (int)e;
  dim3 gx((G * G + 255) / 256, p.n_out);
  k_wide_box<<<gx, 256, 0, s>>>(F, L, p.h, bbox, transposed ? 1 : 0);
  if ((e = cudaGetLastError()) != cudaSuccess) return (int)e;
  if (ev) cudaEventRecord(ev[0], s);
  for (int o0 = 0; o0 < p.n_out; o0 += 2 * kWideSpecPairs) {
    const int no = (p.n_out - o0) < 2 * kWideSpecPairs ? (p.n_out - o0) : 2 * kWideSpecPairs;
    const int pairs = (no + 1) / 2;
    e = wide_synth_pairs_w(bbox, o0, p.n_out, 2 * p.h, n, pairs, twN, norm, image, blockmax, spec, s);
    if (e != cudaSuccess) return (int)e;
  }
  if (ev) cudaEventRecord(ev[1], s);
  dim3 gn((unsigned)((NN + 255) / 256 < 512 ? (NN + 255) / 256 : 512), p.n_out);
  k_normalise<<<gn, 256, 0, s>>>(blockmax, kWideMaxBlk, norm, n, image, peak, 0);
  e = cudaGetLastError();
  return e == cudaSuccess ? LITHO_OK : (int)e;
}

int wide_finish(const LithoAbbePlan& p, const void* blob, float* image, float* peak, void* ws, const WideLayout& l,
                bool transposed, cudaStream_t s) {
  return wide_finish_ev(p, blob, image, peak, ws, l, transposed, s, nullptr);
}

int abbe_wide_run(const LithoAbbePlan& p, const void* blob, const void* table_in, const void* mask, float* image,
                  float* peak, void* ws, cudaStream_t s, int num_sms, cudaEvent_t* ev) {
  const WideLayout l = wide_layout(p);
  const char* b = static_cast<const char*>(blob);
  const LithoJob* jobs = reinterpret_cast<const LithoJob*>(b + p.off_jobs);
  const LithoItem* items = reinterpret_cast<const LithoItem*>(b + p.off_items);
  char* w = static_cast<char*>(ws);
  float2* mb = reinterpret_cast<float2*>(w + l.mb);
  float2* table = table_in ? (float2*)table_in : reinterpret_cast<float2*>(w + l.table);
  float2* T = reinterpret_cast<float2*>(w + l.T);
  float* partial = reinterpret_cast<float*>(w + l.partial);
  const int L = p.L;
  cudaError_t e;
  auto mark = [&](int i) { if (ev) cudaEventRecord(ev[i], s); };

  mark(0);
  if (!table_in && (e = launch_pupil_table(p, blob, table, s)) != cudaSuccess) return (int)e;
  if ((e = cudaGetLastError()) != cudaSuccess) return (int)e;
  mark(1);
  int st = wide_prepare(p, mask, ws, l, s, num_sms);
  if (st) return st;
  mark(2);
  mark(3);
  // coarse passes, chunk by chunk of jobs
  const float2* twL = twiddles_for(L, reinterpret_cast<float2*>(w + l.twL), s);
  if ((e = cudaMemsetAsync(partial, 0, (size_t)p.n_items * L * L * 4, s)) != cudaSuccess) return (int)e;
  for (int j0 = 0; j0 < p.n_jobs; j0 += l.jobs_per_chunk) {
    const int nj = (p.n_jobs - j0) < l.jobs_per_chunk ? (p.n_jobs - j0) : l.jobs_per_chunk;
    if ((e = launch_wide_passes(p, j0, nj, items, jobs, table, mb, twL, T, partial, s)) != cudaSuccess) return (int)e;
  }
  mark(4);
  st = wide_finish_ev(p, blob, image, peak, ws, l, false, s, ev ? ev + 5 : nullptr);
  if (st) return st;
  mark(7);
  return LITHO_OK;
}

// ---------------------------------------------------------------------------
// wide pieces for the SOCS / ILT stages
// ---------------------------------------------------------------------------
static int wide_L_for(int h) {
  int L = 32;
  while (L < 4 * h + 1) L *= 2;
  return L;
}

bool wide_adjoint_ok(int h) { return h >= 1 && wide_L_for(h) >= 128 && wide_L_for(h) <= 1024; }

static int64_t adj_jobs_per_chunk(int h) {
  const int64_t side = 2 * h + 1, L = wide_L_for(h);
  int64_t jc = kWideTBudget / (side * L * 8 * 2 + side * side * 8);
  return jc < 1 ? 1 : jc;
}

struct WideAdjLayout {
  int64_t twL, gL, T, T2, Yt, A, total;
  int jobs_per_chunk;
};

static WideAdjLayout wide_adj_layout(int n_clips, int h) {
  WideAdjLayout l{};
  const int64_t side = 2 * h + 1, L = wide_L_for(h), jc = adj_jobs_per_chunk(h);
  l.jobs_per_chunk = (int)jc;
  int64_t off = 0;
  l.twL = off; off = align16(off + L * 8);
  l.gL = off;  off = align16(off + (int64_t)n_clips * L * L * 8);
  l.T = off;   off = align16(off + jc * side * L * 8);
  l.T2 = off;  off = align16(off + jc * side * L * 8);
  l.Yt = off;  off = align16(off + jc * side * side * 8);
  l.A = off;   off = align16(off + (int64_t)n_clips * side * side * 8);
  l.total = off;
  return l;
}

int64_t wide_adjoint_ws(int n_clips, int h) { return wide_adj_layout(n_clips, h).total; }

// The SOCS adjoint band box for a plan with one job per (clip, kernel):
// mask_box [clip][(2h+1)^2] (scaled 1/N^2), sens_box [clip][(4h+1)^2] (scale/N^2).
int wide_socs_adjoint(const LithoAbbePlan& p, const void* blob, const float2* table, const float2* mask_box,
                      const float2* sens_box, float2* grad_box, void* ws, cudaStream_t s) {
  const int h = p.h, L = wide_L_for(h), side = 2 * h + 1, npts = side * side;
  const WideAdjLayout l = wide_adj_layout(p.n_clips, h);
  const LithoJob* jobs = reinterpret_cast<const LithoJob*>(static_cast<const char*>(blob) + p.off_jobs);
  char* w = static_cast<char*>(ws);
  float2* twL_own = reinterpret_cast<float2*>(w + l.twL);
  float2* gL = reinterpret_cast<float2*>(w + l.gL);
  float2* T = reinterpret_cast<float2*>(w + l.T);
  float2* T2 = reinterpret_cast<float2*>(w + l.T2);
  float2* Yt = reinterpret_cast<float2*>(w + l.Yt);
  float2* A = reinterpret_cast<float2*>(w + l.A);
  cudaError_t e;
  const float2* twL = twiddles_for(L, twL_own, s);
  if ((e = cudaMemsetAsync(gL, 0, (size_t)p.n_clips * L * L * 8, s)) != cudaSuccess) return (int)e;
  if ((e = cudaMemsetAsync(A, 0, (size_t)p.n_clips * npts * 8, s)) != cudaSuccess) return (int)e;
  const int G = 4 * h + 1;
  k_wide_scatter_box<<<dim3((G * G + 255) / 256, p.n_clips), 256, 0, s>>>(sens_box, 2 * h, L, gL);
  e = wide_fft2(nullptr, false, gL, p.n_clips, L, +1, 1.0f, 1.0f, twL, s);
  if (e != cudaSuccess) return (int)e;
  for (int j0 = 0; j0 < p.n_jobs; j0 += l.jobs_per_chunk) {
    const int nj = (p.n_jobs - j0) < l.jobs_per_chunk ? (p.n_jobs - j0) : l.jobs_per_chunk;
    if ((e = launch_wide_adjoint(L, j0, nj, jobs, table, h, mask_box, twL, T, gL, T2, Yt, s)) != cudaSuccess)
      return (int)e;
    k_wide_adj_acc<<<(npts + 255) / 256, 256, 0, s>>>(jobs, j0, nj, npts, Yt, A);
    if ((e = cudaGetLastError()) != cudaSuccess) return (int)e;
  }
  k_wide_adj_final<<<dim3((npts + 255) / 256, p.n_clips), 256, 0, s>>>(A, h, grad_box);
  e = cudaGetLastError();
  return e == cudaSuccess ? LITHO_OK : (int)e;
}

// The image band box of litho_coarse_image on a wide plan.
int wide_coarse_box(const LithoAbbePlan& p, const void* blob, const float2* table, const float2* mb, float2* bbox_out,
                    void* ws, cudaStream_t s) {
  const WideLayout l = wide_layout(p);
  const char* b = static_cast<const char*>(blob);
  const LithoJob* jobs = reinterpret_cast<const LithoJob*>(b + p.off_jobs);
  const LithoItem* items = reinterpret_cast<const LithoItem*>(b + p.off_items);
  const int32_t* out_items = reinterpret_cast<const int32_t*>(b + p.off_out_items);
  char* w = static_cast<char*>(ws);
  float2* twL_own = reinterpret_cast<float2*>(w + l.twL);
  float2* T = reinterpret_cast<float2*>(w + l.T);
  float* partial = reinterpret_cast<float*>(w + l.partial);
  float* J = reinterpret_cast<float*>(w + l.J);
  float2* F = reinterpret_cast<float2*>(w + l.F);
  const int L = p.L, G = 4 * p.h + 1;
  cudaError_t e;
  const float2* twL = twiddles_for(L, twL_own, s);
  if ((e = cudaMemsetAsync(partial, 0, (size_t)p.n_items * L * L * 4, s)) != cudaSuccess) return (int)e;
  for (int j0 = 0; j0 < p.n_jobs; j0 += l.jobs_per_chunk) {
    const int nj = (p.n_jobs - j0) < l.jobs_per_chunk ? (p.n_jobs - j0) : l.jobs_per_chunk;
    if ((e = launch_wide_passes(p, j0, nj, items, jobs, table, mb, twL, T, partial, s)) != cudaSuccess) return (int)e;
  }
  const int LL = L * L;
  k_wide_reduce<<<dim3((LL + 255) / 256 < 1024 ? (LL + 255) / 256 : 1024, p.n_out), 256, 0, s>>>(out_items, partial,
                                                                                                 LL, J);
  e = wide_fft2(J, true, F, p.n_out, L, -1, 1.0f, 1.0f / ((float)L * (float)L), twL, s);
  if (e != cudaSuccess) return (int)e;
  k_wide_box<<<dim3((G * G + 255) / 256, p.n_out), 256, 0, s>>>(F, L, p.h, bbox_out, 0);
  e = cudaGetLastError();
  return e == cudaSuccess ? LITHO_OK : (int)e;
}

// Real synthesis of n_fields Hermitian boxes of half-width g0 (2 g0 + 1 <= n),
// two boxes per complex transform by the column and row stages above.
// spec: kWideSpecPairs x n x n complex (the column stage's buffer, which
// needs kWideSpecPairs x (2 g0 + 1) x n); twN: exp(+2 pi i j / n).
int64_t wide_synth_spec_bytes(int n_fields, int n) {
  const int64_t pairs = (n_fields + 1) / 2 < kWideSpecPairs ? (n_fields + 1) / 2 : kWideSpecPairs;
  return pairs * (int64_t)n * n * 8;
}

cudaError_t wide_synth_real(const float2* box, int g0, int n, int n_fields, float* out, float2* spec,
                            const float2* twN, cudaStream_t s) {
  cudaError_t e;
  for (int o0 = 0; o0 < n_fields; o0 += 2 * kWideSpecPairs) {
    const int no = (n_fields - o0) < 2 * kWideSpecPairs ? (n_fields - o0) : 2 * kWideSpecPairs;
    const int pairs = (no + 1) / 2;
    if ((e = wide_synth_pairs_w(box, o0, n_fields, g0, n, pairs, twN, nullptr, out, nullptr, spec, s)) != cudaSuccess)
      return e;
  }
  return cudaSuccess;
}

}  // namespace litho
