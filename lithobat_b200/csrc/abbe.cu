// Abbe imaging on the band-limited coarse grid.
//
// The reference sums, per source point s (expose/aerial_image.py:421-488),
//     I(x) = sum_s w_s |ifft2_N(M(f) P(f - f_s))|^2
// with one dense N x N inverse FFT per coherent system. Each coherent field
// E_s has its spectrum on a disc of radius R = NA N px / lambda bins around
// the source offset, so its intensity |E_s|^2 is band-limited to |g| <= 2R.
// Shifting the disc by its integer centre c_s (which leaves |E_s|^2
// unchanged) puts its spectrum in [-h, h]^2, and on any L x L grid with
// L >= 4h + 1 the circular autocorrelation of that spectrum is exact. So:
//
//   1. pupil table : P_s(c_s + d) (x V_c for the vector model), FP64 math,
//                    exact IEEE aperture test — k_pupil_table
//   2. mask band   : M(k) / N^2 for |kx|, |ky| <= bm — band.cu, twice
//   3. coarse      : e = IFFT_L(M P), J += w |e|^2, on chip — k_coarse32
//   4. reduce      : J summed over thread blocks in a fixed order, then
//                    B(g) = FFT_L(J)(g) / L^2 for |g| <= 2h — k_coarse_reduce
//   5. synthesis   : I(x) = sum_g B(g) exp(2 pi i g.x / N), the only pass
//                    over N^2 pixels — k_synth
//   6. normalise   : peak / clear / none (aerial_image.py:217-241) — k_normalise
//
// Every step is deterministic (no floating-point atomics).
#include <cstdio>
#include <cstring>

#include "common.cuh"
#include "pupil.cuh"
#include "rows.cuh"

namespace litho {

cudaError_t launch_row_band_dft(const void* in, bool cplx, int n_rows, int rows_per_clip, int n,
                                int bm, float2* out, float scale, const float2* tw_inv,
                                int num_sms, cudaStream_t st, int* status);
cudaError_t launch_row_band_dft_levels(const uint8_t* in, const float2* levels, int n_levels, int n_rows,
                                       int rows_per_clip, int n, int bm, float2* out, float scale,
                                       const float2* tw_inv, int num_sms, cudaStream_t st);
bool row_band_levels_ok(int n, int bm);
bool wide_plan_ok(const LithoAbbePlan& p);
int64_t wide_workspace_bytes(const LithoAbbePlan& p);
int abbe_wide_run(const LithoAbbePlan& p, const void* blob, const void* table_in, const void* mask, float* image,
                  float* peak, void* ws, cudaStream_t s, int num_sms, cudaEvent_t* ev);
int wide_coarse_box(const LithoAbbePlan& p, const void* blob, const float2* table, const float2* mb, float2* bbox_out,
                    void* ws, cudaStream_t s);

// ---------------------------------------------------------------------------
// 1. pupil table: table[slot][comp][(dy+h)(2h+1) + dx+h], one block per slot,
//    evaluated for the slot's representative job.
// ---------------------------------------------------------------------------
// mirrors (nullptr for thin masks): the blank's reflection per order is
// multiplied in (mask_model="multilayer", expose/m3d/provider.py:280-281).
__global__ void k_pupil_table(const LithoJob* __restrict__ jobs, const int32_t* __restrict__ slots,
                              const LithoPupil* __restrict__ pupils, const LithoMirror* __restrict__ mirrors,
                              int n_tab, int n, double pixel_size, int h, int ncomp_max,
                              float2* __restrict__ table) {
  const int t = blockIdx.x;
  if (t >= n_tab) return;
  const LithoJob job = jobs[slots[t]];
  const LithoPupil P = pupils[job.pupil];
  LithoMirror M{};
  const double* mtab = nullptr;
  if (mirrors) {
    M = mirrors[job.pupil];
    mtab = reinterpret_cast<const double*>(reinterpret_cast<const char*>(mirrors) + M.off_table);
  }
  const int side = 2 * h + 1, npts = side * side;
  const double val = ddiv(1.0, dmul((double)n, pixel_size));
  const double kmax = ddiv(P.NA, P.wavelength);
  float2* out = table + (size_t)t * ncomp_max * npts;
  for (int p = threadIdx.x; p < npts; p += blockDim.x) {
    const int dy = p / side - h, dx = p % side - h;
    const int kx = job.cx + dx, ky = job.cy + dy;
    float2 v[3] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
    if (bin_valid(kx, n) && bin_valid(ky, n)) {
      double fx, fy;
      const double rho = aperture_rho(kx, ky, val, job.fsx, job.fsy, kmax, fx, fy);
      if (rho <= 1.0) {
        if (M.n_theta >= 2) {
          double rr, ri;
          mirror_reflection(M, mtab, bin_freq(kx, val), bin_freq(ky, val), job.fsx, job.fsy, rr, ri);
          pupil_values_scaled(P, rho, fx, fy, job.jx, job.jy, rr, ri, v);
        } else {
          pupil_values(P, rho, fx, fy, job.jx, job.jy, v);
        }
      }
    }
    for (int c = 0; c < ncomp_max; ++c) out[(size_t)c * npts + p] = v[c];
  }
}

// What an unpatterned mask images to, per output: the clear throughput of
// expose/aerial_image.py:_abbe_sum (:464 scalar, :482-486 vector, times the
// blank's specular reflectance |r|^2 for a mirrored mask, :431-438), in FP64.
// At the DC order |exp(iW)| = 1, so a job adds weight x [rho(DC) <= 1] x
// (vector: sum_c |V_c(DC)|^2) x |r|^2. One block per output; each thread sums
// a fixed stride of the output's jobs, then a fixed-order tree: deterministic.
__global__ void k_abbe_clear(const LithoJob* __restrict__ jobs, const LithoItem* __restrict__ items,
                             const int32_t* __restrict__ out_items, const LithoPupil* __restrict__ pupils,
                             const LithoMirror* __restrict__ mirrors, int n, double pixel_size,
                             double* __restrict__ clear_out) {
  __shared__ double red[128];
  const int o = blockIdx.x;
  const double val = ddiv(1.0, dmul((double)n, pixel_size));
  double acc = 0.0;
  for (int it = out_items[o]; it < out_items[o + 1]; ++it) {
    const LithoItem item = items[it];
    for (int j = item.job_begin + (int)threadIdx.x; j < item.job_end; j += blockDim.x) {
      const LithoJob job = jobs[j];
      const LithoPupil P = pupils[job.pupil];
      double fx, fy;
      const double rho = aperture_rho(0, 0, val, job.fsx, job.fsy, ddiv(P.NA, P.wavelength), fx, fy);
      if (!(rho <= 1.0)) continue;
      double t = 1.0;
      if (P.vector) {
        double cp, sp;
        pupil_direction(fx, fy, cp, sp);
        const double s = rho * (P.NA / P.n_image);
        const double s2 = fmin(fmax(s * s, 0.0), 1.0);
        const double ct = sqrt(1.0 - s2), st = sqrt(s2);
        const double es = -job.jx * sp + job.jy * cp, ep = job.jx * cp + job.jy * sp;
        const double vx = -es * sp + ep * ct * cp, vy = es * cp + ep * ct * sp, vz = -ep * st;
        t = vx * vx + vy * vy + vz * vz;
        if (P.obliquity) t *= ct;
      }
      if (mirrors && mirrors[job.pupil].n_theta >= 2) {
        const LithoMirror M = mirrors[job.pupil];
        const double* mtab = reinterpret_cast<const double*>(reinterpret_cast<const char*>(mirrors) + M.off_table);
        double rr, ri;
        mirror_reflection(M, mtab, 0.0, 0.0, job.fsx, job.fsy, rr, ri);
        t *= rr * rr + ri * ri;
      }
      acc += job.weight * t;
    }
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) clear_out[o] = red[0];
}

// The pupil table of a plan (every engine builds it the same way).
cudaError_t launch_pupil_table(const LithoAbbePlan& p, const void* blob, float2* table, cudaStream_t s) {
  const char* b = static_cast<const char*>(blob);
  const LithoMirror* mirrors = p.mirrored ? reinterpret_cast<const LithoMirror*>(b + p.off_mirrors) : nullptr;
  k_pupil_table<<<p.n_tab, 128, 0, s>>>(reinterpret_cast<const LithoJob*>(b + p.off_jobs),
                                         reinterpret_cast<const int32_t*>(b + p.off_slots),
                                         reinterpret_cast<const LithoPupil*>(b + p.off_pupils), mirrors, p.n_tab,
                                         p.n, p.pixel_size, p.h, p.ncomp_max, table);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// 3. coarse accumulation, L = 32 (h <= 7). A block takes one work item (a run
//    of one output's jobs, all on the same clip); the clip's mask band box is
//    staged once in shared memory. A warp takes the item's coherent transforms
//    two at a time: in pass 1 (inverse over ky) lanes 0-15 are the spectral
//    columns of the first transform and lanes 16-31 those of the second, so
//    no lane idles on an empty column; in pass 2 (inverse over kx) lane = row
//    v, once per transform, and J(u, v) += w |e|^2 stays in the lane's 32
//    registers. Both transforms are pruned FFTs (only d in [-h, h] non-zero).
//    The next pair's pupil-table blocks are fetched with cp.async while the
//    current pair's pass 2 runs.
// ---------------------------------------------------------------------------
constexpr int kCoarseWarps = 4;
constexpr int kCoarseHMax32 = 7;  // 4h + 1 <= 32
constexpr int kC32TLd = 33;

struct C32Smem {
  int side, npts, npad, Bm;
  size_t off_warp, per_warp, total;
};

__host__ __device__ inline C32Smem c32_smem(int h, int bm) {
  C32Smem g{};
  g.side = 2 * h + 1;
  g.npts = g.side * g.side;
  g.npad = (g.npts + 1) & ~1;
  g.Bm = 2 * bm + 1;
  g.off_warp = (((size_t)g.Bm * g.Bm * 8) + 15) & ~(size_t)15;
  g.per_warp = (size_t)2 * g.npad * 8 + (size_t)2 * g.side * kC32TLd * 8;
  g.total = g.off_warp + kCoarseWarps * g.per_warp;
  const size_t red = (size_t)kCoarseWarps * 1024 * 4;  // the final reduction reuses the buffer
  if (g.total < red) g.total = red;
  return g;
}

// H: the pupil half-width as a compile-time constant (instantiated for 0..7),
// so the band tests and the pruned FFTs' zero masks fold away.
template <int H>
__global__ void __launch_bounds__(kCoarseWarps * 32, 4)
k_coarse32(const LithoItem* __restrict__ items, const LithoJob* __restrict__ jobs,
           const float2* __restrict__ table, int ncomp_max, const float2* __restrict__ Mb,
           int bm, float* __restrict__ partial) {
  constexpr int h = H;
  extern __shared__ __align__(16) unsigned char c32_raw[];
  const C32Smem g = c32_smem(h, bm);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int side = g.side, npts = g.npts, npad = g.npad, Bm = g.Bm;
  float2* msk = reinterpret_cast<float2*>(c32_raw);
  float2* TAB = reinterpret_cast<float2*>(c32_raw + g.off_warp + warp * g.per_warp);   // [2][npad]
  float2* T = TAB + 2 * npad;                                                          // [2][side][kC32TLd]
  const LithoItem it = items[blockIdx.x];
  const int clip = jobs[it.job_begin].clip, ncomp = jobs[it.job_begin].ncomp;
  {
    const float2* src = Mb + (size_t)clip * Bm * Bm;
    for (int i = threadIdx.x; i < Bm * Bm; i += blockDim.x) msk[i] = src[i];
  }
  const int n_t = (it.job_end - it.job_begin) * ncomp;
  const int n_pairs = (n_t + 1) >> 1;
  const int half = lane >> 4, col = lane & 15;
  // This lane's transform t = 2 pp + half of a pair: its job's centre, weight
  // and pupil-table offset (toff < 0: past the end). Loaded one pair ahead so
  // the global loads overlap the current pair's transforms.
  struct Rec {
    int cx, cy, toff;
    float w;
  };
  auto load_rec = [&](int pp) {
    Rec r{0, 0, -1, 0.f};
    const int t = 2 * pp + half;
    if (pp < n_pairs && t < n_t) {
      const int tj = div_ncomp(t, ncomp), c = t - tj * ncomp;
      const LithoJob* jb = jobs + it.job_begin + tj;
      r.cx = __ldg(&jb->cx);
      r.cy = __ldg(&jb->cy);
      r.w = (float)__ldg(&jb->weight);
      r.toff = (__ldg(&jb->tab) * ncomp_max + c) * npts;
    }
    return r;
  };
  // the pair's two pupil-table blocks into TAB (every lane copies part of both)
  auto fetch = [&](const Rec& r) {
    const int off[2] = {__shfl_sync(0xffffffffu, r.toff, 0), __shfl_sync(0xffffffffu, r.toff, 16)};
#pragma unroll
    for (int hf = 0; hf < 2; ++hf)
      if (off[hf] >= 0)
        for (int e = lane; e < npts; e += 32) cp_async8(TAB + hf * npad + e, table + off[hf] + e);
    cp_async_commit();
  };
  Rec cur = load_rec(warp);
  if (warp < n_pairs) fetch(cur);
  __syncthreads();  // mask box staged

  float J[32];
#pragma unroll
  for (int u = 0; u < 32; ++u) J[u] = 0.f;
  constexpr uint64_t kNZ = band_mask32(H);
  for (int pp = warp; pp < n_pairs; pp += kCoarseWarps) {
    const Rec nxt = load_rec(pp + kCoarseWarps);
    cp_async_wait_all();
    __syncwarp();
    {
      float2 v[32];
#pragma unroll
      for (int i = 0; i < 32; ++i) v[i] = make_float2(0.f, 0.f);
      if (cur.toff >= 0 && col < side) {
        const int mx = cur.cx + (col - h) + bm;
        // sqrt|w| rides in the field, so pass 2 accumulates |e|^2 without a multiply
        const float sw = sqrtf(fabsf(cur.w));
        if (mx >= 0 && mx < Bm) {
          const float2* tp = TAB + half * npad + col;
#pragma unroll
          for (int d = -kCoarseHMax32; d <= kCoarseHMax32; ++d) {
            const int my = cur.cy + d + bm;
            if (d >= -h && d <= h && my >= 0 && my < Bm)
              v[d & 31] = cmul(__fmul2_rn(tp[(d + h) * side], make_float2(sw, sw)), msk[my * Bm + mx]);
          }
        }
      }
      fft_reg_sparse<32, +1, kNZ>(v);  // over ky: T(kx = col - h, v)
      if (col < side) {
        float2* tr = T + (half * side + col) * kC32TLd;
#pragma unroll
        for (int i = 0; i < 32; ++i) tr[i] = v[i];
      }
    }
    __syncwarp();
    if (pp + kCoarseWarps < n_pairs) fetch(nxt);  // TAB is free again
#pragma unroll
    for (int hh = 0; hh < 2; ++hh) {
      if (2 * pp + hh >= n_t) break;
      const float w = __shfl_sync(0xffffffffu, cur.w, 16 * hh);
      float2 r[32];
#pragma unroll
      for (int i = 0; i < 32; ++i) r[i] = make_float2(0.f, 0.f);
      const float2* tc = T + (hh * side) * kC32TLd + lane;
#pragma unroll
      for (int d = -kCoarseHMax32; d <= kCoarseHMax32; ++d)
        if (d >= -h && d <= h) r[d & 31] = tc[(d + h) * kC32TLd];
      fft_reg_sparse<32, +1, kNZ>(r);  // over kx: sqrt|w| e(u, v = lane)
      if (w >= 0.f) {  // warp-uniform: one transform per warp here
#pragma unroll
        for (int u = 0; u < 32; ++u) J[u] = fmaf(r[u].x, r[u].x, fmaf(r[u].y, r[u].y, J[u]));
      } else {
#pragma unroll
        for (int u = 0; u < 32; ++u) J[u] = fmaf(-r[u].x, r[u].x, fmaf(-r[u].y, r[u].y, J[u]));
      }
    }
    __syncwarp();
    cur = nxt;
  }

  // Fixed-order reduction of the warps' J into this block's partial.
  __syncthreads();
  float* js = reinterpret_cast<float*>(c32_raw);  // [warp][v][u]
#pragma unroll
  for (int u = 0; u < 32; ++u) js[warp * 1024 + lane * 32 + u] = J[u];
  __syncthreads();
  float* dst = partial + (size_t)blockIdx.x * 1024;
  for (int idx = threadIdx.x; idx < 1024; idx += blockDim.x) {
    float s = 0.f;
#pragma unroll
    for (int wp = 0; wp < kCoarseWarps; ++wp) s += js[wp * 1024 + idx];
    dst[idx] = s;  // idx = v * 32 + u  (row = y, column = x)
  }
}

template <int H>
static cudaError_t launch_coarse32_h(int n_items, size_t sm, cudaStream_t s, const LithoItem* items,
                                     const LithoJob* jobs, const float2* table, int ncomp_max, const float2* mb,
                                     int bm, float* partial) {
  cudaFuncSetAttribute(k_coarse32<H>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  k_coarse32<H><<<n_items, kCoarseWarps * 32, sm, s>>>(items, jobs, table, ncomp_max, mb, bm, partial);
  return cudaGetLastError();
}

static cudaError_t launch_coarse32(int h, int n_items, size_t sm, cudaStream_t s, const LithoItem* items,
                                   const LithoJob* jobs, const float2* table, int ncomp_max, const float2* mb,
                                   int bm, float* partial) {
  switch (h) {
    case 0: return launch_coarse32_h<0>(n_items, sm, s, items, jobs, table, ncomp_max, mb, bm, partial);
    case 1: return launch_coarse32_h<1>(n_items, sm, s, items, jobs, table, ncomp_max, mb, bm, partial);
    case 2: return launch_coarse32_h<2>(n_items, sm, s, items, jobs, table, ncomp_max, mb, bm, partial);
    case 3: return launch_coarse32_h<3>(n_items, sm, s, items, jobs, table, ncomp_max, mb, bm, partial);
    case 4: return launch_coarse32_h<4>(n_items, sm, s, items, jobs, table, ncomp_max, mb, bm, partial);
    case 5: return launch_coarse32_h<5>(n_items, sm, s, items, jobs, table, ncomp_max, mb, bm, partial);
    case 6: return launch_coarse32_h<6>(n_items, sm, s, items, jobs, table, ncomp_max, mb, bm, partial);
    case 7: return launch_coarse32_h<7>(n_items, sm, s, items, jobs, table, ncomp_max, mb, bm, partial);
    default: return cudaErrorInvalidValue;
  }
}

// ---------------------------------------------------------------------------
// 3b. coarse accumulation, L = 64 (h <= 15): one warp per coherent system.
//    A 64-point transform of a sequence supported on [-15, 15] is two 32-point
//    FFTs: X(2v') = FFT32[g](v'), X(2v'+1) = FFT32[g(d) w64^d](v'), with
//    w64 = exp(2 pi i / 64). Pass 1 (over ky): lane = column kx, results to a
//    per-warp T[kx][v]; pass 2 (over kx): lane owns rows v and v + 32, and
//    J(v, u) += w |e|^2 lives in a per-warp shared-memory tile.
// ---------------------------------------------------------------------------
constexpr int kCoarse64Warps = 2;
constexpr int kCoarseHMax64 = 15;  // 4h + 1 <= 64
constexpr int kT64Ld = 65;         // T row pitch (complex), J row pitch (float)

__device__ __forceinline__ void fft64_of_box(float2 (&a)[32], float2 (&b)[32]) {
  // a holds g(d) at position d & 31 for d in [-15, 15]; on return a = X(2v'),
  // b = X(2v'+1), v' = 0..31.
#pragma unroll
  for (int i = 0; i < 32; ++i) {
    const int d = i < 16 ? i : i - 32;  // signed position
    b[i] = twiddle64<+1>(a[i], d & 63);
  }
  fft_reg<32, +1>(a);
  fft_reg<32, +1>(b);
}

__global__ void __launch_bounds__(kCoarse64Warps * 32)
k_coarse64(const LithoItem* __restrict__ items, const LithoJob* __restrict__ jobs,
           const float2* __restrict__ table, int h, int ncomp_max, const float2* __restrict__ Mb,
           int bm, float* __restrict__ partial) {
  extern __shared__ float2 smem64[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // per warp: T [31][kT64Ld] complex, then J [64][kT64Ld] float
  const int per_warp = 31 * kT64Ld + (64 * kT64Ld + 1) / 2;
  float2* T = smem64 + warp * per_warp;
  float* Jw = reinterpret_cast<float*>(T + 31 * kT64Ld);
  const LithoItem it = items[blockIdx.x];
  const int side = 2 * h + 1, npts = side * side, Bm = 2 * bm + 1;
  const int dx = lane - h;
  const bool col_live = lane < side;
  for (int i = lane; i < 64 * kT64Ld; i += 32) Jw[i] = 0.f;
  __syncwarp();

  for (int j = it.job_begin + warp; j < it.job_end; j += kCoarse64Warps) {
    const LithoJob job = jobs[j];
    const float w = (float)job.weight;
    const float sw = sqrtf(fabsf(w));  // carried in the field; the sign is applied in pass 2
    const float2* m = Mb + (size_t)job.clip * Bm * Bm;
    const int mx = job.cx + dx + bm;
    for (int c = 0; c < job.ncomp; ++c) {
      const float2* tp = table + ((size_t)job.tab * ncomp_max + c) * npts;
      float2 a[32], b[32];
#pragma unroll
      for (int i = 0; i < 32; ++i) a[i] = make_float2(0.f, 0.f);
      if (col_live && mx >= 0 && mx < Bm) {
#pragma unroll
        for (int d = -kCoarseHMax64; d <= kCoarseHMax64; ++d) {
          const int my = job.cy + d + bm;
          if (d >= -h && d <= h && my >= 0 && my < Bm)
            a[d & 31] = cmul(__fmul2_rn(__ldg(tp + (d + h) * side + (dx + h)), make_float2(sw, sw)),
                             __ldg(m + (size_t)my * Bm + mx));
        }
      }
      fft64_of_box(a, b);  // column kx = dx: T(kx, 2v') = a[v'], T(kx, 2v'+1) = b[v']
      __syncwarp();
      if (col_live) {
#pragma unroll
        for (int i = 0; i < 32; ++i) {
          T[lane * kT64Ld + 2 * i] = a[i];
          T[lane * kT64Ld + 2 * i + 1] = b[i];
        }
      }
      __syncwarp();
#pragma unroll 1
      for (int half = 0; half < 2; ++half) {
        const int v = lane + 32 * half;
#pragma unroll
        for (int i = 0; i < 32; ++i) a[i] = make_float2(0.f, 0.f);
#pragma unroll
        for (int d = -kCoarseHMax64; d <= kCoarseHMax64; ++d)
          if (d >= -h && d <= h) a[d & 31] = T[(d + h) * kT64Ld + v];
        fft64_of_box(a, b);  // e(2u', v) = a[u'], e(2u'+1, v) = b[u']
        float* jr = Jw + v * kT64Ld;
        const float sg = w >= 0.f ? 1.f : -1.f;
#pragma unroll
        for (int i = 0; i < 32; ++i) {
          jr[2 * i] = fmaf(sg * a[i].x, a[i].x, fmaf(sg * a[i].y, a[i].y, jr[2 * i]));
          jr[2 * i + 1] = fmaf(sg * b[i].x, b[i].x, fmaf(sg * b[i].y, b[i].y, jr[2 * i + 1]));
        }
      }
    }
  }
  __syncthreads();
  // fixed-order reduction over the block's warps: partial[item][v * 64 + u]
  float* dst = partial + (size_t)blockIdx.x * 4096;
  for (int idx = threadIdx.x; idx < 4096; idx += blockDim.x) {
    const int v = idx >> 6, u = idx & 63;
    float s = 0.f;
#pragma unroll
    for (int wp = 0; wp < kCoarse64Warps; ++wp) {
      const float* jw = reinterpret_cast<const float*>(smem64 + wp * per_warp + 31 * kT64Ld);
      s += jw[v * kT64Ld + u];
    }
    dst[idx] = s;
  }
}

static size_t coarse64_smem() {
  const int per_warp = 31 * kT64Ld + (64 * kT64Ld + 1) / 2;
  return (size_t)kCoarse64Warps * per_warp * sizeof(float2);
}

// ---------------------------------------------------------------------------
// 4. per output: J = sum of its items' partials (in item order), then
//    B(gx, gy) = (1/L^2) sum_{u,v} J(v, u) exp(-2 pi i (gx u + gy v) / L).
//    Blocks of kReduceThreads per output (grid.y of them split its box rows);
//    L is a power of two.
// ---------------------------------------------------------------------------
constexpr int kReduceThreads = 256;

__global__ void __launch_bounds__(kReduceThreads)
k_coarse_reduce(const int32_t* __restrict__ out_items, const float* __restrict__ partial, int L, int h,
                float2* __restrict__ Bout) {
  extern __shared__ float sm_f[];
  const int o = blockIdx.x;
  const int LL = L * L, G = 4 * h + 1, g0 = 2 * h, msk = L - 1;
  float* J = sm_f;                                         // [v][u]
  float2* R = reinterpret_cast<float2*>(sm_f + LL);        // [u][gy]
  float2* tw = R + (size_t)L * G;                          // exp(-2 pi i t / L)
  for (int t = threadIdx.x; t < L; t += blockDim.x) {
    double sn, cs;
    sincospi(2.0 * t / (double)L, &sn, &cs);
    tw[t] = make_float2((float)cs, (float)-sn);
  }
  const int i0 = out_items[o], i1 = out_items[o + 1];
  for (int idx = threadIdx.x; idx < LL; idx += blockDim.x) {
    float s0 = 0.f, s1 = 0.f, s2 = 0.f, s3 = 0.f;
    int i = i0;
    for (; i + 3 < i1; i += 4) {
      s0 += partial[(size_t)i * LL + idx];
      s1 += partial[(size_t)(i + 1) * LL + idx];
      s2 += partial[(size_t)(i + 2) * LL + idx];
      s3 += partial[(size_t)(i + 3) * LL + idx];
    }
    for (; i < i1; ++i) s0 += partial[(size_t)i * LL + idx];
    J[idx] = (s0 + s1) + (s2 + s3);
  }
  __syncthreads();
  // this block's rows gy of the box: [r0, r1) (grid.y splits an output when
  // there are too few outputs to fill the GPU)
  const int per = (G + gridDim.y - 1) / gridDim.y;
  const int r0 = blockIdx.y * per, r1 = (r0 + per) < G ? (r0 + per) : G;
  const int nr = r1 - r0;
  for (int id = threadIdx.x; id < L * nr; id += blockDim.x) {
    const int u = id / nr, gyi = r0 + id % nr, gy = gyi - g0;
    float2 acc = make_float2(0.f, 0.f);
    for (int v = 0; v < L; ++v) acc = cadd(acc, cscale(tw[(gy * v) & msk], J[v * L + u]));
    R[u * G + gyi] = acc;
  }
  __syncthreads();
  const float inv = 1.0f / (float)LL;
  float2* B = Bout + (size_t)o * G * G;
  for (int id = threadIdx.x; id < nr * G; id += blockDim.x) {
    const int gyi = r0 + id / G, gx = id % G - g0;
    float2 acc = make_float2(0.f, 0.f);
    for (int u = 0; u < L; ++u) acc = cadd(acc, cmul(R[u * G + gyi], tw[(gx * u) & msk]));
    B[gyi * G + (gx + g0)] = cscale(acc, inv);
  }
}

// Blocks per output of k_coarse_reduce: split the box rows until there are
// about 8 blocks per SM (each block of a split output sums the output's
// partials again, in the same order, and forms its share of the box rows).
static unsigned reduce_split(int n_out, int G) {
  int s = 1;
  while (s < 8 && (long long)n_out * s < 8 * 148 && s * 2 <= G) s *= 2;
  return (unsigned)s;
}

// ---------------------------------------------------------------------------
// 5. synthesis: I(x, y) = Re C(y, 0) + 2 sum_{gx >= 1} Re[C(y, gx) w^(gx x)],
//    C(y, gx) = sum_gy B(gx, gy) w^(gy y), w = exp(2 pi i / N).
//    A block writes kSynthRows full rows; a thread owns kSynthCols columns
//    and reuses each twiddle for all the block's rows.
// ---------------------------------------------------------------------------
constexpr int kSynthRows = 8;
constexpr int kSynthCols = 4;
constexpr int kSynthThreads = 256;

__global__ void __launch_bounds__(kSynthThreads, 3)
k_synth(const float2* __restrict__ Bbox, int G, int n, const float2* __restrict__ tw_inv,
        const LithoNorm* __restrict__ norm, float* __restrict__ image, float* __restrict__ blockmax) {
  extern __shared__ float2 sm2[];
  const int gh = G / 2, gp = gh + 1;
  float2* tw = sm2;                       // n entries
  float2* C = sm2 + n;                    // [kSynthRows][gp]
  float2* B = C + kSynthRows * gp;        // [G][G]
  __shared__ float red[kSynthThreads / 32];
  const int o = blockIdx.y, y0 = blockIdx.x * kSynthRows;
  const bool pow2 = (n & (n - 1)) == 0;
  for (int j = threadIdx.x; j < n; j += blockDim.x) tw[j] = tw_inv[j];
  for (int j = threadIdx.x; j < G * G; j += blockDim.x) B[j] = Bbox[(size_t)o * G * G + j];
  __syncthreads();
  for (int id = threadIdx.x; id < kSynthRows * gp; id += blockDim.x) {
    const int r = id / gp, gx = id % gp, y = y0 + r;
    float2 acc = make_float2(0.f, 0.f);
    if (y < n) {
      for (int gy = -gh; gy <= gh; ++gy) {
        const int e = gy * y;
        const int t = pow2 ? (e & (n - 1)) : ((e % n) + n) % n;
        acc = cadd(acc, cmul(B[(gy + gh) * G + (gx + gh)], tw[t]));
      }
    }
    C[r * gp + gx] = acc;
  }
  __syncthreads();
  const LithoNorm nm = norm ? norm[o] : LithoNorm{0, 1.0f};
  const float sc = nm.mode == 0 ? nm.scale : 1.0f;
  const int rows = (n - y0) < kSynthRows ? (n - y0) : kSynthRows;
  float mx = 0.f;
  for (int xb = threadIdx.x; xb < n; xb += kSynthThreads * kSynthCols) {
    float acc[kSynthRows][kSynthCols];
#pragma unroll
    for (int r = 0; r < kSynthRows; ++r)
#pragma unroll
      for (int j = 0; j < kSynthCols; ++j) acc[r][j] = 0.f;
    for (int gx = 1; gx <= gh; ++gx) {
      float2 w[kSynthCols];
#pragma unroll
      for (int j = 0; j < kSynthCols; ++j) {
        const int x = xb + j * kSynthThreads;
        const int e = gx * x;
        w[j] = x < n ? tw[pow2 ? (e & (n - 1)) : (e % n)] : make_float2(0.f, 0.f);
      }
#pragma unroll
      for (int r = 0; r < kSynthRows; ++r) {
        const float2 c = C[r * gp + gx];
#pragma unroll
        for (int j = 0; j < kSynthCols; ++j) acc[r][j] = fmaf(c.x, w[j].x, fmaf(-c.y, w[j].y, acc[r][j]));
      }
    }
#pragma unroll
    for (int r = 0; r < kSynthRows; ++r) {
      if (r >= rows) break;
      const float c0 = C[r * gp].x;
      float* dst = image + ((size_t)o * n + y0 + r) * n;
#pragma unroll
      for (int j = 0; j < kSynthCols; ++j) {
        const int x = xb + j * kSynthThreads;
        if (x < n) {
          const float val = fmaf(2.f, acc[r][j], c0);
          mx = fmaxf(mx, val);
          dst[x] = val * sc;
        }
      }
    }
  }
  // block max of the raw intensity
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, off));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
  __syncthreads();
  if (threadIdx.x == 0) {
    float m = red[0];
    for (int i = 1; i < kSynthThreads / 32; ++i) m = fmaxf(m, red[i]);
    blockmax[(size_t)o * gridDim.x + blockIdx.x] = m;
  }
}

int synth_blocks_for(int n) { return (n + kSynthRows - 1) / kSynthRows; }

static int num_sms_cached();

// Real synthesis of n_fields Hermitian boxes of side G into n x n images.
// cbuf: max(synth_mma_bytes, synth_cols_bytes) of workspace for the tensor-core
// or pair synthesis (nullptr: the direct kernel).
cudaError_t launch_synth_real(const float2* box, int G, int n, int n_fields, const float2* tw, const LithoNorm* norm,
                              float* out, float* blockmax, cudaStream_t s, float2* cbuf, int* status) {
  const int gh = G / 2;
  if (!norm && cbuf && status && synth_mma_pick(n_fields, n, gh))
    return launch_synth_mma(box, gh, n, n_fields, tw, nullptr, out, nullptr, blockmax, s, nullptr, cbuf, status,
                            num_sms_cached());
  if (!norm && synth_pairs_ok(n, gh))
    return launch_synth_pairs(box, gh, n, n_fields, tw, nullptr, out, nullptr, blockmax, s, nullptr, cbuf);
  const size_t sm = (size_t)n * 8 + (size_t)kSynthRows * (gh + 1) * 8 + (size_t)G * G * 8;
  cudaFuncSetAttribute(k_synth, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  dim3 gs((n + kSynthRows - 1) / kSynthRows, n_fields);
  k_synth<<<gs, kSynthThreads, sm, s>>>(box, G, n, tw, norm, out, blockmax);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// 6. peak and peak normalisation
// ---------------------------------------------------------------------------
__global__ void k_normalise(const float* __restrict__ blockmax, int nblk, const LithoNorm* __restrict__ norm,
                            int n, float* __restrict__ image, float* __restrict__ peak, int apply_mode0) {
  __shared__ float s_peak;
  const int o = blockIdx.y;
  if (threadIdx.x < 32) {
    float m = 0.f;
    for (int i = threadIdx.x; i < nblk; i += 32) m = fmaxf(m, blockmax[(size_t)o * nblk + i]);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, off));
    if (threadIdx.x == 0) {
      s_peak = m;
      if (blockIdx.x == 0) peak[o] = m;
    }
  }
  __syncthreads();
  const LithoNorm nm = norm[o];
  float sc;
  if (nm.mode == 1) {
    const float pk = s_peak;
    sc = pk > 0.f ? nm.scale / pk : nm.scale;
  } else {
    if (!apply_mode0 || nm.scale == 1.0f) return;  // already applied by the producer
    sc = nm.scale;
  }
  const size_t NN = (size_t)n * n;
  float* img = image + (size_t)o * NN;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  if ((NN & 3) == 0 && (((uintptr_t)img) & 15) == 0) {
    float4* v4 = reinterpret_cast<float4*>(img);
    const size_t n4 = NN >> 2;
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    for (; i + stride < n4; i += 2 * stride) {
      float4 a = v4[i], b = v4[i + stride];
      a.x *= sc; a.y *= sc; a.z *= sc; a.w *= sc;
      b.x *= sc; b.y *= sc; b.z *= sc; b.w *= sc;
      v4[i] = a;
      v4[i + stride] = b;
    }
    for (; i < n4; i += stride) {
      float4 a = v4[i];
      a.x *= sc; a.y *= sc; a.z *= sc; a.w *= sc;
      v4[i] = a;
    }
  } else {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < NN; i += stride) img[i] *= sc;
  }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
static int synth_blocks(int n) { return (n + kSynthRows - 1) / kSynthRows; }

struct AbbeLayout {
  int64_t status, tw, u1, mb, table, partial, bbox, blockmax, cbuf, total;
};


static AbbeLayout abbe_layout(const LithoAbbePlan& p) {
  AbbeLayout l{};
  if (p.L > 64) {  // wide engine (wide.cu); its status word is also at offset 0
    l.total = wide_workspace_bytes(p);
    return l;
  }
  const int64_t Bm = 2 * p.bm + 1, side = 2 * p.h + 1, G = 4 * p.h + 1;
  int64_t off = 0;
  l.status = off;   off = align16(off + 16);
  l.tw = off;       off = align16(off + (int64_t)p.n * 8);
  l.u1 = off;       off = align16(off + (int64_t)p.n_clips * Bm * p.n * 8);
  l.mb = off;       off = align16(off + (int64_t)p.n_clips * Bm * Bm * 8);
  l.table = off;    off = align16(off + (int64_t)p.n_tab * p.ncomp_max * side * side * 8);
  l.partial = off;  off = align16(off + (int64_t)p.n_items * p.L * p.L * 4);
  l.bbox = off;     off = align16(off + (int64_t)p.n_out * G * G * 8);
  l.blockmax = off; off = align16(off + (int64_t)p.n_out * synth_blocks(p.n) * 4);
  l.cbuf = off;
  if (synth_mma_pick(p.n_out, p.n, 2 * p.h)) off = align16(off + synth_mma_bytes(p.n_out, p.n, 2 * p.h));
  else if (synth_pairs_ok(p.n, 2 * p.h)) off = align16(off + synth_cols_bytes(p.n_out, p.n, 2 * p.h));
  l.total = off;
  return l;
}

static int check_plan(const LithoAbbePlan* p) {
  if (!p) return LITHO_E_NULL;
  if (p->n < 2 || p->n > 8192 || p->n_clips < 1 || p->n_out < 1 || p->n_jobs < 0 || p->n_items < 0 ||
      p->n_pupils < 1 || p->h < 0 || p->bm < 0 || p->n_tab < 1 || p->n_tab > p->n_jobs)
    return LITHO_E_SIZE;
  if (p->ncomp_max != 1 && p->ncomp_max != 3) return LITHO_E_SIZE;
  if (p->L == 32 || p->L == 64) {
    if (4 * p->h + 1 > p->L || p->h > (p->L == 32 ? kCoarseHMax32 : kCoarseHMax64)) return LITHO_E_BAND;
  } else if (!wide_plan_ok(*p)) {
    return LITHO_E_UNSUPPORTED;
  }
  if (p->bm < p->h) return LITHO_E_BAND;
  // the coarse kernels address the pupil table with 32-bit element offsets
  if ((int64_t)p->n_tab * p->ncomp_max * (2 * p->h + 1) * (2 * p->h + 1) >= ((int64_t)1 << 31)) return LITHO_E_SIZE;
  if (!(p->pixel_size > 0.0)) return LITHO_E_SIZE;
  const int64_t offs[7] = {p->off_jobs, p->off_pupils, p->off_items, p->off_out_items, p->off_norm,
                           p->off_slots, p->mirrored ? p->off_mirrors : 0};
  for (int i = 0; i < 7; ++i)
    if (offs[i] < 0 || (offs[i] & 15)) return LITHO_E_ALIGN;
  if (p->mirrored != 0 && p->mirrored != 1) return LITHO_E_SIZE;
  return LITHO_OK;
}

static int num_sms_cached() {
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

extern "C" int litho_abbe_workspace(const LithoAbbePlan* plan, size_t* bytes) {
  const int st = check_plan(plan);
  if (st) return st;
  if (!bytes) return LITHO_E_NULL;
  *bytes = (size_t)abbe_layout(*plan).total;
  return LITHO_OK;
}

namespace litho {

// The pipeline, optionally bracketing each stage with events ev[0..7].
// table == nullptr: the pupil table is built into the workspace first.
// levels != nullptr: mask is a level map (uint8 per pixel indexing
// levels[clip][0 .. n_levels)), on the coarse engines only.
static int abbe_run(const LithoAbbePlan* plan, const void* blob, const void* table_in, const void* mask,
                    float* image, float* peak, void* ws, size_t ws_bytes, cudaStream_t s, cudaEvent_t* ev,
                    const float2* levels = nullptr, int n_levels = 0) {
  int st = check_plan(plan);
  if (st) return st;
  if (!blob || !mask || !image || !peak || !ws) return LITHO_E_NULL;
  if (((uintptr_t)ws & 15) || ((uintptr_t)blob & 15) || (!levels && ((uintptr_t)mask & 7)) ||
      ((uintptr_t)table_in & 7) || ((uintptr_t)levels & 7))
    return LITHO_E_ALIGN;
  const LithoAbbePlan& p = *plan;
  const AbbeLayout l = abbe_layout(p);
  if ((int64_t)ws_bytes < l.total) return LITHO_E_WORKSPACE;
  if (p.n_items == 0 || p.n_jobs == 0) return LITHO_E_SIZE;
  if (levels && (p.L > 64 || !row_band_levels_ok(p.n, p.bm))) return LITHO_E_UNSUPPORTED;

  if (p.L > 64) return abbe_wide_run(p, blob, table_in, mask, image, peak, ws, s, num_sms_cached(), ev);
  const char* b = static_cast<const char*>(blob);
  const LithoJob* jobs = reinterpret_cast<const LithoJob*>(b + p.off_jobs);
  const LithoItem* items = reinterpret_cast<const LithoItem*>(b + p.off_items);
  const int32_t* out_items = reinterpret_cast<const int32_t*>(b + p.off_out_items);
  const LithoNorm* norm = reinterpret_cast<const LithoNorm*>(b + p.off_norm);

  char* w = static_cast<char*>(ws);
  int* status = reinterpret_cast<int*>(w + l.status);
  float2* tw_own = reinterpret_cast<float2*>(w + l.tw);
  float2* u1 = reinterpret_cast<float2*>(w + l.u1);
  float2* mb = reinterpret_cast<float2*>(w + l.mb);
  float2* table = table_in ? (float2*)table_in : reinterpret_cast<float2*>(w + l.table);
  float* partial = reinterpret_cast<float*>(w + l.partial);
  float2* bbox = reinterpret_cast<float2*>(w + l.bbox);
  float* blockmax = reinterpret_cast<float*>(w + l.blockmax);

  const int sms = num_sms_cached();
  const int Bm = 2 * p.bm + 1, G = 4 * p.h + 1;
  cudaError_t e;
  auto mark = [&](int i) { if (ev) cudaEventRecord(ev[i], s); };

  mark(0);
  if ((e = cudaMemsetAsync(status, 0, sizeof(int), s)) != cudaSuccess) return (int)e;
  const float2* tw = twiddles_for(p.n, tw_own, s);
  if (!table_in)
    if ((e = launch_pupil_table(p, blob, table, s)) != cudaSuccess) return (int)e;
  mark(1);
  // mask band spectrum: rows then columns, 1/N^2 folded into the second pass
  e = levels ? launch_row_band_dft_levels(static_cast<const uint8_t*>(mask), levels, n_levels, p.n_clips * p.n, p.n,
                                          p.n, p.bm, u1, 1.0f, tw, sms, s)
             : launch_row_band_dft(mask, p.mask_complex != 0, p.n_clips * p.n, p.n, p.n, p.bm, u1, 1.0f, tw, sms, s,
                                   status);
  if (e != cudaSuccess) return (int)e;
  mark(2);
  e = launch_row_band_dft(u1, true, p.n_clips * Bm, Bm, p.n, p.bm, mb, 1.0f / ((float)p.n * (float)p.n), tw,
                          sms, s, status);
  if (e != cudaSuccess) return (int)e;
  mark(3);
  if (p.L == 32) {
    const size_t sm_coarse = c32_smem(p.h, p.bm).total;
    e = launch_coarse32(p.h, p.n_items, sm_coarse, s, items, jobs, table, p.ncomp_max, mb, p.bm, partial);
    if (e != cudaSuccess) return (int)e;
  } else {
    const size_t sm_coarse = coarse64_smem();
    cudaFuncSetAttribute(k_coarse64, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_coarse);
    k_coarse64<<<p.n_items, kCoarse64Warps * 32, sm_coarse, s>>>(items, jobs, table, p.h, p.ncomp_max, mb, p.bm,
                                                                  partial);
  }
  if ((e = cudaGetLastError()) != cudaSuccess) return (int)e;
  mark(4);
  const size_t sm_red = (size_t)p.L * p.L * 4 + (size_t)p.L * G * 8 + (size_t)p.L * 8;
  cudaFuncSetAttribute(k_coarse_reduce, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_red);
  k_coarse_reduce<<<dim3(p.n_out, reduce_split(p.n_out, G)), kReduceThreads, sm_red, s>>>(out_items, partial, p.L,
                                                                                          p.h, bbox);
  if ((e = cudaGetLastError()) != cudaSuccess) return (int)e;
  mark(5);
  if (synth_mma_pick(p.n_out, p.n, 2 * p.h)) {
    // peak pass (peak-normalised outputs), then the writing pass, on the tensor cores
    e = launch_synth_mma(bbox, 2 * p.h, p.n, p.n_out, tw, norm, image, peak, blockmax, s, ev ? ev[6] : nullptr,
                         w + l.cbuf, status, sms);
    if (e != cudaSuccess) return (int)e;
  } else if (synth_pairs_ok(p.n, 2 * p.h)) {
    e = launch_synth_pairs(bbox, 2 * p.h, p.n, p.n_out, tw, norm, image, peak, blockmax, s, ev ? ev[6] : nullptr,
                           reinterpret_cast<float2*>(w + l.cbuf));
    if (e != cudaSuccess) return (int)e;
  } else {
    const int gh = G / 2;
    const size_t sm_syn = (size_t)p.n * 8 + (size_t)kSynthRows * (gh + 1) * 8 + (size_t)G * G * 8;
    cudaFuncSetAttribute(k_synth, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_syn);
    dim3 gs(synth_blocks(p.n), p.n_out);
    k_synth<<<gs, kSynthThreads, sm_syn, s>>>(bbox, G, p.n, tw, norm, image, blockmax);
    if ((e = cudaGetLastError()) != cudaSuccess) return (int)e;
    mark(6);
    dim3 gn((unsigned)((((size_t)p.n * p.n + 255) / 256) < 512 ? (((size_t)p.n * p.n + 255) / 256) : 512),
            p.n_out);
    k_normalise<<<gn, 256, 0, s>>>(blockmax, synth_blocks(p.n), norm, p.n, image, peak, 0);
    if ((e = cudaGetLastError()) != cudaSuccess) return (int)e;
  }
  mark(7);
  return LITHO_OK;
}

}  // namespace litho

extern "C" int litho_abbe(const LithoAbbePlan* plan, const void* blob, const void* mask, float* image,
                          float* peak, void* ws, size_t ws_bytes, cudaStream_t s) {
  return abbe_run(plan, blob, nullptr, mask, image, peak, ws, ws_bytes, s, nullptr);
}

extern "C" int litho_abbe_tabled(const LithoAbbePlan* plan, const void* blob, const void* table, const void* mask,
                                 float* image, float* peak, void* ws, size_t ws_bytes, cudaStream_t s) {
  if (!table) return LITHO_E_NULL;
  return abbe_run(plan, blob, table, mask, image, peak, ws, ws_bytes, s, nullptr);
}

extern "C" int litho_abbe_levels(const LithoAbbePlan* plan, const void* blob, const void* table,
                                 const uint8_t* mask_idx, const void* levels, int n_levels, float* image, float* peak,
                                 void* ws, size_t ws_bytes, cudaStream_t s) {
  if (!table || !levels) return LITHO_E_NULL;
  if (n_levels < 1 || n_levels > 256) return LITHO_E_SIZE;
  return abbe_run(plan, blob, table, mask_idx, image, peak, ws, ws_bytes, s, nullptr,
                  static_cast<const float2*>(levels), n_levels);
}

extern "C" int litho_coarse_image(const LithoAbbePlan* plan, const void* blob, const void* table, const void* mb,
                                  void* bbox_out, void* ws, size_t ws_bytes, cudaStream_t s) {
  const int st = check_plan(plan);
  if (st) return st;
  if (!blob || !table || !mb || !bbox_out || !ws) return LITHO_E_NULL;
  const LithoAbbePlan& p = *plan;
  if (p.L > 64) {
    if ((int64_t)ws_bytes < wide_workspace_bytes(p)) return LITHO_E_WORKSPACE;
    return wide_coarse_box(p, blob, static_cast<const float2*>(table), static_cast<const float2*>(mb),
                           static_cast<float2*>(bbox_out), ws, s);
  }
  const AbbeLayout l = abbe_layout(p);
  if ((int64_t)ws_bytes < l.total) return LITHO_E_WORKSPACE;
  const char* b = static_cast<const char*>(blob);
  const LithoJob* jobs = reinterpret_cast<const LithoJob*>(b + p.off_jobs);
  const LithoItem* items = reinterpret_cast<const LithoItem*>(b + p.off_items);
  const int32_t* out_items = reinterpret_cast<const int32_t*>(b + p.off_out_items);
  float* partial = reinterpret_cast<float*>(static_cast<char*>(ws) + l.partial);
  const int G = 4 * p.h + 1;
  if (p.L == 32) {
    const size_t sm = c32_smem(p.h, p.bm).total;
    const cudaError_t e32 = launch_coarse32(p.h, p.n_items, sm, s, items, jobs, static_cast<const float2*>(table),
                                            p.ncomp_max, static_cast<const float2*>(mb), p.bm, partial);
    if (e32 != cudaSuccess) return (int)e32;
  } else {
    const size_t sm = coarse64_smem();
    cudaFuncSetAttribute(k_coarse64, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k_coarse64<<<p.n_items, kCoarse64Warps * 32, sm, s>>>(items, jobs, static_cast<const float2*>(table), p.h,
                                                          p.ncomp_max, static_cast<const float2*>(mb), p.bm, partial);
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return (int)e;
  const size_t sm_red = (size_t)p.L * p.L * 4 + (size_t)p.L * G * 8 + (size_t)p.L * 8;
  cudaFuncSetAttribute(k_coarse_reduce, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_red);
  k_coarse_reduce<<<dim3(p.n_out, reduce_split(p.n_out, G)), kReduceThreads, sm_red, s>>>(out_items, partial, p.L, p.h,
                                                                                 static_cast<float2*>(bbox_out));
  e = cudaGetLastError();
  return e == cudaSuccess ? LITHO_OK : (int)e;
}

extern "C" int litho_abbe_status(const LithoAbbePlan* plan, const void* ws, cudaStream_t s) {
  const int st = check_plan(plan);
  if (st) return st;
  if (!ws) return LITHO_E_NULL;
  int h = 0;
  cudaError_t e = cudaMemcpyAsync(&h, static_cast<const char*>(ws) + abbe_layout(*plan).status, sizeof(int),
                                  cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return (int)e;
  return h;
}

extern "C" int litho_abbe_clear(const LithoAbbePlan* plan, const void* blob, double* clear_out, cudaStream_t s) {
  const int st = check_plan(plan);
  if (st) return st;
  if (!blob || !clear_out) return LITHO_E_NULL;
  if (((uintptr_t)blob & 15) || ((uintptr_t)clear_out & 7)) return LITHO_E_ALIGN;
  const LithoAbbePlan& p = *plan;
  const char* b = static_cast<const char*>(blob);
  const LithoMirror* mirrors = p.mirrored ? reinterpret_cast<const LithoMirror*>(b + p.off_mirrors) : nullptr;
  k_abbe_clear<<<p.n_out, 128, 0, s>>>(reinterpret_cast<const LithoJob*>(b + p.off_jobs),
                                       reinterpret_cast<const LithoItem*>(b + p.off_items),
                                       reinterpret_cast<const int32_t*>(b + p.off_out_items),
                                       reinterpret_cast<const LithoPupil*>(b + p.off_pupils), mirrors, p.n,
                                       p.pixel_size, clear_out);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? LITHO_OK : (int)e;
}

extern "C" int litho_abbe_engine(const LithoAbbePlan* plan, int32_t* info, int n) {
  const int st = check_plan(plan);
  if (st) return st;
  if (!info || n < 1) return LITHO_E_NULL;
  const LithoAbbePlan& p = *plan;
  int32_t v[2];
  if (p.L > 64) {
    v[0] = 2;
    v[1] = 3;
  } else {
    v[0] = 1;
    v[1] = synth_mma_pick(p.n_out, p.n, 2 * p.h) ? 2 : synth_pairs_ok(p.n, 2 * p.h) ? 1 : 0;
  }
  for (int i = 0; i < n && i < 2; ++i) info[i] = v[i];
  return LITHO_OK;
}

extern "C" int litho_abbe_table_bytes(const LithoAbbePlan* plan, size_t* bytes) {
  const int st = check_plan(plan);
  if (st) return st;
  if (!bytes) return LITHO_E_NULL;
  const int64_t side = 2 * plan->h + 1;
  *bytes = (size_t)plan->n_tab * plan->ncomp_max * side * side * 8;
  return LITHO_OK;
}

extern "C" int litho_abbe_pupil_table(const LithoAbbePlan* plan, const void* blob, void* table, cudaStream_t s) {
  const int st = check_plan(plan);
  if (st) return st;
  if (!blob || !table) return LITHO_E_NULL;
  if (((uintptr_t)blob & 15) || ((uintptr_t)table & 7)) return LITHO_E_ALIGN;
  const cudaError_t e = launch_pupil_table(*plan, blob, static_cast<float2*>(table), s);
  return e == cudaSuccess ? LITHO_OK : (int)e;
}

extern "C" int litho_abbe_profile(const LithoAbbePlan* plan, const void* blob, const void* table,
                                  const void* mask, float* image,
                                  float* peak, void* ws, size_t ws_bytes, cudaStream_t s, int reps,
                                  float* stage_ms) {
  if (!stage_ms || reps < 1) return LITHO_E_SIZE;
  const int K = 8;
  cudaEvent_t ev[K];
  for (int i = 0; i < K; ++i)
    if (cudaEventCreate(&ev[i]) != cudaSuccess) return (int)cudaErrorUnknown;
  double acc[K - 1] = {0};
  int st = LITHO_OK;
  for (int r = 0; r < reps && st == LITHO_OK; ++r) {
    st = abbe_run(plan, blob, table, mask, image, peak, ws, ws_bytes, s, ev);
    if (st) break;
    cudaError_t e = cudaEventSynchronize(ev[K - 1]);
    if (e != cudaSuccess) { st = (int)e; break; }
    for (int i = 0; i < K - 1; ++i) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, ev[i], ev[i + 1]);
      acc[i] += ms;
    }
  }
  for (int i = 0; i < K; ++i) cudaEventDestroy(ev[i]);
  for (int i = 0; i < K - 1; ++i) stage_ms[i] = (float)(acc[i] / reps);
  return st;
}
