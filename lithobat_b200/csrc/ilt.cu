// Inverse lithography on the GPU: the SOCS adjoint and the relaxed-resist
// objective, as composable device stages.
//
// Reference: opc/ilt.py — socs_fields (:208-232), socs_gradient (:235-266),
// _blur (:274-289), _Objective.__call__ (:311-360), _mask_of (:368-378),
// _grad_theta (:381-389) and the Adam update of run_ilt (:582-591).
//
// The adjoint, with E_k = F^-1(phi_k F(m)) and sensitivity G = dJ/dI,
//     grad(x) = 2 Re sum_k lambda_k F^-1( conj(phi_k) F(G E_k) )(x),
// needs F(G E_k) only on the kernel band |f| <= h, where it is the circular
// convolution of E_k's band spectrum (|h'| <= h) with G's spectrum on
// |g| <= 2h. On a 64 x 64 grid that convolution is exact, so per kernel:
//     e_k = IFFT64(phi_k M),  g = IFFT64(G band),  Y_k = FFT64(e_k g) / 64^2,
//     A(f) += lambda_k conj(phi_k(f)) Y_k(f)     for |f| <= h,
// and grad(x) = sum_f H(f) exp(2 pi i f.x / N) with H(f) = A(f) + conj(A(-f)),
// one band-limited synthesis (csrc/abbe.cu k_synth). Scale: M = F(m) / N^2,
// G band = F(G) / N^2, as the band-spectrum stage produces them.
#include <algorithm>

#include "common.cuh"
#include "ilt_math.cuh"

namespace litho {

cudaError_t launch_row_band_dft(const void* in, bool cplx, int n_rows, int rows_per_clip, int n, int bm,
                                float2* out, float scale, const float2* tw_inv, int num_sms, cudaStream_t st,
                                int* status);
cudaError_t launch_synth_real(const float2* box, int G, int n, int n_fields, const float2* tw, const LithoNorm* norm,
                              float* out, float* blockmax, cudaStream_t s, float2* cbuf, int* status);
bool synth_mma_ok(int n, int g0);
int64_t synth_mma_bytes(int n_out, int n, int g0);
int64_t synth_cols_bytes(int n_out, int n, int g0);
bool synth_pairs_ok(int n, int g0);
int synth_pairs_blocks(int n);
bool synth_objective_ok(int n, int g0);
cudaError_t launch_synth_objective(const float2* box, int g0, int n, int n_out, const float2* tw, float* blockmax,
                                   float2* cbuf, const SynthObj& obj, cudaStream_t s);
bool synth_objective_band_ok(int n, int g0, int kb);
cudaError_t launch_synth_objective_band(const float2* box, int g0, int n, int n_out, const float2* tw,
                                        float* blockmax, float2* cbuf, const SynthObj& obj, cudaStream_t s);
bool wide_adjoint_ok(int h);
int64_t wide_adjoint_ws(int n_clips, int h);
int wide_socs_adjoint(const LithoAbbePlan& p, const void* blob, const float2* table, const float2* mask_box,
                      const float2* sens_box, float2* grad_box, void* ws, cudaStream_t s);
int64_t wide_synth_spec_bytes(int n_fields, int n);
cudaError_t wide_synth_real(const float2* box, int g0, int n, int n_fields, float* out, float2* spec,
                            const float2* twN, cudaStream_t s);
int synth_blocks_for(int n);

// ---------------------------------------------------------------------------
// g_L(u, v) = sum_{|g| <= 2h} Gb(g) w64^(g.(u, v)). Grid (clip, 64 / kGlRows):
// a block forms kGlRows rows v of one clip. Gb: (4h+1)^2 box [gy][gx].
// Output [clip][v][u] complex.
// ---------------------------------------------------------------------------
constexpr int kGlRows = 4;

__global__ void k_gl64(const float2* __restrict__ Gb, int h, float2* __restrict__ gl) {
  __shared__ float2 T[kGlRows * 61];   // [v][gx], gx index < 4h+1 <= 61
  __shared__ float2 tw[64];
  const int c = blockIdx.x, v0 = blockIdx.y * kGlRows, G = 4 * h + 1, g0 = 2 * h;
  for (int t = threadIdx.x; t < 64; t += blockDim.x) {
    double s, co;
    sincospi(2.0 * t / 64.0, &s, &co);
    tw[t] = make_float2((float)co, (float)s);
  }
  __syncthreads();
  const float2* B = Gb + (size_t)c * G * G;
  for (int id = threadIdx.x; id < kGlRows * G; id += blockDim.x) {
    const int r = id / G, gx = id % G, v = v0 + r;
    float2 acc = make_float2(0.f, 0.f);
    for (int gy = 0; gy < G; ++gy) acc = cadd(acc, cmul(__ldg(B + gy * G + gx), tw[((gy - g0) * v) & 63]));
    T[r * 61 + gx] = acc;
  }
  __syncthreads();
  float2* out = gl + (size_t)c * 4096 + (size_t)v0 * 64;
  for (int id = threadIdx.x; id < kGlRows * 64; id += blockDim.x) {
    const int r = id >> 6, u = id & 63;
    float2 acc = make_float2(0.f, 0.f);
    for (int gx = 0; gx < G; ++gx) acc = cadd(acc, cmul(T[r * 61 + gx], tw[((gx - g0) * u) & 63]));
    out[id] = acc;
  }
}

// ---------------------------------------------------------------------------
// Coarse adjoint, one pair of warps per (clip, kernel) job; h <= 15. The
// two warps of a pair split each job's work in half (the even and odd
// halves of the 64-point transforms in passes 1 and 3, the two halves of the
// rows in pass 2), so a job's serial latency halves; a block holds two pairs.
// ---------------------------------------------------------------------------
constexpr int kAdjPairs = 2;
constexpr int kAdjHMax = 15;
constexpr int kAdjLd = 65;
constexpr int kAdjXLd = 33;
// per pair: T [31][kAdjLd], Xa and Xb [31][kAdjXLd], Aw [31][32] (complex)
constexpr int kAdjPerPair = 31 * kAdjLd + 2 * 31 * kAdjXLd + 31 * 32;

// 64-point forward DFT outputs X(k), k in [-h, h], of a full sequence held as
// even (ev[i] = x(2i)) and odd (od[i] = x(2i+1)) halves:
//   X(k) = FFT32(ev)(k mod 32) + w64^(-k) FFT32(od)(k mod 32).
__device__ __forceinline__ float2 combine64(const float2 (&ev)[32], const float2 (&od)[32], int kk) {
  // kk compile-time in [-15, 15]
  return cadd(ev[kk & 31], twiddle64<-1>(od[kk & 31], kk & 63));
}

__device__ __forceinline__ void pair_sync(int pair) {
  asm volatile("bar.sync %0, 64;" ::"r"(1 + pair) : "memory");
}

__global__ void __launch_bounds__(kAdjPairs * 64)
k_coarse64_adjoint(const LithoItem* __restrict__ items, const LithoJob* __restrict__ jobs,
                   const float2* __restrict__ table, int h, const float2* __restrict__ Mb,
                   const float2* __restrict__ etab, const float2* __restrict__ gl, float2* __restrict__ partial) {
  extern __shared__ float2 adj_sm[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int pair = warp >> 1, role = warp & 1;
  const int side = 2 * h + 1, npts = side * side;
  float2* T = adj_sm + pair * kAdjPerPair;       // [kx or fx][v]
  float2* Xa = T + 31 * kAdjLd;                   // pass 3: forward of the even v, per column
  float2* Xb = Xa + 31 * kAdjXLd;                 // pass 3: forward of the odd v
  float2* Aw = Xb + 31 * kAdjXLd;                 // [fx][fy] accumulator
  const LithoItem it = items[blockIdx.x];
  const int dx = lane - h;
  const bool col_live = lane < side;
  for (int i = threadIdx.x & 63; i < 31 * 32; i += 64) Aw[i] = make_float2(0.f, 0.f);
  pair_sync(pair);
  const float inv = 1.0f / 4096.0f;
  for (int j = it.job_begin + pair; j < it.job_end; j += kAdjPairs) {
    const LithoJob job = jobs[j];
    const float lam = (float)job.weight;
    const float2* tp = table + (size_t)job.tab * npts;
    const float2* m = Mb + (size_t)job.clip * npts;
    const float2* g = gl + (size_t)job.clip * 4096;
    float2 a[32], b[32];
    // pass 1: columns kx = dx of E = phi M, inverse over ky; role 0 the even
    // outputs T(kx, 2v'), role 1 the odd ones T(kx, 2v'+1)
#pragma unroll
    for (int i = 0; i < 32; ++i) a[i] = make_float2(0.f, 0.f);
    if (col_live) {
#pragma unroll
      for (int d = -kAdjHMax; d <= kAdjHMax; ++d)
        if (d >= -h && d <= h) {
          const int p = (d + h) * side + (dx + h);
          a[d & 31] = etab ? __ldg(etab + (size_t)j * npts + p) : cmul(__ldg(tp + p), __ldg(m + p));
        }
    }
    if (role == 1) {
#pragma unroll
      for (int i = 0; i < 32; ++i) {
        const int d = i < 16 ? i : i - 32;
        a[i] = twiddle64<+1>(a[i], d & 63);
      }
    }
    fft_reg<32, +1>(a);
    if (col_live) {
#pragma unroll
      for (int i = 0; i < 32; ++i) T[lane * kAdjLd + 2 * i + role] = a[i];
    }
    pair_sync(pair);
    // pass 2: rows v = lane + 32 role: e(u, v) over kx, times g(u, v), then
    // the forward DFT over u restricted to fx in [-h, h]; in place in T[., v].
    {
      const int v = lane + 32 * role;
#pragma unroll
      for (int i = 0; i < 32; ++i) a[i] = make_float2(0.f, 0.f);
#pragma unroll
      for (int d = -kAdjHMax; d <= kAdjHMax; ++d)
        if (d >= -h && d <= h) a[d & 31] = T[(d + h) * kAdjLd + v];
#pragma unroll
      for (int i = 0; i < 32; ++i) {
        const int d = i < 16 ? i : i - 32;
        b[i] = twiddle64<+1>(a[i], d & 63);
      }
      fft_reg<32, +1>(a);   // e(2u', v)
      fft_reg<32, +1>(b);   // e(2u'+1, v)
      const float2* gr = g + (size_t)v * 64;
#pragma unroll
      for (int i = 0; i < 32; ++i) {
        a[i] = cmul(a[i], __ldg(gr + 2 * i));
        b[i] = cmul(b[i], __ldg(gr + 2 * i + 1));
      }
      fft_reg<32, -1>(a);
      fft_reg<32, -1>(b);
      pair_sync(pair);   // every read of this job's pass-1 columns is done
#pragma unroll
      for (int f = -kAdjHMax; f <= kAdjHMax; ++f)
        if (f >= -h && f <= h) T[(f + h) * kAdjLd + v] = combine64(a, b, f);
    }
    pair_sync(pair);
    // pass 3: lane = fx, forward over v restricted to fy in [-h, h]; role 0
    // transforms the even v, role 1 the odd v, then each role combines half
    // of the fy band
    if (col_live) {
      const float2* tr = T + lane * kAdjLd;
#pragma unroll
      for (int i = 0; i < 32; ++i) a[i] = tr[2 * i + role];
      fft_reg<32, -1>(a);
      float2* X = role ? Xb : Xa;
#pragma unroll
      for (int i = 0; i < 32; ++i) X[lane * kAdjXLd + i] = a[i];
    }
    pair_sync(pair);
    if (col_live) {
#pragma unroll
      for (int i = 0; i < 32; ++i) {
        a[i] = Xa[lane * kAdjXLd + i];
        b[i] = Xb[lane * kAdjXLd + i];
      }
      float2* arow = Aw + lane * 32;
#pragma unroll
      for (int f = -kAdjHMax; f <= kAdjHMax; ++f)
        if (f >= -h && f <= h && (f > 0) == (role == 1)) {
          const float2 y = cscale(combine64(a, b, f), inv);
          const float2 ph = __ldg(tp + (f + h) * side + lane);   // phi(fx = dx, fy = f)
          const float2 acc = arow[f + h];
          arow[f + h] = cadd(acc, cscale(cmulc(y, ph), lam));    // lambda conj(phi) Y
        }
    }
    pair_sync(pair);
  }
  __syncthreads();
  // fixed-order sum over the block's pairs -> partial[item][(fy+h) side + fx+h]
  float2* dst = partial + (size_t)blockIdx.x * npts;
  for (int id = threadIdx.x; id < npts; id += blockDim.x) {
    const int fy = id / side, fx = id % side;
    float2 s = make_float2(0.f, 0.f);
    for (int pp = 0; pp < kAdjPairs; ++pp)
      s = cadd(s, adj_sm[pp * kAdjPerPair + 31 * kAdjLd + 2 * 31 * kAdjXLd + fx * 32 + fy]);
    dst[id] = s;
  }
}

// Per clip: A = sum of its items' partials (item order); H(f) = A(f) + conj(A(-f)).
__global__ void k_adjoint_reduce(const int32_t* __restrict__ out_items, const float2* __restrict__ partial, int h,
                                 float2* __restrict__ Hbox) {
  const int c = blockIdx.x, side = 2 * h + 1, npts = side * side;
  const int i0 = out_items[c], i1 = out_items[c + 1];
  for (int id = threadIdx.x; id < npts; id += blockDim.x) {
    const int fy = id / side, fx = id % side;
    const int mid = (2 * h - fy) * side + (2 * h - fx);  // -f
    float2 s = make_float2(0.f, 0.f), t = make_float2(0.f, 0.f);
    for (int i = i0; i < i1; ++i) {
      s = cadd(s, partial[(size_t)i * npts + id]);
      t = cadd(t, partial[(size_t)i * npts + mid]);
    }
    Hbox[(size_t)c * npts + id] = cadd(s, cconj(t));
  }
}

// ---------------------------------------------------------------------------
// Complex band-limited synthesis: out(x, y) = sum_{|g| <= h} box(g) w^(g.(x, y)).
// ---------------------------------------------------------------------------
constexpr int kCsRows = 8, kCsCols = 2;

__global__ void __launch_bounds__(256)
k_synth_complex(const float2* __restrict__ box, int h, int n, const float2* __restrict__ tw_inv,
                float2* __restrict__ out) {
  extern __shared__ float2 cs_sm[];
  const int side = 2 * h + 1;
  float2* tw = cs_sm;
  float2* C = cs_sm + n;          // [kCsRows][side]
  const int f = blockIdx.y, y0 = blockIdx.x * kCsRows;
  const bool pow2 = (n & (n - 1)) == 0;
  for (int j = threadIdx.x; j < n; j += blockDim.x) tw[j] = tw_inv[j];
  __syncthreads();
  const float2* B = box + (size_t)f * side * side;
  for (int id = threadIdx.x; id < kCsRows * side; id += blockDim.x) {
    const int r = id / side, gx = id % side, y = y0 + r;
    float2 acc = make_float2(0.f, 0.f);
    if (y < n)
      for (int gy = -h; gy <= h; ++gy) {
        const int e = gy * y;
        acc = cadd(acc, cmul(B[(gy + h) * side + gx], tw[pow2 ? (e & (n - 1)) : ((e % n) + n) % n]));
      }
    C[id] = acc;
  }
  __syncthreads();
  for (int xb = threadIdx.x; xb < n; xb += blockDim.x * kCsCols) {
    float2 acc[kCsRows][kCsCols];
#pragma unroll
    for (int r = 0; r < kCsRows; ++r)
#pragma unroll
      for (int j = 0; j < kCsCols; ++j) acc[r][j] = make_float2(0.f, 0.f);
    for (int gx = -h; gx <= h; ++gx) {
      float2 w[kCsCols];
#pragma unroll
      for (int j = 0; j < kCsCols; ++j) {
        const int x = xb + j * blockDim.x, e = gx * x;
        w[j] = x < n ? tw[pow2 ? (e & (n - 1)) : ((e % n) + n) % n] : make_float2(0.f, 0.f);
      }
#pragma unroll
      for (int r = 0; r < kCsRows; ++r) {
        const float2 c = C[r * side + gx + h];
#pragma unroll
        for (int j = 0; j < kCsCols; ++j) acc[r][j] = cadd(acc[r][j], cmul(c, w[j]));
      }
    }
#pragma unroll
    for (int r = 0; r < kCsRows; ++r) {
      const int y = y0 + r;
      if (y >= n) break;
#pragma unroll
      for (int j = 0; j < kCsCols; ++j) {
        const int x = xb + j * blockDim.x;
        if (x < n) out[((size_t)f * n + y) * n + x] = acc[r][j];
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Elementwise stages (n_fields x N x N, row-major).
// ---------------------------------------------------------------------------
// Relaxed resist objective (opc/ilt.py:313-336), after the optional blur of
// the image: fld = scale * img; signed = sign (fld - level);
// z = sigmoid(a signed); resid = z - target; dfield = sign (2/npix) resid a z (1 - z).
// TOTALS: the last block of each field to finish (counted in counters[field],
// which it resets) also sums that field's partials in block order into
// cost_out = sum / npix and perr_out.
template <bool TOTALS>
__global__ void k_ilt_objective(const float* __restrict__ img, const float* __restrict__ target, long long npix,
                                float scale, float level, float sign, float a, float inv_npix2,
                                float* __restrict__ dfield, float* __restrict__ signed_out,
                                double* __restrict__ cost_part, unsigned int* __restrict__ perr_part,
                                unsigned int* __restrict__ counters, double* __restrict__ cost_out,
                                long long* __restrict__ perr_out) {
  __shared__ double sc[32];
  __shared__ unsigned int sp[32];
  double cost = 0.0;
  unsigned int perr = 0;
  const long long base = (long long)blockIdx.y * npix;
  auto one = [&](long long i) -> void {
    const float fld = img[i] * scale;
    const float s = sign * (fld - level);
    const float z = objective_sigmoid(a * s);
    const float t = target[i];
    const float r = z - t;
    cost += (double)r * (double)r;
    dfield[i] = (sign * inv_npix2 * a) * r * (z * (1.0f - z));
    if (signed_out) signed_out[i] = s;
    perr += ((s > 0.f) != (t > 0.5f)) ? 1u : 0u;
  };
  const long long stride = (long long)gridDim.x * blockDim.x;
  if ((npix & 3) == 0 && ((base & 3) == 0) && (((uintptr_t)img | (uintptr_t)target | (uintptr_t)dfield) & 15) == 0 &&
      (!signed_out || ((uintptr_t)signed_out & 15) == 0)) {
    // four pixels per thread per iteration with 16-byte loads and stores
    const long long n4 = npix >> 2;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n4; k += stride) {
      const long long i = base + 4 * k;
      const float4 iv = *reinterpret_cast<const float4*>(img + i);
      const float4 tv = *reinterpret_cast<const float4*>(target + i);
      const float ii[4] = {iv.x, iv.y, iv.z, iv.w}, tt[4] = {tv.x, tv.y, tv.z, tv.w};
      float d[4], sg[4];
      float c4 = 0.f;
#pragma unroll
      for (int q = 0; q < 4; ++q)
        d[q] = ilt_objective_pixel(ii[q], tt[q], scale, level, sign, a, inv_npix2, c4, perr, &sg[q]);
      cost += (double)c4;
      *reinterpret_cast<float4*>(dfield + i) = make_float4(d[0], d[1], d[2], d[3]);
      if (signed_out) *reinterpret_cast<float4*>(signed_out + i) = make_float4(sg[0], sg[1], sg[2], sg[3]);
    }
  } else {
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < npix; k += stride) one(base + k);
  }
  for (int o = 16; o > 0; o >>= 1) {
    cost += __shfl_xor_sync(0xffffffffu, cost, o);
    perr += __shfl_xor_sync(0xffffffffu, perr, o);
  }
  if ((threadIdx.x & 31) == 0) {
    sc[threadIdx.x >> 5] = cost;
    sp[threadIdx.x >> 5] = perr;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double c = 0.0;
    unsigned int p = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      c += sc[w];
      p += sp[w];
    }
    cost_part[(size_t)blockIdx.y * gridDim.x + blockIdx.x] = c;
    perr_part[(size_t)blockIdx.y * gridDim.x + blockIdx.x] = p;
  }
  if (TOTALS) {
    __shared__ bool last;
    if (threadIdx.x == 0) {
      __threadfence();  // this block's partials are visible before it is counted
      last = atomicAdd(&counters[blockIdx.y], 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
      __threadfence();
      const double* cp = cost_part + (size_t)blockIdx.y * gridDim.x;
      const unsigned int* pq = perr_part + (size_t)blockIdx.y * gridDim.x;
      double c = 0.0;
      long long p = 0;
      for (unsigned int b = 0; b < gridDim.x; ++b) {
        c += __ldcg(cp + b);
        p += __ldcg(pq + b);
      }
      cost_out[blockIdx.y] = c / (double)npix;
      perr_out[blockIdx.y] = p;
      counters[blockIdx.y] = 0u;
    }
  }
}

// One ILT update per pixel (opc/ilt.py:381-389, 587-591, 368-378 without
// smoothing): m = sigmoid(beta theta), q = g beta m (1 - m), Adam on theta,
// mask = sigmoid(beta_next theta). Four pixels per thread per iteration.
__device__ __forceinline__ void ilt_update_body(const float* __restrict__ g, long long total, float beta,
                                                float beta_next, float step, float b1, float b2, float eps, float c1,
                                                float c2, float* __restrict__ theta, float* __restrict__ m1,
                                                float* __restrict__ m2, float* __restrict__ mask);

__global__ void k_ilt_update(const float* __restrict__ g, long long total, float beta, float beta_next, float step,
                             float b1, float b2, float eps, float c1, float c2, float* __restrict__ theta,
                             float* __restrict__ m1, float* __restrict__ m2, float* __restrict__ mask) {
  ilt_update_body(g, total, beta, beta_next, step, b1, b2, eps, c1, c2, theta, m1, m2, mask);
}

// The schedule one step on: beta = beta_next, it + 1, beta_next = beta x
// growth, Adam's bias corrections 1 - b^it (FP64, rounded to FP32).
__device__ __forceinline__ LithoIltSched sched_next(LithoIltSched v, double b1, double b2) {
  v.beta = v.beta_next;
  v.it += 1;
  v.beta_next = v.beta * v.growth;
  v.c1 = (float)(1.0 - pow(b1, (double)v.it));
  v.c2 = (float)(1.0 - pow(b2, (double)v.it));
  return v;
}

// litho_ilt_update_sched in one launch: every block takes the advanced
// schedule from the previous one, runs the update, and the last block to
// finish (counted in sc->pad, which it resets) stores the advanced schedule
// for the next step. Every block read the schedule before it was counted,
// so the store cannot overtake a read.
__global__ void k_ilt_update_sf(const float* __restrict__ g, long long total, LithoIltSched* __restrict__ sc,
                                float step, float b1, float b2, float eps, float* __restrict__ theta,
                                float* __restrict__ m1, float* __restrict__ m2, float* __restrict__ mask) {
  __shared__ LithoIltSched s_v;
  if (threadIdx.x == 0) s_v = sched_next(*sc, (double)b1, (double)b2);
  __syncthreads();
  ilt_update_body(g, total, (float)s_v.beta, (float)s_v.beta_next, step, b1, b2, eps, s_v.c1, s_v.c2, theta, m1, m2,
                  mask);
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned int done = atomicAdd(reinterpret_cast<unsigned int*>(&sc->pad), 1u);
    if (done == gridDim.x - 1) {
      LithoIltSched v = s_v;
      v.pad = 0;
      *sc = v;
    }
  }
}

__device__ __forceinline__ void ilt_update_body(const float* __restrict__ g, long long total, float beta,
                                                float beta_next, float step, float b1, float b2, float eps, float c1,
                                                float c2, float* __restrict__ theta, float* __restrict__ m1,
                                                float* __restrict__ m2, float* __restrict__ mask) {
  const long long n4 = total >> 2, stride = (long long)gridDim.x * blockDim.x;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n4; k += stride) {
    const long long i = 4 * k;
    const float4 gv = *reinterpret_cast<const float4*>(g + i);
    const float4 tv = *reinterpret_cast<const float4*>(theta + i);
    const float4 av = *reinterpret_cast<const float4*>(m1 + i);
    const float4 vv = *reinterpret_cast<const float4*>(m2 + i);
    float gg[4] = {gv.x, gv.y, gv.z, gv.w}, th[4] = {tv.x, tv.y, tv.z, tv.w};
    float a1[4] = {av.x, av.y, av.z, av.w}, a2[4] = {vv.x, vv.y, vv.z, vv.w}, mk[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const float m = sigmoid_clipped(beta * th[q]);
      const float gi = gg[q] * (beta * m * (1.f - m));
      a1[q] = b1 * a1[q] + (1.f - b1) * gi;
      a2[q] = b2 * a2[q] + (1.f - b2) * gi * gi;
      th[q] -= step * (a1[q] / c1) / (sqrtf(a2[q] / c2) + eps);
      mk[q] = sigmoid_clipped(beta_next * th[q]);
    }
    *reinterpret_cast<float4*>(theta + i) = make_float4(th[0], th[1], th[2], th[3]);
    *reinterpret_cast<float4*>(m1 + i) = make_float4(a1[0], a1[1], a1[2], a1[3]);
    *reinterpret_cast<float4*>(m2 + i) = make_float4(a2[0], a2[1], a2[2], a2[3]);
    *reinterpret_cast<float4*>(mask + i) = make_float4(mk[0], mk[1], mk[2], mk[3]);
  }
}

// TV and discreteness penalties (opc/ilt.py:339-357) on the mask, periodic
// neighbours, added to grad; their costs to cost_part (per block).
__global__ void k_ilt_penalties(const float* __restrict__ mask, int n_fields, int n, float w_tv, float w_disc,
                                float inv_npix, float* __restrict__ grad, double* __restrict__ cost_part) {
  __shared__ double sc[32];
  double cost = 0.0;
  const long long npix = (long long)n * n;
  const long long f = blockIdx.y;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < npix;
       k += (long long)gridDim.x * blockDim.x) {
    const long long i = f * npix + k;
    const int rem = (int)k, y = rem / n, x = rem % n;
    const float* m = mask + f * npix;
    const float c = m[rem];
    float g = 0.f;
    if (w_tv > 0.f) {
      const float up = m[((y + n - 1) % n) * n + x], dn = m[((y + 1) % n) * n + x];
      const float lf = m[y * n + (x + n - 1) % n], rt = m[y * n + (x + 1) % n];
      const float lap = up + dn + lf + rt - 4.f * c;
      const float gx = c - lf, gy = c - up;
      cost += (double)w_tv * ((double)gx * gx + (double)gy * gy) * inv_npix;
      g += w_tv * (-2.f * inv_npix) * lap;
    }
    if (w_disc > 0.f) {
      cost += (double)w_disc * (double)c * (1.0 - (double)c) * inv_npix;
      g += w_disc * (1.f - 2.f * c) * inv_npix;
    }
    grad[i] += g;
  }
  for (int o = 16; o > 0; o >>= 1) cost += __shfl_xor_sync(0xffffffffu, cost, o);
  if ((threadIdx.x & 31) == 0) sc[threadIdx.x >> 5] = cost;
  __syncthreads();
  if (threadIdx.x == 0) {
    double c = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) c += sc[w];
    cost_part[(size_t)blockIdx.y * gridDim.x + blockIdx.x] = c;
  }
}

// m = sigmoid(clip(beta * field, +-60))  (opc/ilt.py:368-378)
__global__ void k_ilt_mask(const float* __restrict__ field, long long total, float beta, float* __restrict__ mask) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x)
    mask[i] = sigmoid_clipped(beta * field[i]);
}

// q = grad_m * beta * m (1 - m)  (opc/ilt.py:381-389, before its blur)
__global__ void k_ilt_theta_grad(const float* __restrict__ grad_m, const float* __restrict__ mask, long long total,
                                 float beta, float* __restrict__ q) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const float m = mask[i];
    q[i] = grad_m[i] * (beta * m * (1.f - m));
  }
}

// Adam (opc/ilt.py:582-591) with bias corrections c1 = 1 - b1^t, c2 = 1 - b2^t.
__global__ void k_ilt_adam(const float* __restrict__ g, long long total, float step, float b1, float b2, float eps,
                           float c1, float c2, float* __restrict__ theta, float* __restrict__ m1,
                           float* __restrict__ m2) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float a = b1 * m1[i] + (1.f - b1) * gi;
    const float v = b2 * m2[i] + (1.f - b2) * gi * gi;
    m1[i] = a;
    m2[i] = v;
    theta[i] -= step * (a / c1) / (sqrtf(v / c2) + eps);
  }
}

// One axis of scipy.ndimage.gaussian_filter (mode 'reflect', i.e. the edge
// sample repeated: ... b a | a b ... ), weights w[0..2r] (host-built, FP64
// normalised). axis 0: along y (rows), axis 1: along x.
__device__ __forceinline__ int reflect_idx(int j, int n) {
  const int p = 2 * n;
  j %= p;
  if (j < 0) j += p;
  return j < n ? j : p - 1 - j;
}

__global__ void k_blur_axis(const float* __restrict__ in, float* __restrict__ out, int n_fields, int n,
                            const float* __restrict__ w, int r, int axis) {
  const long long total = (long long)n_fields * n * n;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const long long f = i / ((long long)n * n);
    const int rem = (int)(i - f * n * n), y = rem / n, x = rem % n;
    const float* src = in + f * (long long)n * n;
    float acc = 0.f;
    if (axis == 0) {
      for (int k = -r; k <= r; ++k) acc = fmaf(w[k + r], src[reflect_idx(y + k, n) * n + x], acc);
    } else {
      for (int k = -r; k <= r; ++k) acc = fmaf(w[k + r], src[y * n + reflect_idx(x + k, n)], acc);
    }
    out[i] = acc;
  }
}

static int grid_for(long long total, int threads, int cap) {
  long long b = (total + threads - 1) / threads;
  if (b > cap) b = cap;
  return (int)(b < 1 ? 1 : b);
}

static int sms_here() {
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

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
static int64_t band_ws(int n_fields, int n, int bm) {
  return align16(16) + align16((int64_t)n * 8) + align16((int64_t)n_fields * (2 * bm + 1) * n * 8);
}

extern "C" int litho_band_spectrum_workspace(int n_fields, int n, int bm, size_t* bytes) {
  if (!bytes) return LITHO_E_NULL;
  if (n_fields < 1 || n < 2 || bm < 0) return LITHO_E_SIZE;
  *bytes = (size_t)band_ws(n_fields, n, bm);
  return LITHO_OK;
}

extern "C" int litho_band_spectrum(const void* in, int is_complex, int n_fields, int n, int bm, float scale,
                                   void* box_out, void* ws, size_t ws_bytes, cudaStream_t s) {
  if (!in || !box_out || !ws) return LITHO_E_NULL;
  if (n_fields < 1 || n < 2 || bm < 0) return LITHO_E_SIZE;
  if ((int64_t)ws_bytes < band_ws(n_fields, n, bm)) return LITHO_E_WORKSPACE;
  if (((uintptr_t)ws & 15) || ((uintptr_t)in & 7)) return LITHO_E_ALIGN;
  char* w = static_cast<char*>(ws);
  int* status = reinterpret_cast<int*>(w);
  float2* tw_own = reinterpret_cast<float2*>(w + align16(16));
  float2* u1 = reinterpret_cast<float2*>(w + align16(16) + align16((int64_t)n * 8));
  const int Bm = 2 * bm + 1;
  cudaError_t e = cudaMemsetAsync(status, 0, sizeof(int), s);
  if (e != cudaSuccess) return (int)e;
  const float2* tw = twiddles_for(n, tw_own, s);
  e = launch_row_band_dft(in, is_complex != 0, n_fields * n, n, n, bm, u1, 1.0f, tw, sms_here(), s, status);
  if (e != cudaSuccess) return (int)e;
  e = launch_row_band_dft(u1, true, n_fields * Bm, Bm, n, bm, static_cast<float2*>(box_out), scale, tw, sms_here(), s,
                          status);
  return e == cudaSuccess ? LITHO_OK : (int)e;
}

// status word, twiddles, block maxima, then one region for the synthesis
// engine in use: the operand planes of the tensor-core synthesis or the column
// buffer of the pair synthesis (boxes up to half-width 31), or the spectrum of
// the synthesis of wider boxes
constexpr int64_t kColsAheadMin = 148 * 8;   // columns (fields x (h + 1)) for a separate column stage

static int64_t band_synth_region(int n_fields, int n) {
  int64_t r = align16(synth_cols_bytes(n_fields, n, 31));
  if (synth_mma_ok(n, 31)) r = std::max(r, align16(synth_mma_bytes(n_fields, n, 31)));
  return std::max(r, align16(wide_synth_spec_bytes(n_fields, n)));
}

static int64_t band_synth_ws(int n_fields, int n) {
  return align16(16) + align16((int64_t)n * 8) + align16((int64_t)n_fields * synth_blocks_for(n) * 4) +
         band_synth_region(n_fields, n);
}

extern "C" int litho_band_synthesis_workspace(int n_fields, int n, size_t* bytes) {
  if (!bytes) return LITHO_E_NULL;
  if (n_fields < 1 || n < 2) return LITHO_E_SIZE;
  *bytes = (size_t)band_synth_ws(n_fields, n);
  return LITHO_OK;
}

extern "C" int litho_band_synthesis(const void* box, int n_fields, int n, int h, int complex_out, void* out,
                                   void* ws, size_t ws_bytes, cudaStream_t s) {
  if (!box || !out || !ws) return LITHO_E_NULL;
  if (n_fields < 1 || n < 2 || h < 0) return LITHO_E_SIZE;
  size_t need = 0;
  litho_band_synthesis_workspace(n_fields, n, &need);
  if (ws_bytes < need) return LITHO_E_WORKSPACE;
  if ((uintptr_t)ws & 15) return LITHO_E_ALIGN;
  char* w0 = static_cast<char*>(ws);
  int* status = reinterpret_cast<int*>(w0);
  float2* tw_own = reinterpret_cast<float2*>(w0 + align16(16));
  float* blockmax = reinterpret_cast<float*>(w0 + align16(16) + align16((int64_t)n * 8));
  cudaError_t e = cudaMemsetAsync(status, 0, sizeof(int), s);
  if (e != cudaSuccess) return (int)e;
  const float2* tw = twiddles_for(n, tw_own, s);
  if (complex_out) {
    const int side = 2 * h + 1;
    const size_t sm = (size_t)n * 8 + (size_t)kCsRows * side * 8;
    cudaFuncSetAttribute(k_synth_complex, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    dim3 g((n + kCsRows - 1) / kCsRows, n_fields);
    k_synth_complex<<<g, 256, sm, s>>>(static_cast<const float2*>(box), h, n, tw, static_cast<float2*>(out));
    e = cudaGetLastError();
  } else {
    char* wb = w0 + align16(16) + align16((int64_t)n * 8) + align16((int64_t)n_fields * synth_blocks_for(n) * 4);
    if (!synth_pairs_ok(n, h) && h > 31 && n >= 32 && n <= 4096 && (n & (n - 1)) == 0 &&
        2 * h + 1 <= n) {
      // boxes too wide for the row synthesis: scatter and one inverse FFT per two fields
      e = wide_synth_real(static_cast<const float2*>(box), h, n, n_fields, static_cast<float*>(out),
                          reinterpret_cast<float2*>(wb), tw, s);
    } else {
      // column stage ahead (k_synth_cols) for batches with enough columns to
      // fill the GPU; smaller batches form it inside each synthesis block
      const bool cols_ahead = (int64_t)n_fields * (h + 1) >= kColsAheadMin;
      float2* cbuf = h <= 31 && cols_ahead ? reinterpret_cast<float2*>(wb) : nullptr;
      e = launch_synth_real(static_cast<const float2*>(box), 2 * h + 1, n, n_fields, tw, nullptr,
                            static_cast<float*>(out), blockmax, s, cbuf, status);
    }
  }
  return e == cudaSuccess ? LITHO_OK : (int)e;
}

static int64_t adj_ws(int n_clips, int n_items, int h) {
  const int npts = (2 * h + 1) * (2 * h + 1);
  return align16((int64_t)n_clips * 4096 * 8) + align16((int64_t)n_items * npts * 8);
}

extern "C" int litho_socs_adjoint_workspace(int n_clips, int n_items, int h, size_t* bytes) {
  if (!bytes) return LITHO_E_NULL;
  if (n_clips < 1 || n_items < 1 || h < 0) return LITHO_E_SIZE;
  if (h > kAdjHMax) {
    if (!wide_adjoint_ok(h)) return LITHO_E_SIZE;
    *bytes = (size_t)wide_adjoint_ws(n_clips, h);
    return LITHO_OK;
  }
  *bytes = (size_t)adj_ws(n_clips, n_items, h);
  return LITHO_OK;
}

// Band of the SOCS adjoint: see the file comment. The job list is the SOCS
// forward's (one job per clip x kernel: weight lambda_k, table slot k, clip c),
// grouped per clip by items/out_items as in LithoAbbePlan.
extern "C" int litho_socs_adjoint(const LithoAbbePlan* plan, const void* blob, const void* table, const void* mask_box,
                                  const void* field_box, const void* sens_box, void* grad_box_out, void* ws,
                                  size_t ws_bytes, cudaStream_t s) {
  if (!plan || !blob || !table || !sens_box || !grad_box_out || !ws) return LITHO_E_NULL;
  if (!mask_box && !field_box) return LITHO_E_NULL;
  const LithoAbbePlan& p = *plan;
  if (p.h < 0 || p.n_clips < 1 || p.n_items < 1 || p.bm != p.h) return LITHO_E_SIZE;
  if (p.h > kAdjHMax) {   // kernel bands wider than the 64-point grid: coarse grids of 128..1024
    if (!wide_adjoint_ok(p.h)) return LITHO_E_SIZE;
    if (!mask_box) return LITHO_E_NULL;
    if ((int64_t)ws_bytes < wide_adjoint_ws(p.n_clips, p.h)) return LITHO_E_WORKSPACE;
    return wide_socs_adjoint(p, blob, static_cast<const float2*>(table), static_cast<const float2*>(mask_box),
                             static_cast<const float2*>(sens_box), static_cast<float2*>(grad_box_out), ws, s);
  }
  if ((int64_t)ws_bytes < adj_ws(p.n_clips, p.n_items, p.h)) return LITHO_E_WORKSPACE;
  const char* b = static_cast<const char*>(blob);
  const LithoJob* jobs = reinterpret_cast<const LithoJob*>(b + p.off_jobs);
  const LithoItem* items = reinterpret_cast<const LithoItem*>(b + p.off_items);
  const int32_t* out_items = reinterpret_cast<const int32_t*>(b + p.off_out_items);
  float2* gl = static_cast<float2*>(ws);
  float2* part = reinterpret_cast<float2*>(static_cast<char*>(ws) + align16((int64_t)p.n_clips * 4096 * 8));
  k_gl64<<<dim3(p.n_clips, 64 / kGlRows), 256, 0, s>>>(static_cast<const float2*>(sens_box), p.h, gl);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return (int)e;
  const size_t sm = (size_t)kAdjPairs * kAdjPerPair * sizeof(float2);
  cudaFuncSetAttribute(k_coarse64_adjoint, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  k_coarse64_adjoint<<<p.n_items, kAdjPairs * 64, sm, s>>>(items, jobs, static_cast<const float2*>(table), p.h,
                                                            static_cast<const float2*>(mask_box),
                                                            static_cast<const float2*>(field_box), gl, part);
  if ((e = cudaGetLastError()) != cudaSuccess) return (int)e;
  k_adjoint_reduce<<<p.n_clips, 256, 0, s>>>(out_items, part, p.h, static_cast<float2*>(grad_box_out));
  e = cudaGetLastError();
  return e == cudaSuccess ? LITHO_OK : (int)e;
}

extern "C" int litho_ilt_objective(const float* img, const float* target, int n_fields, int n, float scale,
                                   float level, float sign, float steepness_a, float* dfield, float* signed_out,
                                   double* cost_part, unsigned int* perr_part, int n_part, cudaStream_t s) {
  if (!img || !target || !dfield || !cost_part || !perr_part) return LITHO_E_NULL;
  if (n_fields < 1 || n < 1 || n_part < 1) return LITHO_E_SIZE;
  const double npix = (double)n * n;
  dim3 g(n_part, n_fields);
  k_ilt_objective<false><<<g, 256, 0, s>>>(img, target, (long long)n * n, scale, level, sign, steepness_a,
                                           (float)(2.0 / npix), dfield, signed_out, cost_part, perr_part, nullptr,
                                           nullptr, nullptr);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? LITHO_OK : (int)e;
}

extern "C" int litho_ilt_objective_totals(const float* img, const float* target, int n_fields, int n, float scale,
                                          float level, float sign, float steepness_a, float* dfield,
                                          float* signed_out, double* cost_part, unsigned int* perr_part, int n_part,
                                          unsigned int* counters, double* cost_out, long long* perr_out,
                                          cudaStream_t s) {
  if (!img || !target || !dfield || !cost_part || !perr_part || !counters || !cost_out || !perr_out)
    return LITHO_E_NULL;
  if (n_fields < 1 || n < 1 || n_part < 1) return LITHO_E_SIZE;
  const double npix = (double)n * n;
  dim3 g(n_part, n_fields);
  k_ilt_objective<true><<<g, 256, 0, s>>>(img, target, (long long)n * n, scale, level, sign, steepness_a,
                                          (float)(2.0 / npix), dfield, signed_out, cost_part, perr_part, counters,
                                          cost_out, perr_out);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? LITHO_OK : (int)e;
}

// tw, block maxima, cost and pattern-error partials, then the column stage
static int64_t image_obj_ws(int n_fields, int n, int g0) {
  const int64_t nb = (int64_t)n_fields * synth_pairs_blocks(n);
  return align16((int64_t)n * 8) + align16(nb * 4) + align16(nb * 8) + align16(nb * 4) +
         align16(synth_cols_bytes(n_fields, n, g0));
}

extern "C" int litho_ilt_image_objective_workspace(int n_fields, int n, int g0, size_t* bytes) {
  if (!bytes) return LITHO_E_NULL;
  if (n_fields < 1 || n < 2 || g0 < 0) return LITHO_E_SIZE;
  if (!synth_objective_ok(n, g0)) return LITHO_E_UNSUPPORTED;
  *bytes = (size_t)image_obj_ws(n_fields, n, g0);
  return LITHO_OK;
}

extern "C" int litho_ilt_image_objective(const void* image_box, int n_fields, int n, int g0, const float* target,
                                         float scale, float level, float sign, float steepness_a, float* dfield,
                                         unsigned int* counters, double* cost_out, long long* perr_out, void* ws,
                                         size_t ws_bytes, cudaStream_t s) {
  if (!image_box || !target || !dfield || !counters || !cost_out || !perr_out || !ws) return LITHO_E_NULL;
  size_t need = 0;
  const int st = litho_ilt_image_objective_workspace(n_fields, n, g0, &need);
  if (st) return st;
  if (ws_bytes < need) return LITHO_E_WORKSPACE;
  if (((uintptr_t)ws | (uintptr_t)target) & 15) return LITHO_E_ALIGN;  // target rows are copied in 16-byte pieces
  const int64_t nb = (int64_t)n_fields * synth_pairs_blocks(n);
  char* w = static_cast<char*>(ws);
  float2* tw_own = reinterpret_cast<float2*>(w);
  w += align16((int64_t)n * 8);
  float* blockmax = reinterpret_cast<float*>(w);
  w += align16(nb * 4);
  double* cpart = reinterpret_cast<double*>(w);
  w += align16(nb * 8);
  unsigned int* ppart = reinterpret_cast<unsigned int*>(w);
  w += align16(nb * 4);
  float2* cbuf = reinterpret_cast<float2*>(w);
  const float2* tw = twiddles_for(n, tw_own, s);
  const double npix = (double)n * n;
  const SynthObj obj{target, scale, level, sign, steepness_a, (float)(2.0 / npix), dfield, cpart, ppart, counters,
                     cost_out, perr_out};
  const cudaError_t e = launch_synth_objective(static_cast<const float2*>(image_box), g0, n, n_fields, tw, blockmax,
                                               cbuf, obj, s);
  return e == cudaSuccess ? LITHO_OK : (int)e;
}

// status word, then image_obj_ws, then the band rows [field][2 kb + 1][n]
static int64_t image_obj_band_ws(int n_fields, int n, int g0, int kb) {
  return 16 + image_obj_ws(n_fields, n, g0) + align16((int64_t)n_fields * (2 * kb + 1) * n * 8);
}

extern "C" int litho_ilt_image_objective_band_workspace(int n_fields, int n, int g0, int band_half, size_t* bytes) {
  if (!bytes) return LITHO_E_NULL;
  if (n_fields < 1 || n < 2 || g0 < 0 || band_half < 0) return LITHO_E_SIZE;
  if (!synth_objective_band_ok(n, g0, band_half)) return LITHO_E_UNSUPPORTED;
  *bytes = (size_t)image_obj_band_ws(n_fields, n, g0, band_half);
  return LITHO_OK;
}

extern "C" int litho_ilt_image_objective_band(const void* image_box, int n_fields, int n, int g0, const float* target,
                                              float scale, float level, float sign, float steepness_a, int band_half,
                                              float band_scale, void* band_box_out, unsigned int* counters,
                                              double* cost_out, long long* perr_out, void* ws, size_t ws_bytes,
                                              cudaStream_t s) {
  if (!image_box || !target || !band_box_out || !counters || !cost_out || !perr_out || !ws) return LITHO_E_NULL;
  size_t need = 0;
  const int st = litho_ilt_image_objective_band_workspace(n_fields, n, g0, band_half, &need);
  if (st) return st;
  if (ws_bytes < need) return LITHO_E_WORKSPACE;
  if (((uintptr_t)ws | (uintptr_t)target) & 15) return LITHO_E_ALIGN;
  const int64_t nb = (int64_t)n_fields * synth_pairs_blocks(n);
  char* w = static_cast<char*>(ws);
  int* status = reinterpret_cast<int*>(w);
  w += 16;
  float2* tw_own = reinterpret_cast<float2*>(w);
  w += align16((int64_t)n * 8);
  float* blockmax = reinterpret_cast<float*>(w);
  w += align16(nb * 4);
  double* cpart = reinterpret_cast<double*>(w);
  w += align16(nb * 8);
  unsigned int* ppart = reinterpret_cast<unsigned int*>(w);
  w += align16(nb * 4);
  float2* cbuf = reinterpret_cast<float2*>(w);
  w += align16(synth_cols_bytes(n_fields, n, g0));
  float2* u1 = reinterpret_cast<float2*>(w);
  cudaError_t e = cudaMemsetAsync(status, 0, sizeof(int), s);
  if (e != cudaSuccess) return (int)e;
  const float2* tw = twiddles_for(n, tw_own, s);
  const double npix = (double)n * n;
  SynthObj obj{target, scale, level, sign, steepness_a, (float)(2.0 / npix), nullptr, cpart, ppart, counters,
               cost_out, perr_out};
  obj.band_rows = u1;
  obj.band_half = band_half;
  e = launch_synth_objective_band(static_cast<const float2*>(image_box), g0, n, n_fields, tw, blockmax, cbuf, obj, s);
  if (e != cudaSuccess) return (int)e;
  const int Bm = 2 * band_half + 1;
  e = launch_row_band_dft(u1, true, n_fields * Bm, Bm, n, band_half, static_cast<float2*>(band_box_out), band_scale,
                          tw, sms_here(), s, status);
  return e == cudaSuccess ? LITHO_OK : (int)e;
}

extern "C" int litho_ilt_penalties(const float* mask, int n_fields, int n, float w_tv, float w_disc, float* grad,
                                   double* cost_part, int n_part, cudaStream_t s) {
  if (!mask || !grad || !cost_part) return LITHO_E_NULL;
  if (n_fields < 1 || n < 1 || n_part < 1) return LITHO_E_SIZE;
  dim3 g(n_part, n_fields);
  k_ilt_penalties<<<g, 256, 0, s>>>(mask, n_fields, n, w_tv, w_disc, (float)(1.0 / ((double)n * n)), grad,
                                    cost_part);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? LITHO_OK : (int)e;
}

extern "C" int litho_ilt_mask(const float* field, long long count, float beta, float* mask, cudaStream_t s) {
  if (!field || !mask) return LITHO_E_NULL;
  if (count < 0) return LITHO_E_SIZE;
  k_ilt_mask<<<grid_for(count, 256, sms_here() * 16), 256, 0, s>>>(field, count, beta, mask);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? LITHO_OK : (int)e;
}

extern "C" int litho_ilt_theta_grad(const float* grad_m, const float* mask, long long count, float beta, float* q,
                                    cudaStream_t s) {
  if (!grad_m || !mask || !q) return LITHO_E_NULL;
  if (count < 0) return LITHO_E_SIZE;
  k_ilt_theta_grad<<<grid_for(count, 256, sms_here() * 16), 256, 0, s>>>(grad_m, mask, count, beta, q);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? LITHO_OK : (int)e;
}

extern "C" int litho_ilt_adam(const float* g, long long count, float step, float b1, float b2, float eps, int it,
                              float* theta, float* m1, float* m2, cudaStream_t s) {
  if (!g || !theta || !m1 || !m2) return LITHO_E_NULL;
  if (count < 0 || it < 1) return LITHO_E_SIZE;
  const float c1 = (float)(1.0 - pow((double)b1, it)), c2 = (float)(1.0 - pow((double)b2, it));
  k_ilt_adam<<<grid_for(count, 256, sms_here() * 16), 256, 0, s>>>(g, count, step, b1, b2, eps, c1, c2, theta, m1,
                                                                   m2);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? LITHO_OK : (int)e;
}

extern "C" int litho_ilt_update(const float* g, long long count, float beta, float beta_next, float step, float b1,
                                float b2, float eps, int it, float* theta, float* m1, float* m2, float* mask,
                                cudaStream_t s) {
  if (!g || !theta || !m1 || !m2 || !mask) return LITHO_E_NULL;
  if (count < 0 || (count & 3) || it < 1) return LITHO_E_SIZE;
  if (((uintptr_t)g | (uintptr_t)theta | (uintptr_t)m1 | (uintptr_t)m2 | (uintptr_t)mask) & 15) return LITHO_E_ALIGN;
  const float c1 = (float)(1.0 - pow((double)b1, it)), c2 = (float)(1.0 - pow((double)b2, it));
  k_ilt_update<<<grid_for(count / 4, 256, sms_here() * 16), 256, 0, s>>>(g, count, beta, beta_next, step, b1, b2,
                                                                         eps, c1, c2, theta, m1, m2, mask);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? LITHO_OK : (int)e;
}

extern "C" int litho_ilt_update_sched(const float* g, long long count, LithoIltSched* sched, float step, float b1,
                                      float b2, float eps, float* theta, float* m1, float* m2, float* mask,
                                      cudaStream_t s) {
  if (!g || !sched || !theta || !m1 || !m2 || !mask) return LITHO_E_NULL;
  if (count < 0 || (count & 3)) return LITHO_E_SIZE;
  if (((uintptr_t)g | (uintptr_t)theta | (uintptr_t)m1 | (uintptr_t)m2 | (uintptr_t)mask) & 15) return LITHO_E_ALIGN;
  if ((uintptr_t)sched & 7) return LITHO_E_ALIGN;
  k_ilt_update_sf<<<grid_for(count / 4, 256, sms_here() * 16), 256, 0, s>>>(g, count, sched, step, b1, b2, eps,
                                                                           theta, m1, m2, mask);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? LITHO_OK : (int)e;
}

extern "C" int litho_gaussian_blur(const float* in, float* out, float* tmp, int n_fields, int n,
                                   const float* weights_dev, int radius, cudaStream_t s) {
  if (!in || !out || !tmp || !weights_dev) return LITHO_E_NULL;
  if (n_fields < 1 || n < 1 || radius < 0) return LITHO_E_SIZE;
  const long long total = (long long)n_fields * n * n;
  const int g = grid_for(total, 256, sms_here() * 16);
  k_blur_axis<<<g, 256, 0, s>>>(in, tmp, n_fields, n, weights_dev, radius, 0);
  k_blur_axis<<<g, 256, 0, s>>>(tmp, out, n_fields, n, weights_dev, radius, 1);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? LITHO_OK : (int)e;
}
