// The plain per-source-point Abbe loop on full N x N grids — the comparison
// baseline for the band-limited engine in abbe.cu, and a general fallback.
//
// It is the reference's algorithm (expose/aerial_image.py:_abbe_sum,
// :421-488, with the batched flush of :336-348) moved to the GPU without
// restructuring: the full mask spectrum is one 2-D FFT; then, batch by
// batch, every coherent system's N x N spectrum M(f) P(f - f_s) V_c is
// built in HBM, inverse transformed by a row pass and a column pass, and
// w |E|^2 is accumulated into the image by a separate kernel.
//
// Transforms: power-of-two N in [16, 4096], radix-2, in place in shared
// memory, twiddles from an FP64-built table.
#include "common.cuh"
#include "fftsmem.cuh"

namespace litho {

// Row transforms. in: rows of n float (REAL) or float2; out: float2 rows.
template <int SIGN, bool REAL>
__global__ void k_fft_rows(const void* __restrict__ in, float2* __restrict__ out, long long n_rows, int n,
                           int log2n, int rows_per_block, float scale, const float2* __restrict__ tw_inv) {
  extern __shared__ float2 sm[];
  float2* tw = sm;
  float2* s = sm + n;
  for (int j = threadIdx.x; j < n; j += blockDim.x) tw[j] = tw_inv[j];
  const long long r0 = (long long)blockIdx.x * rows_per_block;
  for (int id = threadIdx.x; id < rows_per_block * n; id += blockDim.x) {
    const int r = id / n, x = id - r * n;
    float2 v = make_float2(0.f, 0.f);
    if (r0 + r < n_rows) {
      const size_t g = (size_t)(r0 + r) * n + x;
      v = REAL ? make_float2(reinterpret_cast<const float*>(in)[g], 0.f) : reinterpret_cast<const float2*>(in)[g];
    }
    s[r * n + brev(x, log2n)] = v;
  }
  block_fft_lines<SIGN>(s, n, rows_per_block, n, tw);
  for (int id = threadIdx.x; id < rows_per_block * n; id += blockDim.x) {
    const int r = id / n, x = id - r * n;
    if (r0 + r < n_rows) out[(size_t)(r0 + r) * n + x] = cscale(s[r * n + x], scale);
  }
}

// Column transforms of n x n planes, in place; a block owns `tc` columns.
template <int SIGN>
__global__ void k_fft_cols(float2* __restrict__ buf, int n, int log2n, int tc, float scale,
                           const float2* __restrict__ tw_inv) {
  extern __shared__ float2 sm[];
  float2* tw = sm;
  float2* s = sm + n;  // [tc][n]
  const int col_blocks = n / tc;
  const long long plane = blockIdx.x / col_blocks;
  const int c0 = (blockIdx.x % col_blocks) * tc;
  float2* base = buf + (size_t)plane * n * n;
  for (int j = threadIdx.x; j < n; j += blockDim.x) tw[j] = tw_inv[j];
  for (int id = threadIdx.x; id < tc * n; id += blockDim.x) {
    const int y = id / tc, c = id - y * tc;
    s[c * n + brev(y, log2n)] = base[(size_t)y * n + c0 + c];
  }
  block_fft_lines<SIGN>(s, n, tc, n, tw);
  for (int id = threadIdx.x; id < tc * n; id += blockDim.x) {
    const int y = id / tc, c = id - y * tc;
    base[(size_t)y * n + c0 + c] = cscale(s[c * n + y], scale);
  }
}

// Build the batch's spectra: spec[jb][c] = M(k) * table(k) on each disc.
__global__ void k_plain_scatter(const LithoJob* __restrict__ jobs, int j0, int nb, const float2* __restrict__ table,
                                int h, int ncomp_max, const float2* __restrict__ Mfull, int n,
                                float2* __restrict__ spec) {
  const int side = 2 * h + 1, npts = side * side;
  const long long total = (long long)nb * ncomp_max * npts;
  for (long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x; id < total;
       id += (long long)gridDim.x * blockDim.x) {
    const int p = (int)(id % npts);
    const long long jc = id / npts;
    const int c = (int)(jc % ncomp_max), jb = (int)(jc / ncomp_max);
    const int j = j0 + jb;
    const LithoJob job = jobs[j];
    if (c >= job.ncomp) continue;
    const int kx = job.cx + p % side - h, ky = job.cy + p / side - h;
    if (!bin_valid(kx, n) || !bin_valid(ky, n)) continue;
    const int ix = (kx + n) % n, iy = (ky + n) % n;
    const float2 t = table[((size_t)job.tab * ncomp_max + c) * npts + p];
    const float2 m = Mfull[((size_t)job.clip * n + iy) * n + ix];
    spec[(((size_t)jb * ncomp_max + c) * n + iy) * n + ix] = cmul(t, m);
  }
}

// image[out_j] += w_j |E_jc|^2, in job order per pixel (deterministic).
__global__ void k_plain_accumulate(const LithoJob* __restrict__ jobs, int j0, int nb, int ncomp_max,
                                   const float2* __restrict__ E, int n, float* __restrict__ image) {
  const size_t NN = (size_t)n * n;
  for (size_t px = blockIdx.x * (size_t)blockDim.x + threadIdx.x; px < NN; px += (size_t)gridDim.x * blockDim.x) {
    int cur = -1;
    float acc = 0.f;
    for (int jb = 0; jb < nb; ++jb) {
      const LithoJob job = jobs[j0 + jb];
      if (job.out != cur) {
        if (cur >= 0) image[(size_t)cur * NN + px] += acc;
        cur = job.out;
        acc = 0.f;
      }
      float s = 0.f;
      for (int c = 0; c < job.ncomp; ++c) s += cabs2(E[((size_t)jb * ncomp_max + c) * NN + px]);
      acc = fmaf((float)job.weight, s, acc);
    }
    if (cur >= 0) image[(size_t)cur * NN + px] += acc;
  }
}

__global__ void k_plain_blockmax(const float* __restrict__ image, int n, int nblk, float* __restrict__ blockmax) {
  __shared__ float red[32];
  const int o = blockIdx.y;
  const size_t NN = (size_t)n * n;
  float mx = 0.f;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < NN; i += (size_t)nblk * blockDim.x)
    mx = fmaxf(mx, image[(size_t)o * NN + i]);
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, off));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
  __syncthreads();
  if (threadIdx.x == 0) {
    float m = red[0];
    for (int i = 1; i < (int)(blockDim.x >> 5); ++i) m = fmaxf(m, red[i]);
    blockmax[(size_t)o * nblk + blockIdx.x] = m;
  }
}

static int ilog2i(int n) {
  int l = 0;
  while ((1 << l) < n) ++l;
  return l;
}

static int rows_per_block_for(int n) { return n >= 1024 ? 2 : (2048 / n); }

// 2-D transform of `planes` n x n planes in buf (in place unless `in` given).
cudaError_t plain_fft2(const void* in, bool in_real, float2* buf, long long planes, int n, int sign, float scale_rows,
                       float scale_cols, const float2* tw, cudaStream_t st) {
  const int lg = ilog2i(n);
  const int rpb = rows_per_block_for(n);
  const long long rows = planes * n;
  const size_t smr = (size_t)(n + rpb * n) * sizeof(float2);
  const unsigned gr = (unsigned)((rows + rpb - 1) / rpb);
  const void* src = in ? in : buf;
  if (sign > 0) {
    cudaFuncSetAttribute(k_fft_rows<1, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smr);
    k_fft_rows<1, false><<<gr, 256, smr, st>>>(src, buf, rows, n, lg, rpb, scale_rows, tw);
  } else if (in_real) {
    cudaFuncSetAttribute(k_fft_rows<-1, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smr);
    k_fft_rows<-1, true><<<gr, 256, smr, st>>>(src, buf, rows, n, lg, rpb, scale_rows, tw);
  } else {
    cudaFuncSetAttribute(k_fft_rows<-1, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smr);
    k_fft_rows<-1, false><<<gr, 256, smr, st>>>(src, buf, rows, n, lg, rpb, scale_rows, tw);
  }
  const int tc = n >= 8 ? 8 : n;
  const size_t smc = (size_t)(n + tc * n) * sizeof(float2);
  const unsigned gc = (unsigned)(planes * (n / tc));
  if (sign > 0) {
    cudaFuncSetAttribute(k_fft_cols<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smc);
    k_fft_cols<1><<<gc, 256, smc, st>>>(buf, n, lg, tc, scale_cols, tw);
  } else {
    cudaFuncSetAttribute(k_fft_cols<-1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smc);
    k_fft_cols<-1><<<gc, 256, smc, st>>>(buf, n, lg, tc, scale_cols, tw);
  }
  return cudaGetLastError();
}

}  // namespace litho

// ---------------------------------------------------------------------------
// host entry (C ABI)
// ---------------------------------------------------------------------------
using namespace litho;

namespace litho {
cudaError_t launch_pupil_table(const LithoAbbePlan& p, const void* blob, float2* table, cudaStream_t s);
__global__ void k_normalise(const float* __restrict__ blockmax, int nblk, const LithoNorm* __restrict__ norm,
                            int n, float* __restrict__ image, float* __restrict__ peak, int apply_mode0);
}

struct PlainLayout {
  int64_t tw, mfull, table, batch, blockmax, total;
};

static const int kPlainMaxBlk = 256;

static PlainLayout plain_layout(const LithoAbbePlan& p, int batch) {
  PlainLayout l{};
  const int64_t NN = (int64_t)p.n * p.n, side = 2 * p.h + 1;
  int64_t off = 0;
  l.tw = off;       off = align16(off + (int64_t)p.n * 8);
  l.mfull = off;    off = align16(off + (int64_t)p.n_clips * NN * 8);
  l.table = off;    off = align16(off + (int64_t)p.n_tab * p.ncomp_max * side * side * 8);
  l.batch = off;    off = align16(off + (int64_t)batch * p.ncomp_max * NN * 8);
  l.blockmax = off; off = align16(off + (int64_t)p.n_out * kPlainMaxBlk * 4);
  l.total = off;
  return l;
}

static int check_plain(const LithoAbbePlan* p, int batch) {
  if (!p) return LITHO_E_NULL;
  if (p->n < 16 || p->n > 4096 || (p->n & (p->n - 1))) return LITHO_E_UNSUPPORTED;
  if (p->n_clips < 1 || p->n_out < 1 || p->n_jobs < 1 || p->n_pupils < 1 || p->h < 0 || batch < 1 ||
      p->n_tab < 1 || p->n_tab > p->n_jobs)
    return LITHO_E_SIZE;
  if (p->ncomp_max != 1 && p->ncomp_max != 3) return LITHO_E_SIZE;
  if (!(p->pixel_size > 0.0)) return LITHO_E_SIZE;
  const int64_t offs[7] = {p->off_jobs, p->off_pupils, p->off_items, p->off_out_items, p->off_norm,
                           p->off_slots, p->mirrored ? p->off_mirrors : 0};
  for (int i = 0; i < 7; ++i)
    if (offs[i] < 0 || (offs[i] & 15)) return LITHO_E_ALIGN;
  if (p->mirrored != 0 && p->mirrored != 1) return LITHO_E_SIZE;
  return LITHO_OK;
}

extern "C" int litho_abbe_plain_workspace(const LithoAbbePlan* plan, int batch, size_t* bytes) {
  const int st = check_plain(plan, batch);
  if (st) return st;
  if (!bytes) return LITHO_E_NULL;
  *bytes = (size_t)plain_layout(*plan, batch).total;
  return LITHO_OK;
}

extern "C" int litho_abbe_plain(const LithoAbbePlan* plan, int batch, const void* blob, const void* mask,
                                float* image, float* peak, void* ws, size_t ws_bytes, cudaStream_t s) {
  int st = check_plain(plan, batch);
  if (st) return st;
  if (!blob || !mask || !image || !peak || !ws) return LITHO_E_NULL;
  if (((uintptr_t)ws & 15) || ((uintptr_t)blob & 15) || ((uintptr_t)mask & 7)) return LITHO_E_ALIGN;
  const LithoAbbePlan& p = *plan;
  const PlainLayout l = plain_layout(p, batch);
  if ((int64_t)ws_bytes < l.total) return LITHO_E_WORKSPACE;
  const char* b = static_cast<const char*>(blob);
  const LithoJob* jobs = reinterpret_cast<const LithoJob*>(b + p.off_jobs);
  const LithoNorm* norm = reinterpret_cast<const LithoNorm*>(b + p.off_norm);
  char* w = static_cast<char*>(ws);
  float2* tw = reinterpret_cast<float2*>(w + l.tw);
  float2* mfull = reinterpret_cast<float2*>(w + l.mfull);
  float2* table = reinterpret_cast<float2*>(w + l.table);
  float2* buf = reinterpret_cast<float2*>(w + l.batch);
  float* blockmax = reinterpret_cast<float*>(w + l.blockmax);
  const int n = p.n;
  const size_t NN = (size_t)n * n;
  cudaError_t e;

  k_twiddle_table<<<(n + 255) / 256, 256, 0, s>>>(tw, n, +1);
  if ((e = launch_pupil_table(p, blob, table, s)) != cudaSuccess) return (int)e;
  // full mask spectrum / N^2 (the inverse below is unnormalised)
  e = plain_fft2(mask, p.mask_complex == 0, mfull, p.n_clips, n, -1, 1.0f, 1.0f / ((float)n * (float)n), tw, s);
  if (e != cudaSuccess) return (int)e;
  if ((e = cudaMemsetAsync(image, 0, (size_t)p.n_out * NN * sizeof(float), s)) != cudaSuccess) return (int)e;
  const int side = 2 * p.h + 1;
  for (int j0 = 0; j0 < p.n_jobs; j0 += batch) {
    const int nb = (p.n_jobs - j0) < batch ? (p.n_jobs - j0) : batch;
    if ((e = cudaMemsetAsync(buf, 0, (size_t)nb * p.ncomp_max * NN * sizeof(float2), s)) != cudaSuccess) return (int)e;
    const long long tot = (long long)nb * p.ncomp_max * side * side;
    k_plain_scatter<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(jobs, j0, nb, table, p.h, p.ncomp_max, mfull, n, buf);
    e = plain_fft2(nullptr, false, buf, (long long)nb * p.ncomp_max, n, +1, 1.0f, 1.0f, tw, s);
    if (e != cudaSuccess) return (int)e;
    const unsigned ga = (unsigned)((NN + 255) / 256 < 4096 ? (NN + 255) / 256 : 4096);
    k_plain_accumulate<<<ga, 256, 0, s>>>(jobs, j0, nb, p.ncomp_max, buf, n, image);
    if ((e = cudaGetLastError()) != cudaSuccess) return (int)e;
  }
  dim3 gm(kPlainMaxBlk, p.n_out);
  k_plain_blockmax<<<gm, 256, 0, s>>>(image, n, kPlainMaxBlk, blockmax);
  dim3 gn((unsigned)((NN + 255) / 256 < 512 ? (NN + 255) / 256 : 512), p.n_out);
  k_normalise<<<gn, 256, 0, s>>>(blockmax, kPlainMaxBlk, norm, n, image, peak, 1);
  if ((e = cudaGetLastError()) != cudaSuccess) return (int)e;
  return LITHO_OK;
}

// ---------------------------------------------------------------------------
// Plain SOCS forward and adjoint on full N x N grids (the reference's
// opc/ilt.py:socs_fields :227-231 and socs_gradient :262-266 moved to the GPU
// unchanged): one full 2-D FFT per kernel and direction, kernels scattered
// from their band values. The comparison baseline for csrc/ilt.cu.
// ---------------------------------------------------------------------------
namespace litho {

// out[c] = 0 off the band, phi(b) * M[c](b) (conj(phi) if CONJ) on it.
template <bool CONJ>
__global__ void k_plain_band_mul(const float2* __restrict__ M, const float2* __restrict__ phi,
                                 const int32_t* __restrict__ bkx, const int32_t* __restrict__ bky, int nb, int n,
                                 int n_clips, float2* __restrict__ out) {
  const long long total = (long long)n_clips * nb;
  for (long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x; id < total;
       id += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(id / nb), b = (int)(id % nb);
    const int ix = (bkx[b] + n) % n, iy = (bky[b] + n) % n;
    const size_t at = ((size_t)c * n + iy) * n + ix;
    const float2 f = phi[b];
    out[at] = CONJ ? cmulc(M[at], f) : cmul(f, M[at]);
  }
}

__global__ void k_plain_intensity(const float2* __restrict__ E, long long total, float lam, int first,
                                  float* __restrict__ I) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const float v = lam * cabs2(E[i]);
    I[i] = first ? v : I[i] + v;
  }
}

__global__ void k_plain_mul_real(const float* __restrict__ g, const float2* __restrict__ E, long long total,
                                 float2* __restrict__ out) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x)
    out[i] = cscale(E[i], g[i]);
}

__global__ void k_plain_grad(const float2* __restrict__ adj, long long total, float two_lam, int first,
                             float* __restrict__ grad) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const float v = two_lam * adj[i].x;
    grad[i] = first ? v : grad[i] + v;
  }
}

static unsigned grid_elems(long long total) {
  long long b = (total + 255) / 256;
  return (unsigned)(b > 8192 ? 8192 : (b < 1 ? 1 : b));
}

}  // namespace litho

static int64_t plain_socs_ws(int n_clips, int n) {
  return align16((int64_t)n * 8) + 2 * align16((int64_t)n_clips * n * n * 8);
}

extern "C" int litho_plain_socs_workspace(int n_clips, int n, size_t* bytes) {
  if (!bytes) return LITHO_E_NULL;
  if (n_clips < 1 || n < 16 || n > 4096 || (n & (n - 1))) return LITHO_E_UNSUPPORTED;
  *bytes = (size_t)plain_socs_ws(n_clips, n);
  return LITHO_OK;
}

// fields_out[k][c] = ifft2(phi_k * fft2(mask_c)), I_out[c] = sum_k lambda_k |fields|^2.
extern "C" int litho_plain_socs_forward(const float* masks, int n_clips, int n, int K, const float2* phi,
                                        const float* lam_host, const int32_t* bkx, const int32_t* bky, int nb,
                                        float2* fields_out, float* I_out, void* ws, size_t ws_bytes,
                                        cudaStream_t s) {
  if (!masks || !phi || !lam_host || !bkx || !bky || !fields_out || !I_out || !ws) return LITHO_E_NULL;
  if (n_clips < 1 || n < 16 || n > 4096 || (n & (n - 1)) || K < 1 || nb < 1) return LITHO_E_UNSUPPORTED;
  if ((int64_t)ws_bytes < plain_socs_ws(n_clips, n)) return LITHO_E_WORKSPACE;
  char* w = static_cast<char*>(ws);
  float2* tw = reinterpret_cast<float2*>(w);
  float2* M = reinterpret_cast<float2*>(w + align16((int64_t)n * 8));
  const long long NN = (long long)n * n, tot = NN * n_clips;
  const float inv = 1.0f / ((float)n * (float)n);
  k_twiddle_table<<<(n + 255) / 256, 256, 0, s>>>(tw, n, +1);
  cudaError_t e = plain_fft2(masks, true, M, n_clips, n, -1, 1.0f, 1.0f, tw, s);
  if (e != cudaSuccess) return (int)e;
  for (int k = 0; k < K; ++k) {
    float2* E = fields_out + (size_t)k * tot;
    if ((e = cudaMemsetAsync(E, 0, (size_t)tot * sizeof(float2), s)) != cudaSuccess) return (int)e;
    k_plain_band_mul<false><<<grid_elems((long long)n_clips * nb), 256, 0, s>>>(M, phi + (size_t)k * nb, bkx, bky,
                                                                                nb, n, n_clips, E);
    e = plain_fft2(nullptr, false, E, n_clips, n, +1, 1.0f, inv, tw, s);
    if (e != cudaSuccess) return (int)e;
    k_plain_intensity<<<grid_elems(tot), 256, 0, s>>>(E, tot, lam_host[k], k == 0, I_out);
  }
  e = cudaGetLastError();
  return e == cudaSuccess ? LITHO_OK : (int)e;
}

// grad_out[c] = 2 Re sum_k lambda_k ifft2(conj(phi_k) fft2(sens_c fields[k][c])).
extern "C" int litho_plain_socs_adjoint(const float2* fields, const float* sens, int n_clips, int n, int K,
                                        const float2* phi, const float* lam_host, const int32_t* bkx,
                                        const int32_t* bky, int nb, float* grad_out, void* ws, size_t ws_bytes,
                                        cudaStream_t s) {
  if (!fields || !sens || !phi || !lam_host || !bkx || !bky || !grad_out || !ws) return LITHO_E_NULL;
  if (n_clips < 1 || n < 16 || n > 4096 || (n & (n - 1)) || K < 1 || nb < 1) return LITHO_E_UNSUPPORTED;
  if ((int64_t)ws_bytes < plain_socs_ws(n_clips, n)) return LITHO_E_WORKSPACE;
  char* w = static_cast<char*>(ws);
  float2* tw = reinterpret_cast<float2*>(w);
  float2* Bk = reinterpret_cast<float2*>(w + align16((int64_t)n * 8));
  float2* Sk = reinterpret_cast<float2*>(w + align16((int64_t)n * 8) + align16((int64_t)n_clips * n * n * 8));
  const long long NN = (long long)n * n, tot = NN * n_clips;
  const float inv = 1.0f / ((float)n * (float)n);
  k_twiddle_table<<<(n + 255) / 256, 256, 0, s>>>(tw, n, +1);
  cudaError_t e;
  for (int k = 0; k < K; ++k) {
    k_plain_mul_real<<<grid_elems(tot), 256, 0, s>>>(sens, fields + (size_t)k * tot, tot, Bk);
    e = plain_fft2(nullptr, false, Bk, n_clips, n, -1, 1.0f, 1.0f, tw, s);
    if (e != cudaSuccess) return (int)e;
    if ((e = cudaMemsetAsync(Sk, 0, (size_t)tot * sizeof(float2), s)) != cudaSuccess) return (int)e;
    k_plain_band_mul<true><<<grid_elems((long long)n_clips * nb), 256, 0, s>>>(Bk, phi + (size_t)k * nb, bkx, bky,
                                                                               nb, n, n_clips, Sk);
    e = plain_fft2(nullptr, false, Sk, n_clips, n, +1, 1.0f, inv, tw, s);
    if (e != cudaSuccess) return (int)e;
    k_plain_grad<<<grid_elems(tot), 256, 0, s>>>(Sk, tot, 2.0f * lam_host[k], k == 0, grad_out);
  }
  e = cudaGetLastError();
  return e == cudaSuccess ? LITHO_OK : (int)e;
}
