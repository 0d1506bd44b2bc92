// SOCS forward and backward as single calls over a kernel table.
//
// expose/hopkins.py:SOCSKernels.raw (:205-218) images a mask as
// sum_k lambda_k |ifft2(phi_k fft2(mask))|^2 and opc/ilt.py:socs_gradient
// (:235-266) differentiates that sum. Here both run on the band-limited
// engines, composed from the library's own stages: the job list (one job per
// clip x kernel, weight lambda_k, table slot k, no source shift) is written
// into the caller's workspace by a kernel, so a call needs no host buffer
// that outlives it and allocates nothing.
#include "common.cuh"

namespace litho {
namespace {

constexpr int kSocsThreads = 256;

int coarse_side(int h) {
  int L = 32;
  while (L < 4 * h + 1) L *= 2;
  return L;
}

int jobs_per_item(int n_clips, int K, int L) {
  if (L > 64) return 8;
  const int per = (n_clips * K) / (4 * 148);
  return per < 2 ? 2 : per > 8 ? 8 : per;
}

struct SocsPlan {
  LithoAbbePlan p;
  int64_t blob_bytes;
  int items_per_clip, per;
};

SocsPlan socs_plan(int n_clips, int n, int K, int h, int mask_complex, int norm_mode, double pixel_size) {
  SocsPlan s{};
  LithoAbbePlan& p = s.p;
  const int L = coarse_side(h);
  s.per = jobs_per_item(n_clips, K, L);
  s.items_per_clip = (K + s.per - 1) / s.per;
  p.n = n;
  p.n_clips = n_clips;
  p.n_out = n_clips;
  p.n_jobs = n_clips * K;
  p.n_items = n_clips * s.items_per_clip;
  p.n_pupils = 1;
  p.h = h;
  p.bm = h;
  p.L = L;
  p.mask_complex = mask_complex;
  p.ncomp_max = 1;
  p.n_tab = K;
  p.pixel_size = pixel_size;
  int64_t off = 0;
  p.off_jobs = off;      off = align16(off + (int64_t)p.n_jobs * (int64_t)sizeof(LithoJob));
  p.off_pupils = off;    off = align16(off + (int64_t)sizeof(LithoPupil));
  p.off_items = off;     off = align16(off + (int64_t)p.n_items * (int64_t)sizeof(LithoItem));
  p.off_out_items = off; off = align16(off + (int64_t)(n_clips + 1) * 4);
  p.off_norm = off;      off = align16(off + (int64_t)n_clips * (int64_t)sizeof(LithoNorm));
  p.off_slots = off;     off = align16(off + (int64_t)K * 4);
  p.mirrored = 0;
  p.off_mirrors = 0;
  s.blob_bytes = (off + 255) & ~int64_t(255);
  (void)norm_mode;
  return s;
}

__global__ void k_socs_plan(char* blob, LithoAbbePlan p, const double* __restrict__ weights, int K, int per,
                            int items_per_clip, int norm_mode, float norm_scale) {
  LithoJob* jobs = reinterpret_cast<LithoJob*>(blob + p.off_jobs);
  LithoPupil* pupil = reinterpret_cast<LithoPupil*>(blob + p.off_pupils);
  LithoItem* items = reinterpret_cast<LithoItem*>(blob + p.off_items);
  int32_t* out_items = reinterpret_cast<int32_t*>(blob + p.off_out_items);
  LithoNorm* norm = reinterpret_cast<LithoNorm*>(blob + p.off_norm);
  int32_t* slots = reinterpret_cast<int32_t*>(blob + p.off_slots);
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
  for (int j = tid; j < p.n_jobs; j += stride) {
    const int c = j / K, k = j % K;
    LithoJob jb{};
    jb.weight = weights[k];
    jb.pupil = 0;
    jb.clip = c;
    jb.out = c;
    jb.ncomp = 1;
    jb.tab = k;
    jobs[j] = jb;
  }
  for (int i = tid; i < p.n_items; i += stride) {
    const int c = i / items_per_clip, q = i % items_per_clip;
    const int b = c * K + q * per, e = b + per < (c + 1) * K ? b + per : (c + 1) * K;
    items[i] = LithoItem{c, b, e, 0};
  }
  for (int c = tid; c <= p.n_clips; c += stride) out_items[c] = c * items_per_clip;
  for (int c = tid; c < p.n_clips; c += stride) norm[c] = LithoNorm{norm_mode, norm_scale};
  for (int k = tid; k < K; k += stride) slots[k] = k;
  if (tid == 0) {
    LithoPupil pu{};
    pu.wavelength = 1.0;
    pu.NA = 1.0;
    pu.n_image = 1.0;
    *pupil = pu;
  }
}

int check_socs_args(int K, int h, int n_clips, int n) {
  if (K < 1 || h < 0 || n_clips < 1 || n < 2) return LITHO_E_SIZE;
  if (2 * h + 1 > n) return LITHO_E_BAND;
  return LITHO_OK;
}

int64_t al256(int64_t x) { return (x + 255) & ~int64_t(255); }

}  // namespace
}  // namespace litho

using namespace litho;

extern "C" int litho_socs_forward_workspace(int n_clips, int n, int K, int h, int mask_complex, size_t* bytes) {
  if (!bytes) return LITHO_E_NULL;
  int st = check_socs_args(K, h, n_clips, n);
  if (st) return st;
  const SocsPlan sp = socs_plan(n_clips, n, K, h, mask_complex != 0, 0, 1.0);
  size_t ws = 0;
  st = litho_abbe_workspace(&sp.p, &ws);
  if (st) return st;
  *bytes = (size_t)sp.blob_bytes + (size_t)al256((int64_t)ws);
  return LITHO_OK;
}

extern "C" int litho_socs_forward(const void* table_dev, const double* weights_dev, int K, int h,
                                  const void* mask_dev, int mask_complex, int n_clips, int n, int norm_mode,
                                  float norm_scale, float* image_out_dev, float* peak_out_dev, void* workspace_dev,
                                  size_t workspace_bytes, cudaStream_t s) {
  if (!table_dev || !weights_dev || !mask_dev || !image_out_dev || !peak_out_dev || !workspace_dev)
    return LITHO_E_NULL;
  if (norm_mode != 0 && norm_mode != 1) return LITHO_E_SIZE;
  if (((uintptr_t)workspace_dev & 255) || ((uintptr_t)weights_dev & 7)) return LITHO_E_ALIGN;
  size_t need = 0;
  int st = litho_socs_forward_workspace(n_clips, n, K, h, mask_complex, &need);
  if (st) return st;
  if (workspace_bytes < need) return LITHO_E_WORKSPACE;
  const SocsPlan sp = socs_plan(n_clips, n, K, h, mask_complex != 0, norm_mode, 1.0);
  char* blob = static_cast<char*>(workspace_dev);
  const int jobs = sp.p.n_jobs > sp.p.n_items ? sp.p.n_jobs : sp.p.n_items;
  const int blocks = (jobs + kSocsThreads - 1) / kSocsThreads < 1024 ? (jobs + kSocsThreads - 1) / kSocsThreads : 1024;
  k_socs_plan<<<blocks > 0 ? blocks : 1, kSocsThreads, 0, s>>>(blob, sp.p, weights_dev, K, sp.per, sp.items_per_clip,
                                                               norm_mode, norm_scale);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return (int)e;
  return litho_abbe_tabled(&sp.p, blob, table_dev, mask_dev, image_out_dev, peak_out_dev, blob + sp.blob_bytes,
                           workspace_bytes - (size_t)sp.blob_bytes, s);
}

namespace {
struct BackLayout {
  int64_t blob, mbox, gbox, hbox, band_ws, adj_ws, syn_ws, total;
};

int back_layout(const SocsPlan& sp, int n_clips, int n, int h, BackLayout* l) {
  size_t band_m = 0, band_g = 0, adj = 0, syn = 0;
  int st;
  if ((st = litho_band_spectrum_workspace(n_clips, n, h, &band_m))) return st;
  if ((st = litho_band_spectrum_workspace(n_clips, n, 2 * h, &band_g))) return st;
  if ((st = litho_socs_adjoint_workspace(n_clips, sp.p.n_items, h, &adj))) return st;
  if ((st = litho_band_synthesis_workspace(n_clips, n, &syn))) return st;
  const int64_t side = 2 * h + 1, G = 4 * h + 1;
  int64_t off = 0;
  l->blob = off;    off = al256(off + sp.blob_bytes);
  l->mbox = off;    off = al256(off + (int64_t)n_clips * side * side * 8);
  l->gbox = off;    off = al256(off + (int64_t)n_clips * G * G * 8);
  l->hbox = off;    off = al256(off + (int64_t)n_clips * side * side * 8);
  l->band_ws = off; off = al256(off + (int64_t)(band_m > band_g ? band_m : band_g));
  l->adj_ws = off;  off = al256(off + (int64_t)adj);
  l->syn_ws = off;  off = al256(off + (int64_t)syn);
  l->total = off;
  return LITHO_OK;
}
}  // namespace

extern "C" int litho_socs_backward_workspace(int n_clips, int n, int K, int h, size_t* bytes) {
  if (!bytes) return LITHO_E_NULL;
  int st = check_socs_args(K, h, n_clips, n);
  if (st) return st;
  const SocsPlan sp = socs_plan(n_clips, n, K, h, 0, 0, 1.0);
  BackLayout l{};
  if ((st = back_layout(sp, n_clips, n, h, &l))) return st;
  *bytes = (size_t)l.total;
  return LITHO_OK;
}

extern "C" int litho_socs_backward(const void* table_dev, const double* weights_dev, int K, int h,
                                   const float* mask_dev, int n_clips, int n, const float* sens_dev, float sens_scale,
                                   float* grad_out_dev, void* workspace_dev, size_t workspace_bytes, cudaStream_t s) {
  if (!table_dev || !weights_dev || !mask_dev || !sens_dev || !grad_out_dev || !workspace_dev) return LITHO_E_NULL;
  if (((uintptr_t)workspace_dev & 255) || ((uintptr_t)weights_dev & 7)) return LITHO_E_ALIGN;
  size_t need = 0;
  int st = litho_socs_backward_workspace(n_clips, n, K, h, &need);
  if (st) return st;
  if (workspace_bytes < need) return LITHO_E_WORKSPACE;
  const SocsPlan sp = socs_plan(n_clips, n, K, h, 0, 0, 1.0);
  BackLayout l{};
  if ((st = back_layout(sp, n_clips, n, h, &l))) return st;
  char* w = static_cast<char*>(workspace_dev);
  char* blob = w + l.blob;
  const int jobs = sp.p.n_jobs > sp.p.n_items ? sp.p.n_jobs : sp.p.n_items;
  const int blocks = (jobs + kSocsThreads - 1) / kSocsThreads < 1024 ? (jobs + kSocsThreads - 1) / kSocsThreads : 1024;
  k_socs_plan<<<blocks > 0 ? blocks : 1, kSocsThreads, 0, s>>>(blob, sp.p, weights_dev, K, sp.per, sp.items_per_clip,
                                                               0, 1.0f);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return (int)e;
  const float inv_nn = 1.0f / ((float)n * (float)n);
  const size_t band_bytes = (size_t)(l.adj_ws - l.band_ws);
  // M = F(mask) / N^2 on |k| <= h, G = F(sens_scale sens) / N^2 on |g| <= 2h
  if ((st = litho_band_spectrum(mask_dev, 0, n_clips, n, h, inv_nn, w + l.mbox, w + l.band_ws, band_bytes, s)))
    return st;
  if ((st = litho_band_spectrum(sens_dev, 0, n_clips, n, 2 * h, sens_scale * inv_nn, w + l.gbox, w + l.band_ws,
                                band_bytes, s)))
    return st;
  if ((st = litho_socs_adjoint(&sp.p, blob, table_dev, w + l.mbox, nullptr, w + l.gbox, w + l.hbox, w + l.adj_ws,
                               (size_t)(l.syn_ws - l.adj_ws), s)))
    return st;
  return litho_band_synthesis(w + l.hbox, n_clips, n, h, 0, grad_out_dev, w + l.syn_ws,
                              (size_t)(l.total - l.syn_ws), s);
}
