// The band TCC: SOCS image and adjoint band boxes as contractions with the
// truncated transmission cross-coefficient, for kernel bands whose TCC stays
// resident in L2 (half-width h <= 15, e.g. ArF immersion at 1024^2 and 1 nm).
//
// With the K kept kernels phi_k (unit vectors on the band |f| <= 2 NA / lambda,
// expose/hopkins.py:144-198) and weights lambda_k, the image of a mask whose
// band spectrum is M (F(m) / N^2) has the band box
//     B(g) = sum_f Tc(f + g, f) M(f + g) conj M(f),   |g| <= 2h,
// Tc(f1, f2) = sum_k lambda_k phi_k(f1) conj phi_k(f2), and the adjoint of
// sum_x G(x) I(x) (opc/ilt.py:socs_gradient, :262-266) has the band box
//     H(f) = A(f) + conj A(-f),  A(f) = sum_f' T(f, f') M(f') G(f - f'),
// T = conj Tc, G the band box of the sensitivity (F(G) / N^2, |g| <= 2h).
// Both are the reference's per-kernel sums regrouped: the kernel index is
// summed once into T (FP64, once per kernel set), so a step's cost does not
// grow with K and has no chain of small transforms.
//
// Inside the blob the band is sorted in signed row-major order (ky, then kx).
// The band is a disc, so every row is one contiguous run of kx, and it is
// centrally symmetric, so -f of the point with sorted index s has index
// nb - 1 - s. Layout (tcc_layout): map[(2h+1)^2] (box position -> sorted
// index or -1), perm[nb] (sorted -> caller's index), skx[nb], sky[nb] (sorted
// coordinates), rows lo/x0/n [2h+1] (first sorted index, first kx, length of
// each row ky = -h..h), T[nb][nb] and T2[Gh][nb] (complex64, sorted indices;
// T2[q][s] = Tc(f_s + g_q, f_s) for the upper half g_q = box position p_c + q
// of the image box, 0 where f_s + g_q leaves the band).
#include "common.cuh"

namespace litho {
namespace {

struct TccLayout {
  int64_t map, perm, skx, sky, rows, T, T2, total;
  int side, G, Gh;
};

TccLayout tcc_layout(int nb, int h) {
  TccLayout l{};
  l.side = 2 * h + 1;
  l.G = 4 * h + 1;
  l.Gh = (l.G * l.G + 1) / 2;
  int64_t off = 0;
  l.map = off;  off = align16(off + (int64_t)l.side * l.side * 4);
  l.perm = off; off = align16(off + (int64_t)nb * 4);
  l.skx = off;  off = align16(off + (int64_t)nb * 4);
  l.sky = off;  off = align16(off + (int64_t)nb * 4);
  l.rows = off; off = align16(off + (int64_t)3 * l.side * 4);
  l.T = off;    off = align16(off + (int64_t)nb * nb * 8);
  l.T2 = off;   off = align16(off + (int64_t)l.Gh * nb * 8);
  l.total = off;
  return l;
}

constexpr int64_t kTccMaxBytes = (int64_t)96 << 20;   // stays well inside the 126 MB L2
constexpr int kTccHMax = 15;                          // a band row fits a warp (2h + 1 <= 32)

// The sorted band, its maps and row runs (one block). bad = 1 when a point
// lies outside the box, two points share a position, a row is not one run,
// or the band is not centrally symmetric.
__global__ void k_tcc_index(const int32_t* __restrict__ bkx, const int32_t* __restrict__ bky, int nb, int h,
                            int32_t* __restrict__ map, int32_t* __restrict__ perm, int32_t* __restrict__ skx,
                            int32_t* __restrict__ sky, int32_t* __restrict__ rows, int* __restrict__ bad) {
  const int side = 2 * h + 1, npts = side * side;
  int32_t* lo = rows;
  int32_t* x0 = rows + side;
  int32_t* cnt = rows + 2 * side;
  for (int p = threadIdx.x; p < npts; p += blockDim.x) map[p] = -1;
  __syncthreads();
  for (int b = threadIdx.x; b < nb; b += blockDim.x) {
    const int x = bkx[b], y = bky[b];
    if (x < -h || x > h || y < -h || y > h) {
      atomicExch(bad, 1);
      continue;
    }
    if (atomicCAS(&map[(y + h) * side + x + h], -1, b) != -1) atomicExch(bad, 1);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int s = 0;
    for (int y = 0; y < side; ++y) {
      lo[y] = s;
      x0[y] = 0;
      int run = 0, prev = -2;
      for (int x = 0; x < side; ++x) {
        const int p = y * side + x, b = map[p];
        if (b < 0) continue;
        if (run == 0) x0[y] = x - h;
        else if (x != prev + 1) *bad = 1;   // a gap: the row is not one run
        prev = x;
        ++run;
        if (s < nb) {
          perm[s] = b;
          skx[s] = x - h;
          sky[s] = y - h;
        }
        map[p] = s++;
      }
      cnt[y] = run;
    }
    if (s != nb) *bad = 1;
  }
  __syncthreads();
  for (int s = threadIdx.x; s < nb; s += blockDim.x) {
    const int t = nb - 1 - s;
    if (skx[t] != -skx[s] || sky[t] != -sky[s]) atomicExch(bad, 1);
  }
}

// T[s][s'] = sum_k lambda_k conj phi_k(s) phi_k(s') in FP64, stored complex64
__global__ void k_tcc_T(const double2* __restrict__ phi, const double* __restrict__ lam, int K, int nb,
                        const int32_t* __restrict__ perm, float2* __restrict__ T) {
  const int64_t total = (int64_t)nb * nb;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int b = perm[(int)(i / nb)], c = perm[(int)(i % nb)];
    double re = 0.0, im = 0.0;
    for (int k = 0; k < K; ++k) {
      const double2 u = phi[(size_t)k * nb + b], v = phi[(size_t)k * nb + c];
      const double l = lam[k];
      re += l * (u.x * v.x + u.y * v.y);   // conj(u) v
      im += l * (u.x * v.y - u.y * v.x);
    }
    T[i] = make_float2((float)re, (float)im);
  }
}

// T2[q][s] = Tc(f_s + g_q, f_s) = conj T[s(f_s + g_q)][s], 0 off the band
__global__ void k_tcc_T2(const float2* __restrict__ T, const int32_t* __restrict__ map,
                         const int32_t* __restrict__ skx, const int32_t* __restrict__ sky, int nb, int h, int Gh,
                         float2* __restrict__ T2) {
  const int side = 2 * h + 1, G = 4 * h + 1, pc = (G * G - 1) / 2;
  const int64_t total = (int64_t)Gh * nb;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int q = (int)(i / nb), s = (int)(i % nb);
    const int p = pc + q, gy = p / G - 2 * h, gx = p % G - 2 * h;
    const int fx = skx[s] + gx, fy = sky[s] + gy;
    float2 v = make_float2(0.f, 0.f);
    if (fx >= -h && fx <= h && fy >= -h && fy <= h) {
      const int j = map[(fy + h) * side + fx + h];
      if (j >= 0) v = cconj(T[(size_t)j * nb + s]);
    }
    T2[i] = v;
  }
}

constexpr int kTccWarps = 8;
constexpr int kImgClips = 4;     // clips per block of the image contraction
constexpr int kAdjClips = 2;     // clips per block of the adjoint contraction

__device__ __forceinline__ double2 warp_sum(double2 v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    v.x += __shfl_xor_sync(0xffffffffu, v.x, off);
    v.y += __shfl_xor_sync(0xffffffffu, v.y, off);
  }
  return v;
}

// Image band boxes. Grid (blocks over the Gh upper-half positions g, clip
// groups of kImgClips). A warp takes one g at a time: lane r sizes band row
// fy_lo + r's overlap with the band shifted by -g (a run, both rows being
// runs), a warp scan turns the runs into one flat list, and the lanes walk
// the list, so every step of the loop is a term of the sum. Terms are summed
// per lane in FP32, then over the warp in FP64 (fixed order).
__global__ void __launch_bounds__(kTccWarps * 32)
k_tcc_image(const float2* __restrict__ T2, const int32_t* __restrict__ rows, const int32_t* __restrict__ skx,
            const int32_t* __restrict__ sky, int nb, int h, int Gh, const float2* __restrict__ mbox, int n_clips,
            float2* __restrict__ bbox) {
  extern __shared__ float2 tcc_sm[];
  const int side = 2 * h + 1, npts = side * side, G = 4 * h + 1, pc = (G * G - 1) / 2;
  const int c0 = blockIdx.y * kImgClips, nc = min(kImgClips, n_clips - c0);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float2* Ms = tcc_sm;                                                  // [c][box position]
  int* r_lo = reinterpret_cast<int*>(Ms + (size_t)kImgClips * npts);   // [side]
  int* r_x0 = r_lo + side;
  int* r_n = r_x0 + side;
  int* w_start = r_n + side + warp * 64;                                // this warp's runs: start, first fx
  int* w_fx = w_start + 32;
  // the clips' mask boxes (contiguous) copied in without waiting per element
  const float2* msrc = mbox + (size_t)c0 * npts;
  for (int i = threadIdx.x; i < nc * npts; i += blockDim.x) cp_async8(Ms + i, msrc + i);
  cp_async_commit();
  for (int y = threadIdx.x; y < side; y += blockDim.x) {
    r_lo[y] = rows[y];
    r_x0[y] = rows[side + y];
    r_n[y] = rows[2 * side + y];
  }
  cp_async_wait_all();
  __syncthreads();
  // positions interleaved over the blocks (q = block + grid x warp): the term
  // count falls off with |g|, so each block gets near and far shifts alike
  for (int q = blockIdx.x + gridDim.x * warp; q < Gh; q += gridDim.x * kTccWarps) {
    const int p = pc + q, gy = p / G - 2 * h, gx = p % G - 2 * h;
    // rows fy with fy and fy + gy both in [-h, h]; at most side <= 32 of them
    const int fy_lo = gy > 0 ? -h : -h - gy, fy_hi = gy > 0 ? h - gy : h;
    int cnt = 0, fx_first = 0;
    if (lane <= fy_hi - fy_lo) {
      const int a = fy_lo + lane + h, b = a + gy;
      const int lo1 = r_x0[a], hi1 = r_x0[a] + r_n[a] - 1;
      const int lo2 = r_x0[b] - gx, hi2 = r_x0[b] + r_n[b] - 1 - gx;
      fx_first = lo1 > lo2 ? lo1 : lo2;
      const int last = hi1 < hi2 ? hi1 : hi2;
      cnt = (r_n[a] > 0 && r_n[b] > 0 && last >= fx_first) ? last - fx_first + 1 : 0;
    }
    int start = cnt;   // inclusive scan, then made exclusive
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const int v = __shfl_up_sync(0xffffffffu, start, off);
      if (lane >= off) start += v;
    }
    const int total = __shfl_sync(0xffffffffu, start, 31);
    start -= cnt;
    w_start[lane] = start;   // nondecreasing: the last run starting at or before k holds term k
    w_fx[lane] = fx_first;
    __syncwarp();
    float2 acc[kImgClips];
#pragma unroll
    for (int c = 0; c < kImgClips; ++c) acc[c] = make_float2(0.f, 0.f);
    const float2* trow = T2 + (size_t)q * nb;
    // the run holding term k: the last r with w_start[r] <= k (runs are at
    // most 2h + 1 <= 31 terms long and k steps by 32, so r moves on by a few
    // runs per step; the scan starts where the lane's previous term was)
    int r = 0;
#pragma unroll 2
    for (int k = lane; k < total; k += 32) {
      while (r < 31 && w_start[r + 1] <= k) ++r;
      const int fy = fy_lo + r, fx = w_fx[r] + (k - w_start[r]);
      const int a = fy + h, b = a + gy;
      const int s = r_lo[a] + fx - r_x0[a];            // sorted index of f
      if (s < 0 || s >= nb) continue;                  // only a blob whose index build failed
      const int pf = a * side + fx + h, pg = b * side + fx + gx + h;   // box positions of f and f + g
      if (pf < 0 || pf >= npts || pg < 0 || pg >= npts) continue;
      const float2 t = __ldg(trow + s);
#pragma unroll
      for (int c = 0; c < kImgClips; ++c)
        acc[c] = cadd(acc[c], cmul(t, cmulc(Ms[c * npts + pg], Ms[c * npts + pf])));   // M(f + g) conj M(f)
    }
    __syncwarp();   // every lane is done with the runs before the next g rewrites them
#pragma unroll
    for (int c = 0; c < kImgClips; ++c) {
      const double2 sum = warp_sum(make_double2((double)acc[c].x, (double)acc[c].y));
      if (lane == 0 && c < nc) {
        float2* dst = bbox + (size_t)(c0 + c) * G * G;
        const float2 v = make_float2((float)sum.x, (float)sum.y);
        dst[p] = v;
        if (q > 0) dst[G * G - 1 - p] = cconj(v);   // B(-g) = conj B(g)
      }
    }
  }
}

// Gradient band boxes. Grid (blocks of kTccWarps band pairs {f, -f}, clip
// groups of kAdjClips). The clips' sensitivity boxes and band-sampled mask
// boxes are staged in shared memory; a warp streams the rows T(f, .) and
// T(-f, .) while its lanes walk f', and writes H(f) = A(f) + conj A(-f) and
// H(-f) = conj H(f). Box positions off the band are zeroed by the blocks.
__global__ void __launch_bounds__(kTccWarps * 32)
k_tcc_adjoint(const float2* __restrict__ T, const int32_t* __restrict__ map, const int32_t* __restrict__ skx,
              const int32_t* __restrict__ sky, int nb, int h, const float2* __restrict__ mbox,
              const float2* __restrict__ gbox, int n_clips, float2* __restrict__ hbox) {
  extern __shared__ float2 tcc_sm[];
  const int side = 2 * h + 1, npts = side * side, G = 4 * h + 1, GG = G * G;
  const int c0 = blockIdx.y * kAdjClips, nc = min(kAdjClips, n_clips - c0);
  float2* Gs = tcc_sm;                                   // [c][G^2]
  float2* Ms = Gs + (size_t)kAdjClips * GG;              // [c][box position]
  // per band point f': uy G + ux (the sensitivity offset) and its mask box
  // position, (ux, uy) clamped to the box so every index stays inside the
  // staged boxes even for a blob whose index build failed (then the build's
  // status word reports it)
  int* s_off = reinterpret_cast<int*>(Ms + (size_t)kAdjClips * npts);
  int* s_pm = s_off + nb;
  // the clips' sensitivity and mask boxes (contiguous) copied in without
  // waiting per element
  const float2* gsrc = gbox + (size_t)c0 * GG;
  for (int i = threadIdx.x; i < nc * GG; i += blockDim.x) cp_async8(Gs + i, gsrc + i);
  const float2* msrc = mbox + (size_t)c0 * npts;
  for (int i = threadIdx.x; i < nc * npts; i += blockDim.x) cp_async8(Ms + i, msrc + i);
  cp_async_commit();
  for (int s = threadIdx.x; s < nb; s += blockDim.x) {
    const int ux = min(max(skx[s], -h), h), uy = min(max(sky[s], -h), h);
    s_off[s] = uy * G + ux;
    s_pm[s] = (uy + h) * side + ux + h;
  }
  // positions of the output box off the band are zero
  for (int pp = blockIdx.x * blockDim.x + threadIdx.x; pp < npts; pp += gridDim.x * blockDim.x)
    if (map[pp] < 0)
      for (int c = 0; c < nc; ++c) hbox[(size_t)(c0 + c) * npts + pp] = make_float2(0.f, 0.f);
  cp_async_wait_all();
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int s = blockIdx.x * kTccWarps + warp, sn = nb - 1 - s;   // f and -f
  if (s > sn) return;
  const int fx = skx[s], fy = sky[s];
  if (fx < -h || fx > h || fy < -h || fy > h) return;   // only a blob whose index build failed
  const float2* t1 = T + (size_t)s * nb;
  const float2* t2 = T + (size_t)sn * nb;
  float2 a1[kAdjClips], a2[kAdjClips];
#pragma unroll
  for (int c = 0; c < kAdjClips; ++c) a1[c] = a2[c] = make_float2(0.f, 0.f);
  const int base1 = (fy + 2 * h) * G + (fx + 2 * h), base2 = (-fy + 2 * h) * G + (-fx + 2 * h);
#pragma unroll 8
  for (int j = lane; j < nb; j += 32) {
    const int off = s_off[j], pm = s_pm[j];                       // pm: box position of f'
    const int d1 = base1 - off, d2 = base2 - off;                 // f - f', -f - f'
    const float2 w1 = __ldg(t1 + j), w2 = __ldg(t2 + j);
#pragma unroll
    for (int c = 0; c < kAdjClips; ++c) {
      const float2 m = Ms[c * npts + pm];
      a1[c] = cadd(a1[c], cmul(w1, cmul(m, Gs[c * GG + d1])));
      a2[c] = cadd(a2[c], cmul(w2, cmul(m, Gs[c * GG + d2])));
    }
  }
#pragma unroll
  for (int c = 0; c < kAdjClips; ++c) {
    const double2 u = warp_sum(make_double2((double)a1[c].x, (double)a1[c].y));
    const double2 v = warp_sum(make_double2((double)a2[c].x, (double)a2[c].y));
    if (lane == 0 && c < nc) {
      const float2 hf = make_float2((float)(u.x + v.x), (float)(u.y - v.y));   // A(f) + conj A(-f)
      float2* dst = hbox + (size_t)(c0 + c) * npts;
      dst[(fy + h) * side + fx + h] = hf;
      if (sn != s) dst[(-fy + h) * side + (-fx + h)] = cconj(hf);
    }
  }
}

size_t img_smem(int nb, int h) {
  const int side = 2 * h + 1;
  (void)nb;
  return (size_t)kImgClips * side * side * 8 + (size_t)(3 * side + kTccWarps * 64) * 4;
}
size_t adj_smem(int nb, int h) {
  const int side = 2 * h + 1, G = 4 * h + 1;
  return (size_t)kAdjClips * G * G * 8 + (size_t)kAdjClips * side * side * 8 + (size_t)2 * nb * 4;
}

int tcc_check(int nb, int h, size_t* need) {
  if (nb < 1 || h < 0 || nb > (2 * h + 1) * (2 * h + 1)) return LITHO_E_SIZE;
  if (h > kTccHMax) return LITHO_E_UNSUPPORTED;
  const TccLayout l = tcc_layout(nb, h);
  if (l.total > kTccMaxBytes) return LITHO_E_UNSUPPORTED;
  if (img_smem(nb, h) > 200 * 1024 || adj_smem(nb, h) > 200 * 1024) return LITHO_E_UNSUPPORTED;
  if (need) *need = (size_t)l.total;
  return LITHO_OK;
}

}  // namespace
}  // namespace litho

using namespace litho;

extern "C" int litho_socs_tcc_bytes(int n_band, int h, size_t* bytes) {
  if (!bytes) return LITHO_E_NULL;
  return tcc_check(n_band, h, bytes);
}

extern "C" int litho_socs_tcc_build(const void* phi_dev, const double* lam_dev, int K, const int32_t* band_kx_dev,
                                    const int32_t* band_ky_dev, int n_band, int h, void* tcc_dev, size_t tcc_bytes,
                                    int* status_dev, cudaStream_t s) {
  if (!phi_dev || !lam_dev || !band_kx_dev || !band_ky_dev || !tcc_dev || !status_dev) return LITHO_E_NULL;
  if (K < 1) return LITHO_E_SIZE;
  size_t need = 0;
  const int st = tcc_check(n_band, h, &need);
  if (st) return st;
  if (tcc_bytes < need) return LITHO_E_WORKSPACE;
  if (((uintptr_t)tcc_dev & 15) || ((uintptr_t)phi_dev & 15)) return LITHO_E_ALIGN;
  const TccLayout l = tcc_layout(n_band, h);
  char* w = static_cast<char*>(tcc_dev);
  int32_t* map = reinterpret_cast<int32_t*>(w + l.map);
  int32_t* perm = reinterpret_cast<int32_t*>(w + l.perm);
  int32_t* skx = reinterpret_cast<int32_t*>(w + l.skx);
  int32_t* sky = reinterpret_cast<int32_t*>(w + l.sky);
  int32_t* rows = reinterpret_cast<int32_t*>(w + l.rows);
  float2* T = reinterpret_cast<float2*>(w + l.T);
  float2* T2 = reinterpret_cast<float2*>(w + l.T2);
  cudaError_t e = cudaMemsetAsync(status_dev, 0, sizeof(int), s);
  if (e != cudaSuccess) return (int)e;
  k_tcc_index<<<1, 1024, 0, s>>>(band_kx_dev, band_ky_dev, n_band, h, map, perm, skx, sky, rows, status_dev);
  const int64_t nT = (int64_t)n_band * n_band, nT2 = (int64_t)l.Gh * n_band;
  k_tcc_T<<<(int)((nT + 255) / 256 < 8192 ? (nT + 255) / 256 : 8192), 256, 0, s>>>(
      static_cast<const double2*>(phi_dev), lam_dev, K, n_band, perm, T);
  k_tcc_T2<<<(int)((nT2 + 255) / 256 < 8192 ? (nT2 + 255) / 256 : 8192), 256, 0, s>>>(T, map, skx, sky, n_band, h,
                                                                                      l.Gh, T2);
  e = cudaGetLastError();
  return e == cudaSuccess ? LITHO_OK : (int)e;
}

extern "C" int litho_socs_tcc_image(const void* tcc_dev, int n_band, int h, const void* mask_box_dev, int n_clips,
                                    void* image_box_out_dev, cudaStream_t s) {
  if (!tcc_dev || !mask_box_dev || !image_box_out_dev) return LITHO_E_NULL;
  if (n_clips < 1) return LITHO_E_SIZE;
  const int st = tcc_check(n_band, h, nullptr);
  if (st) return st;
  const TccLayout l = tcc_layout(n_band, h);
  const char* w = static_cast<const char*>(tcc_dev);
  const size_t sm = img_smem(n_band, h);
  cudaFuncSetAttribute(k_tcc_image, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  const int groups = (n_clips + kImgClips - 1) / kImgClips;
  const int bx = (l.Gh + kTccWarps - 1) / kTccWarps;
  k_tcc_image<<<dim3(bx, groups), kTccWarps * 32, sm, s>>>(
      reinterpret_cast<const float2*>(w + l.T2), reinterpret_cast<const int32_t*>(w + l.rows),
      reinterpret_cast<const int32_t*>(w + l.skx), reinterpret_cast<const int32_t*>(w + l.sky), n_band, h, l.Gh,
      static_cast<const float2*>(mask_box_dev), n_clips, static_cast<float2*>(image_box_out_dev));
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? LITHO_OK : (int)e;
}

extern "C" int litho_socs_tcc_adjoint(const void* tcc_dev, int n_band, int h, const void* mask_box_dev,
                                      const void* sens_box_dev, int n_clips, void* grad_box_out_dev, cudaStream_t s) {
  if (!tcc_dev || !mask_box_dev || !sens_box_dev || !grad_box_out_dev) return LITHO_E_NULL;
  if (n_clips < 1) return LITHO_E_SIZE;
  const int st = tcc_check(n_band, h, nullptr);
  if (st) return st;
  const TccLayout l = tcc_layout(n_band, h);
  const char* w = static_cast<const char*>(tcc_dev);
  const size_t sm = adj_smem(n_band, h);
  cudaFuncSetAttribute(k_tcc_adjoint, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  const int pairs = (n_band + 1) / 2;
  const int bx = (pairs + kTccWarps - 1) / kTccWarps;
  const int groups = (n_clips + kAdjClips - 1) / kAdjClips;
  k_tcc_adjoint<<<dim3(bx, groups), kTccWarps * 32, sm, s>>>(
      reinterpret_cast<const float2*>(w + l.T), reinterpret_cast<const int32_t*>(w + l.map),
      reinterpret_cast<const int32_t*>(w + l.skx), reinterpret_cast<const int32_t*>(w + l.sky), n_band, h,
      static_cast<const float2*>(mask_box_dev), static_cast<const float2*>(sens_box_dev), n_clips,
      static_cast<float2*>(grad_box_out_dev));
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? LITHO_OK : (int)e;
}
