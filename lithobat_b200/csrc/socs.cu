// SOCS (Hopkins) decomposition of an optical state, on the GPU.
//
// Reference: expose/hopkins.py:SOCSKernels.build (:103-198). There, with
// A[s, f] = sqrt(w_s) P(f - f_s) on the band |f| <= 2 NA / lambda,
//     TCC = A^T conj(A)  (n_band x n_band),  eigh(TCC) in FP64,
//     kernels = leading eigenvectors, weights = their eigenvalues.
// Here the same eigenpairs come from the dual (Gram) form:
//     C = conj(A),  TCC = C^H C,  G = C C^H = conj(A) A^T  (S x S),
//     G u = lambda u  =>  phi = C^H u / sqrt(lambda) = A^T u / sqrt(lambda)
// which is what makes the EUV band (n_band ~ 1e5) tractable: G is S x S.
//
//   k_socs_pupil_matrix : A in FP64 (aperture decided on the host with the
//                         reference's own hypot test)
//   k_gram_umma         : G on the 5th-generation tensor cores (tcgen05.mma
//                         kind::tf32, accumulator in TMEM), operands split
//                         into TF32 hi + lo and combined as hi.hi + hi.lo +
//                         lo.hi; K split over blocks, partials in FP32
//   k_gram_reduce       : FP64 sum of the partials -> G
//   k_jacobi_herm       : FP64 cyclic Jacobi on the Hermitian G
//   k_socs_phi          : phi_j = A^T u_j (FP64) and lambda_j = |A^T u_j|^2,
//                         the Rayleigh quotient with the exact A, so the
//                         weights carry FP64 accuracy whatever the Gram's.
#include "common.cuh"
#include "tcgen05.cuh"
#include "pupil.cuh"

namespace litho {

// ---------------------------------------------------------------------------
// A[s][b] = sqrt(w_s) exp(i W), zero where the host's aperture test failed.
// Layout: Are/Aim [S][ld], ld >= nb, padding zero.
// ---------------------------------------------------------------------------
__global__ void k_socs_pupil_matrix(const double* __restrict__ fsx, const double* __restrict__ fsy,
                                    const double* __restrict__ w, int S, const int32_t* __restrict__ bkx,
                                    const int32_t* __restrict__ bky, int nb, int ld,
                                    const uint8_t* __restrict__ inside, const LithoPupil* __restrict__ pupil,
                                    double val, double* __restrict__ Are, double* __restrict__ Aim) {
  const LithoPupil P = *pupil;
  const double kmax = P.NA / P.wavelength;
  const long long total = (long long)S * ld;
  for (long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x; id < total;
       id += (long long)gridDim.x * blockDim.x) {
    const int s = (int)(id / ld), b = (int)(id % ld);
    double re = 0.0, im = 0.0;
    if (b < nb && inside[(size_t)s * nb + b]) {
      const double dx = (double)bkx[b] * val - fsx[s];
      const double dy = (double)bky[b] * val - fsy[s];
      const double r = hypot(dx, dy);
      const double rho = r / kmax;
      double cp = 1.0, sp = 0.0;
      if (r > 0.0) {
        cp = dx / r;
        sp = dy / r;
      }
      const double W = pupil_phase(P, rho, cp, sp);
      double sW, cW;
      sincos(W, &sW, &cW);
      const double a = sqrt(w[s]);
      re = a * cW;
      im = a * sW;
    }
    Are[id] = re;
    Aim[id] = im;
  }
}

// ---------------------------------------------------------------------------
// Gram on tcgen05. Real formulation with X = [Are | Aim] (S x 2ld) and
// Y = [Aim | -Are]: Re G = X X^T, Im G = X Y^T, i.e. one GEMM
//     D (S x 2S) = X (S x K) . [X; Y]^T,  K = 2 ld.
// One block: a 128 x 256 output tile (M = 128 rows of X, N = 256 rows of
// [X; Y]) over a range of K; 128 threads stage each 32-wide K slab into
// shared memory in the canonical K-major, no-swizzle UMMA layout (8-row x
// 16-byte core matrices; 16-byte K chunks LBO apart, 8-row groups SBO apart)
// as TF32 hi and lo planes; one elected thread issues the MMAs.
// ---------------------------------------------------------------------------
constexpr int kGM = 128, kGN = 256, kGK = 32;
constexpr int kGThreads = 128;
constexpr uint32_t kGAtile = kGM * kGK * 4;  // bytes of one A plane (16 KiB)
constexpr uint32_t kGBtile = kGN * kGK * 4;  // bytes of one B plane (32 KiB)


// Value of row `row` (of the 2S rows of [X; Y]) at column k (< 2 ld).
__device__ __forceinline__ double gram_operand(const double* Are, const double* Aim, int S, int ld, int row,
                                               int k) {
  const bool y = row >= S;
  const int s = y ? row - S : row;
  if (s >= S) return 0.0;
  const size_t base = (size_t)s * ld;
  if (!y) return k < ld ? Are[base + k] : Aim[base + (k - ld)];
  return k < ld ? Aim[base + k] : -Are[base + (k - ld)];
}

__global__ void __launch_bounds__(kGThreads)
k_gram_umma(const double* __restrict__ Are, const double* __restrict__ Aim, int S, int ld, int k_tiles_per_split,
            float* __restrict__ partial, int ldp, int* __restrict__ status) {
  extern __shared__ __align__(1024) unsigned char gsm[];
  __shared__ uint64_t s_mbar;
  __shared__ uint32_t s_tmem;
  __shared__ int s_fail;
  unsigned char* a_hi = gsm;
  unsigned char* a_lo = gsm + kGAtile;
  unsigned char* b_hi = gsm + 2 * kGAtile;
  unsigned char* b_lo = gsm + 2 * kGAtile + kGBtile;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int mt = blockIdx.x, nt = blockIdx.y, ks = blockIdx.z;
  const int K = 2 * ld;
  const int k_tiles = (K + kGK - 1) / kGK;
  const int kt0 = ks * k_tiles_per_split;
  const int kt1 = min(k_tiles, kt0 + k_tiles_per_split);

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                 "r"(kGN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (threadIdx.x == 0) {
    s_fail = 0;
    mbar_init(&s_mbar, 1);
    fence_mbar_init();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s_tmem;
  // instruction descriptor: D f32, A/B tf32, both K-major, N = 256, M = 128
  const uint32_t idesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(kGN >> 3) << 17) |
                         ((uint32_t)(kGM >> 4) << 24);
  uint32_t phase = 0;
  bool issued = false;
  for (int kt = kt0; kt < kt1; ++kt) {
    // stage the slab: element (row, kk) at chunk kk/4, row, word kk%4
    for (int id = threadIdx.x; id < kGM * kGK; id += kGThreads) {
      const int row = id / kGK, kk = id % kGK, k = kt * kGK + kk;
      const int s = mt * kGM + row;
      const double v = (s < S && k < K) ? gram_operand(Are, Aim, S, ld, s, k) : 0.0;
      const float f = (float)v;
      const uint32_t hi = to_tf32(f);
      const uint32_t lo = to_tf32(f - __uint_as_float(hi));
      const uint32_t off = (uint32_t)((kk >> 2) * (kGM * 16) + row * 16 + (kk & 3) * 4);
      *reinterpret_cast<uint32_t*>(a_hi + off) = hi;
      *reinterpret_cast<uint32_t*>(a_lo + off) = lo;
    }
    for (int id = threadIdx.x; id < kGN * kGK; id += kGThreads) {
      const int row = id / kGK, kk = id % kGK, k = kt * kGK + kk;
      const int r = nt * kGN + row;
      const double v = (r < 2 * S && k < K) ? gram_operand(Are, Aim, S, ld, r, k) : 0.0;
      const float f = (float)v;
      const uint32_t hi = to_tf32(f);
      const uint32_t lo = to_tf32(f - __uint_as_float(hi));
      const uint32_t off = (uint32_t)((kk >> 2) * (kGN * 16) + row * 16 + (kk & 3) * 4);
      *reinterpret_cast<uint32_t*>(b_hi + off) = hi;
      *reinterpret_cast<uint32_t*>(b_lo + off) = lo;
    }
    fence_proxy_async();
    __syncthreads();
    tc_fence_after();
    if (threadIdx.x == 0) {
#pragma unroll
      for (int step = 0; step < kGK / 8; ++step) {
        const uint32_t ao = step * 2 * (kGM * 16), bo = step * 2 * (kGN * 16);
        const uint64_t ah = umma_desc(smem_u32(a_hi) + ao, kGM * 16, 128);
        const uint64_t al = umma_desc(smem_u32(a_lo) + ao, kGM * 16, 128);
        const uint64_t bh = umma_desc(smem_u32(b_hi) + bo, kGN * 16, 128);
        const uint64_t bl = umma_desc(smem_u32(b_lo) + bo, kGN * 16, 128);
        umma_tf32(tmem, ah, bh, idesc, (kt > kt0 || step > 0) ? 1u : 0u);
        umma_tf32(tmem, ah, bl, idesc, 1u);
        umma_tf32(tmem, al, bh, idesc, 1u);
      }
      umma_commit(&s_mbar);
    }
    issued = true;
    if (!mbar_wait(&s_mbar, phase)) atomicExch(&s_fail, 1);
    phase ^= 1;
    tc_fence_after();
    __syncthreads();
    if (s_fail) break;
  }
  if (!s_fail && issued) {
    // TMEM -> registers -> global: warp w owns accumulator rows 32w .. 32w+31
    const int row = mt * kGM + warp * 32 + lane;
    float* dst = partial + ((size_t)ks * ldp + row) * (size_t)(2 * ldp);
    for (int c0 = 0; c0 < kGN; c0 += 16) {
      uint32_t r[16];
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
          "%14, %15}, [%16];"
          : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
            "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
          : "r"(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      const int col0 = nt * kGN + c0;
      if (row < ldp) {
#pragma unroll
        for (int i = 0; i < 16; ++i)
          if (col0 + i < 2 * ldp) dst[col0 + i] = __uint_as_float(r[i]);
      }
    }
  }
  if (s_fail && threadIdx.x == 0) {
    // let the MMAs of the last commit (parity phase ^ 1: the loop flipped
    // phase after waiting on it) land before TMEM is released; returns at
    // once if that phase already completed
    if (issued) mbar_wait_drain(&s_mbar, phase ^ 1u);
    atomicExch(status, LITHO_E_TIMEOUT);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kGN));
}

// G[s][t] = sum over splits of the partials, in FP64 (split order fixed).
// partial layout: [split][ldp rows][2 ldp cols]: cols [0, ldp) real part of
// column t, cols [ldp, 2 ldp) hold rows of Y, i.e. Im G at col ldp + t... see
// the host: [X; Y] rows are indexed 0..2S-1, so Im G[s][t] is at col S + t.
__global__ void k_gram_reduce(const float* __restrict__ partial, int splits, int ldp, int S, double2* __restrict__ G,
                              int ldg) {
  for (int id = blockIdx.x * blockDim.x + threadIdx.x; id < ldg * ldg; id += gridDim.x * blockDim.x) {
    const int s = id / ldg, t = id % ldg;
    double re = 0.0, im = 0.0;
    if (s < S && t < S) {
      for (int k = 0; k < splits; ++k) {
        const float* p = partial + ((size_t)k * ldp + s) * (size_t)(2 * ldp);
        re += (double)p[t];
        im += (double)p[S + t];
      }
    }
    G[id] = make_double2(re, im);
  }
}

// FP64 reference Gram on CUDA cores (for checking the tensor-core path).
__global__ void k_gram_fp64(const double* __restrict__ Are, const double* __restrict__ Aim, int S, int ld,
                            double2* __restrict__ G, int ldg) {
  for (int id = blockIdx.x * blockDim.x + threadIdx.x; id < ldg * ldg; id += gridDim.x * blockDim.x) {
    const int s = id / ldg, t = id % ldg;
    double re = 0.0, im = 0.0;
    if (s < S && t < S) {
      const double* ar = Are + (size_t)s * ld;
      const double* ai = Aim + (size_t)s * ld;
      const double* br = Are + (size_t)t * ld;
      const double* bi = Aim + (size_t)t * ld;
      for (int b = 0; b < ld; ++b) {  // conj(A[s][b]) * A[t][b]
        re += ar[b] * br[b] + ai[b] * bi[b];
        im += ar[b] * bi[b] - ai[b] * br[b];
      }
    }
    G[id] = make_double2(re, im);
  }
}

// ---------------------------------------------------------------------------
// Cyclic Jacobi for a Hermitian n x n matrix (n even), one block. Each round
// rotates n/2 disjoint (p, q) pairs (round-robin order), applied as H <- H R
// (columns) then H <- R^H H (rows), V <- V R. R on (p, q) with
// c = H[p][q] = |c| u: R = [[cs, sn], [-sn conj(u), cs conj(u)]],
// t = sgn(tau) / (|tau| + sqrt(1 + tau^2)), tau = (H[q][q] - H[p][p]) / (2 |c|).
// ---------------------------------------------------------------------------
__device__ __forceinline__ double2 zmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

__global__ void __launch_bounds__(1024)
k_jacobi_herm(double2* __restrict__ H, double2* __restrict__ V, int n, int max_sweeps, double tol,
              double* __restrict__ evals, int* __restrict__ sweeps_out) {
  extern __shared__ double jsm[];
  int* rp = reinterpret_cast<int*>(jsm);
  int* rq = rp + n / 2;
  double* rcs = reinterpret_cast<double*>(rq + n / 2);  // 8 * (n/2) bytes in: 8-byte aligned
  double* rsn = rcs + n / 2;
  double* rur = rsn + n / 2;
  double* rui = rur + n / 2;
  __shared__ double red[32];
  __shared__ int s_done;
  const int half = n / 2;
  for (int i = threadIdx.x; i < n * n; i += blockDim.x) V[i] = make_double2((i / n) == (i % n) ? 1.0 : 0.0, 0.0);
  if (threadIdx.x == 0) s_done = 0;
  __syncthreads();
  int sweep = 0;
  for (; sweep < max_sweeps; ++sweep) {
    // convergence: off-diagonal vs diagonal energy
    double off = 0.0, dia = 0.0;
    for (int i = threadIdx.x; i < n * n; i += blockDim.x) {
      const double2 h = H[i];
      const double m = h.x * h.x + h.y * h.y;
      if (i / n == i % n) dia += m; else off += m;
    }
    for (int o = 16; o > 0; o >>= 1) {
      off += __shfl_xor_sync(0xffffffffu, off, o);
      dia += __shfl_xor_sync(0xffffffffu, dia, o);
    }
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = off;
    __syncthreads();
    if (threadIdx.x == 0) {
      double s = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
      red[0] = s;
    }
    __syncthreads();
    const double off_tot = red[0];
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = dia;
    __syncthreads();
    if (threadIdx.x == 0) {
      double s = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
      s_done = off_tot <= tol * tol * s ? 1 : 0;
    }
    __syncthreads();
    if (s_done) break;
    for (int round = 0; round < n - 1; ++round) {
      for (int i = threadIdx.x; i < half; i += blockDim.x) {
        const int a = (i == 0) ? 0 : ((i - 1 + round) % (n - 1)) + 1;
        const int b = ((n - 1 - i - 1 + round) % (n - 1)) + 1;
        const int p = a < b ? a : b, q = a < b ? b : a;
        const double2 c = H[(size_t)p * n + q];
        // |c| by hypot: once converged the couplings fall far below 1e-154,
        // where c.x^2 + c.y^2 underflows and c / |c| would stop being a unit
        // phase (and with degenerate diagonals tau = 0 rotates by 45 degrees
        // whatever |c| is). Couplings below round-off are dropped instead.
        const double ac = hypot(c.x, c.y);
        const double hp = H[(size_t)p * n + p].x, hq = H[(size_t)q * n + q].x;
        double cs = 1.0, sn = 0.0, ur = 1.0, ui = 0.0;
        if (ac > 1e-18 * (fabs(hp) + fabs(hq)) && ac > 1e-300) {
          const double tau = (hq - hp) / (2.0 * ac);
          const double t = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
          cs = 1.0 / sqrt(1.0 + t * t);
          sn = t * cs;
          ur = c.x / ac;
          ui = c.y / ac;
        }
        rp[i] = p; rq[i] = q; rcs[i] = cs; rsn[i] = sn; rur[i] = ur; rui[i] = ui;
      }
      __syncthreads();
      // columns: H <- H R, V <- V R   (item = (row r, pair i), pairs fastest)
      for (int id = threadIdx.x; id < n * half; id += blockDim.x) {
        const int r = id / half, i = id % half;
        const int p = rp[i], q = rq[i];
        const double cs = rcs[i], sn = rsn[i];
        const double2 uc = make_double2(rur[i], -rui[i]);  // conj(u)
        double2* h = H + (size_t)r * n;
        const double2 hp = h[p], hq = h[q];
        const double2 hqu = zmul(hq, uc);
        h[p] = make_double2(cs * hp.x - sn * hqu.x, cs * hp.y - sn * hqu.y);
        h[q] = make_double2(sn * hp.x + cs * hqu.x, sn * hp.y + cs * hqu.y);
        double2* v = V + (size_t)r * n;
        const double2 vp = v[p], vq = v[q];
        const double2 vqu = zmul(vq, uc);
        v[p] = make_double2(cs * vp.x - sn * vqu.x, cs * vp.y - sn * vqu.y);
        v[q] = make_double2(sn * vp.x + cs * vqu.x, sn * vp.y + cs * vqu.y);
      }
      __syncthreads();
      // rows: H <- R^H H   (item = (pair i, column r), columns fastest)
      for (int id = threadIdx.x; id < n * half; id += blockDim.x) {
        const int i = id / n, r = id % n;
        const int p = rp[i], q = rq[i];
        const double cs = rcs[i], sn = rsn[i];
        const double2 u = make_double2(rur[i], rui[i]);
        const double2 hp = H[(size_t)p * n + r], hq = H[(size_t)q * n + r];
        const double2 hqu = zmul(hq, u);
        H[(size_t)p * n + r] = make_double2(cs * hp.x - sn * hqu.x, cs * hp.y - sn * hqu.y);
        H[(size_t)q * n + r] = make_double2(sn * hp.x + cs * hqu.x, sn * hp.y + cs * hqu.y);
      }
      __syncthreads();
      for (int i = threadIdx.x; i < half; i += blockDim.x) {
        const int p = rp[i], q = rq[i];
        H[(size_t)p * n + q] = make_double2(0.0, 0.0);
        H[(size_t)q * n + p] = make_double2(0.0, 0.0);
        H[(size_t)p * n + p].y = 0.0;
        H[(size_t)q * n + q].y = 0.0;
      }
      __syncthreads();
    }
  }
  for (int i = threadIdx.x; i < n; i += blockDim.x) evals[i] = H[(size_t)i * n + i].x;
  if (threadIdx.x == 0) *sweeps_out = sweep;
}

// phi[j][b] = sum_s A[s][b] V[s][j]  (FP64), j < S.
__global__ void k_socs_phi(const double* __restrict__ Are, const double* __restrict__ Aim, int S, int ld, int nb,
                           const double2* __restrict__ V, int ldv, double2* __restrict__ phi) {
  const long long total = (long long)S * nb;
  for (long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x; id < total;
       id += (long long)gridDim.x * blockDim.x) {
    const int j = (int)(id / nb), b = (int)(id % nb);
    double re = 0.0, im = 0.0;
    for (int s = 0; s < S; ++s) {
      const double ar = Are[(size_t)s * ld + b], ai = Aim[(size_t)s * ld + b];
      const double2 v = V[(size_t)s * ldv + j];
      re += ar * v.x - ai * v.y;
      im += ar * v.y + ai * v.x;
    }
    phi[id] = make_double2(re, im);
  }
}

// lambda[j] = sum_b |phi[j][b]|^2, one block per j, fixed-order tree.
__global__ void k_socs_norms(const double2* __restrict__ phi, int nb, double* __restrict__ lam) {
  __shared__ double red[32];
  const int j = blockIdx.x;
  double s = 0.0;
  for (int b = threadIdx.x; b < nb; b += blockDim.x) {
    const double2 v = phi[(size_t)j * nb + b];
    s += v.x * v.x + v.y * v.y;
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    lam[j] = t;
  }
}

}  // namespace litho

// ---------------------------------------------------------------------------
// host entry
// ---------------------------------------------------------------------------
using namespace litho;

struct SocsLayout {
  int ld, ldg, ldp, mt, nt, splits, kt_per;
  int64_t status, Are, Aim, partial, G, V, evals, sweeps, phi, lam, total;
};

static SocsLayout socs_layout(int S, int nb, int num_sms) {
  SocsLayout l{};
  l.ld = (nb + 15) / 16 * 16;
  l.ldg = S + (S & 1);                   // even for the Jacobi round-robin
  l.mt = (S + kGM - 1) / kGM;
  l.nt = (2 * S + kGN - 1) / kGN;
  l.ldp = l.mt * kGM;                    // rows of a partial (>= S)
  if (l.ldp < (l.nt * kGN + 1) / 2) l.ldp = (l.nt * kGN + 1) / 2;
  const int k_tiles = (2 * l.ld + kGK - 1) / kGK;
  int splits = num_sms / (l.mt * l.nt);
  if (splits < 1) splits = 1;
  if (splits > k_tiles) splits = k_tiles;
  l.kt_per = (k_tiles + splits - 1) / splits;
  l.splits = (k_tiles + l.kt_per - 1) / l.kt_per;
  int64_t off = 0;
  l.status = off;  off = align16(off + 16);
  l.Are = off;     off = align16(off + (int64_t)S * l.ld * 8);
  l.Aim = off;     off = align16(off + (int64_t)S * l.ld * 8);
  l.partial = off; off = align16(off + (int64_t)l.splits * l.ldp * 2 * l.ldp * 4);
  l.G = off;       off = align16(off + (int64_t)l.ldg * l.ldg * 16);
  l.V = off;       off = align16(off + (int64_t)l.ldg * l.ldg * 16);
  l.evals = off;   off = align16(off + (int64_t)l.ldg * 8);
  l.sweeps = off;  off = align16(off + 16);
  l.phi = off;     off = align16(off + (int64_t)S * nb * 16);
  l.lam = off;     off = align16(off + (int64_t)S * 8);
  l.total = off;
  return l;
}

static int sms_now() {
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms > 0 ? sms : 148;
}

extern "C" int litho_socs_workspace(int n_source, int n_band, size_t* bytes) {
  if (!bytes) return LITHO_E_NULL;
  if (n_source < 1 || n_source > 2048 || n_band < 1) return LITHO_E_SIZE;
  *bytes = (size_t)socs_layout(n_source, n_band, sms_now()).total;
  return LITHO_OK;
}

extern "C" int litho_socs_build(const LithoPupil* pupil_dev, const double* fsx_dev, const double* fsy_dev,
                                const double* w_dev, int n_source, const int32_t* band_kx_dev,
                                const int32_t* band_ky_dev, int n_band, const uint8_t* inside_dev, int n,
                                double pixel_size, int gram_mode, double2* phi_out_dev, double* lambda_out_dev,
                                double2* gram_out_dev, void* ws, size_t ws_bytes, cudaStream_t s) {
  if (!pupil_dev || !fsx_dev || !fsy_dev || !w_dev || !band_kx_dev || !band_ky_dev || !inside_dev ||
      !phi_out_dev || !lambda_out_dev || !ws)
    return LITHO_E_NULL;
  if (n_source < 1 || n_source > 2048 || n_band < 1 || n < 2 || !(pixel_size > 0.0)) return LITHO_E_SIZE;
  if (gram_mode != 0 && gram_mode != 1) return LITHO_E_SIZE;
  if ((uintptr_t)ws & 15) return LITHO_E_ALIGN;
  const int S = n_source, nb = n_band;
  const SocsLayout l = socs_layout(S, nb, sms_now());
  if ((int64_t)ws_bytes < l.total) return LITHO_E_WORKSPACE;
  char* w = static_cast<char*>(ws);
  int* status = reinterpret_cast<int*>(w + l.status);
  double* Are = reinterpret_cast<double*>(w + l.Are);
  double* Aim = reinterpret_cast<double*>(w + l.Aim);
  float* partial = reinterpret_cast<float*>(w + l.partial);
  double2* G = reinterpret_cast<double2*>(w + l.G);
  double2* V = reinterpret_cast<double2*>(w + l.V);
  double* evals = reinterpret_cast<double*>(w + l.evals);
  int* sweeps = reinterpret_cast<int*>(w + l.sweeps);
  cudaError_t e;
  if ((e = cudaMemsetAsync(status, 0, sizeof(int), s)) != cudaSuccess) return (int)e;
  const double val = 1.0 / ((double)n * pixel_size);
  const long long na = (long long)S * l.ld;
  k_socs_pupil_matrix<<<(unsigned)((na + 255) / 256 < 4096 ? (na + 255) / 256 : 4096), 256, 0, s>>>(
      fsx_dev, fsy_dev, w_dev, S, band_kx_dev, band_ky_dev, nb, l.ld, inside_dev, pupil_dev, val, Are, Aim);
  if ((e = cudaGetLastError()) != cudaSuccess) return (int)e;
  const int gblocks = (l.ldg * l.ldg + 255) / 256;
  if (gram_mode == 0) {
    const size_t sm = 2 * kGAtile + 2 * kGBtile;
    cudaFuncSetAttribute(k_gram_umma, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    dim3 grid(l.mt, l.nt, l.splits);
    k_gram_umma<<<grid, kGThreads, sm, s>>>(Are, Aim, S, l.ld, l.kt_per, partial, l.ldp, status);
    if ((e = cudaGetLastError()) != cudaSuccess) return (int)e;
    k_gram_reduce<<<gblocks, 256, 0, s>>>(partial, l.splits, l.ldp, S, G, l.ldg);
  } else {
    k_gram_fp64<<<gblocks, 256, 0, s>>>(Are, Aim, S, l.ld, G, l.ldg);
  }
  if ((e = cudaGetLastError()) != cudaSuccess) return (int)e;
  if (gram_out_dev)
    if ((e = cudaMemcpyAsync(gram_out_dev, G, (size_t)l.ldg * l.ldg * 16, cudaMemcpyDeviceToDevice, s)) !=
        cudaSuccess)
      return (int)e;
  const int half = l.ldg / 2;
  const size_t jsm = (size_t)half * 2 * sizeof(int) + (size_t)half * 4 * sizeof(double);
  k_jacobi_herm<<<1, 1024, jsm, s>>>(G, V, l.ldg, 40, 1e-14, evals, sweeps);
  if ((e = cudaGetLastError()) != cudaSuccess) return (int)e;
  const long long nphi = (long long)S * nb;
  k_socs_phi<<<(unsigned)((nphi + 255) / 256 < 8192 ? (nphi + 255) / 256 : 8192), 256, 0, s>>>(
      Are, Aim, S, l.ld, nb, V, l.ldg, phi_out_dev);
  if ((e = cudaGetLastError()) != cudaSuccess) return (int)e;
  k_socs_norms<<<S, 256, 0, s>>>(phi_out_dev, nb, lambda_out_dev);
  if ((e = cudaGetLastError()) != cudaSuccess) return (int)e;
  return LITHO_OK;
}

extern "C" int litho_socs_status(int n_source, int n_band, const void* ws, int* sweeps, cudaStream_t s) {
  if (!ws) return LITHO_E_NULL;
  const SocsLayout l = socs_layout(n_source, n_band, sms_now());
  int h[2] = {0, 0};
  cudaError_t e = cudaMemcpyAsync(&h[0], static_cast<const char*>(ws) + l.status, sizeof(int),
                                  cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&h[1], static_cast<const char*>(ws) + l.sweeps, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return (int)e;
  if (sweeps) *sweeps = h[1];
  return h[0];
}

extern "C" int litho_socs_debug(int n_source, int n_band, const void* ws, double2* H_out, double2* V_out,
                                double* evals_out, cudaStream_t s) {
  if (!ws) return LITHO_E_NULL;
  const SocsLayout l = socs_layout(n_source, n_band, sms_now());
  const char* w = static_cast<const char*>(ws);
  const size_t m = (size_t)l.ldg * l.ldg * 16;
  cudaError_t e = cudaSuccess;
  if (H_out) e = cudaMemcpyAsync(H_out, w + l.G, m, cudaMemcpyDeviceToDevice, s);
  if (e == cudaSuccess && V_out) e = cudaMemcpyAsync(V_out, w + l.V, m, cudaMemcpyDeviceToDevice, s);
  if (e == cudaSuccess && evals_out)
    e = cudaMemcpyAsync(evals_out, w + l.evals, (size_t)l.ldg * 8, cudaMemcpyDeviceToDevice, s);
  return e == cudaSuccess ? LITHO_OK : (int)e;
}

namespace litho {
// This module's progress-wait budget on the current device (litho_set_wait_limit).
cudaError_t set_wait_limit_gram(long long cycles) { return set_wait_limit_here(cycles); }
}  // namespace litho
