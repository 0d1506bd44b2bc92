// Shared device helpers for liblitho_b200: complex arithmetic, register-
// resident radix-2 FFTs, twiddle tables and launch checks.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/litho_b200.h"
#include "twiddles.cuh"

namespace litho {

// ---------------------------------------------------------------------------
// complex float2
// ---------------------------------------------------------------------------
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {  // a * conj(b)
  return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
__device__ __forceinline__ float cabs2(float2 a) { return a.x * a.x + a.y * a.y; }
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }

// t / n for a component count n in {1, 3} and 0 <= t < 2^31, without an
// integer division (multiply-high by ceil(2^32 / 3)).
__device__ __forceinline__ int div_ncomp(int t, int n) {
  return n == 3 ? (int)__umulhi((unsigned)t, 0x55555556u) : t;
}

// ---------------------------------------------------------------------------
// Register FFT: natural-order in and out, radix-2 decimation in time,
// SIGN = +1 computes sum_k v_k exp(+2 pi i k j / N) (unnormalised inverse),
// SIGN = -1 the forward transform. N <= 64, fully unrolled so every index and
// twiddle is a compile-time constant and the array stays in registers.
// ---------------------------------------------------------------------------
template <int N>
struct Log2 { static constexpr int value = 1 + Log2<N / 2>::value; };
template <>
struct Log2<1> { static constexpr int value = 0; };

__host__ __device__ constexpr int bitrev(int i, int bits) {
  int r = 0;
  for (int b = 0; b < bits; ++b) r |= ((i >> b) & 1) << (bits - 1 - b);
  return r;
}

// b * exp(SIGN * 2 pi i t / 64), with the four trivial angles special-cased so
// no multiply by an exact 0 or 1 is emitted.
template <int SIGN>
__device__ __forceinline__ float2 twiddle64(float2 b, int t) {
  t &= 63;
  if (t == 0) return b;
  if (t == 32) return make_float2(-b.x, -b.y);
  if (t == 16) return SIGN > 0 ? make_float2(-b.y, b.x) : make_float2(b.y, -b.x);
  if (t == 48) return SIGN > 0 ? make_float2(b.y, -b.x) : make_float2(-b.y, b.x);
  const float c = tw64_re(t);
  const float s = SIGN > 0 ? tw64_im(t) : -tw64_im(t);
  return make_float2(b.x * c - b.y * s, b.x * s + b.y * c);
}

// One radix-2 butterfly (a, b) <- (a + w b, a - w b), w = exp(SIGN 2 pi i t / 64).
// Component-wise sums run as packed FP32 pairs (__fadd2_rn / __ffma2_rn, one
// instruction for both components). A non-trivial w is factored as
// f (1 + i r) (|cos| >= |sin|: f = cos, r = tan) or f (r + i) (f = sin,
// r = cot), |r| <= 1, so u = w b / f costs two FMAs and the scale by f rides
// in the packed FMAs a +- f u. w = +-i keeps the swap-and-add form.
template <int SIGN>
__device__ __forceinline__ void bfly64(float2& a, float2& b, int t) {
  t &= 63;
  const float2 a0 = a;
  if (t == 0 || t == 32) {
    const float2 p = __fadd2_rn(a0, b), m = __fadd2_rn(a0, make_float2(-b.x, -b.y));
    a = t == 0 ? p : m;
    b = t == 0 ? m : p;
    return;
  }
  if (t == 16 || t == 48) {
    const float2 bw = twiddle64<SIGN>(b, t);
    a = cadd(a0, bw);
    b = csub(a0, bw);
    return;
  }
  const float r = SIGN > 0 ? tw64_ratio(t) : -tw64_ratio(t);
  float2 u;
  float f;
  if (tw64_cos_major(t)) {
    u = make_float2(fmaf(-r, b.y, b.x), fmaf(r, b.x, b.y));
    f = tw64_re(t);
  } else {
    u = make_float2(fmaf(r, b.x, -b.y), fmaf(r, b.y, b.x));
    f = SIGN > 0 ? tw64_im(t) : -tw64_im(t);
  }
  a = __ffma2_rn(u, make_float2(f, f), a0);
  b = __ffma2_rn(u, make_float2(-f, -f), a0);
}

template <int N, int SIGN>
__device__ __forceinline__ void fft_reg(float2 (&v)[N]) {
  static_assert(N >= 2 && N <= 64 && (N & (N - 1)) == 0, "fft_reg: N in {2..64}");
  constexpr int LOG = Log2<N>::value;
#pragma unroll
  for (int i = 0; i < N; ++i) {
    const int j = bitrev(i, LOG);
    if (j > i) {
      const float2 t = v[i];
      v[i] = v[j];
      v[j] = t;
    }
  }
#pragma unroll
  for (int half = 1; half < N; half <<= 1) {
#pragma unroll
    for (int base = 0; base < N; base += 2 * half) {
#pragma unroll
      for (int k = 0; k < half; ++k) bfly64<SIGN>(v[base + k], v[base + k + half], k * (64 / (2 * half)));
    }
  }
}

// The same transform for inputs known to be zero outside the bit mask NZ
// (bit i set: v[i] may be non-zero). Butterflies with a known-zero operand
// become copies or a single twiddle, so a pruned transform (a band of 2h+1
// of 32 inputs) costs only the work its non-zeros need. The masks are
// compile-time constants after unrolling, so every test below folds away.
__host__ __device__ constexpr uint64_t nz_bitrev(uint64_t m, int log) {
  uint64_t r = 0;
  for (int i = 0; i < (1 << log); ++i)
    if ((m >> i) & 1ull) r |= 1ull << bitrev(i, log);
  return r;
}
__host__ __device__ constexpr uint64_t nz_after(uint64_t m, int n, int half) {
  // non-zero mask after the butterfly stage of span `half`
  uint64_t r = 0;
  for (int base = 0; base < n; base += 2 * half)
    for (int k = 0; k < half; ++k) {
      const bool any = ((m >> (base + k)) & 1ull) || ((m >> (base + k + half)) & 1ull);
      if (any) r |= (1ull << (base + k)) | (1ull << (base + k + half));
    }
  return r;
}
template <int N, int SIGN, uint64_t M, int HALF>
struct SparseStage {
  // one radix-2 stage of span HALF with non-zero mask M, then the next stage
  static __device__ __forceinline__ void run(float2 (&v)[N]) {
    if constexpr (HALF < N) {
#pragma unroll
      for (int base = 0; base < N; base += 2 * HALF) {
#pragma unroll
        for (int k = 0; k < HALF; ++k) {
          const bool za = !((M >> (base + k)) & 1ull), zb = !((M >> (base + k + HALF)) & 1ull);
          if (za && zb) {
            // both zero: stays zero
          } else if (zb) {
            v[base + k + HALF] = v[base + k];
          } else if (za) {
            const float2 bw = twiddle64<SIGN>(v[base + k + HALF], k * (64 / (2 * HALF)));
            v[base + k] = bw;
            v[base + k + HALF] = make_float2(-bw.x, -bw.y);
          } else {
            bfly64<SIGN>(v[base + k], v[base + k + HALF], k * (64 / (2 * HALF)));
          }
        }
      }
      SparseStage<N, SIGN, nz_after(M, N, HALF), 2 * HALF>::run(v);
    }
  }
};

template <int N, int SIGN, uint64_t NZ>
__device__ __forceinline__ void fft_reg_sparse(float2 (&v)[N]) {
  static_assert(N >= 2 && N <= 64 && (N & (N - 1)) == 0, "fft_reg_sparse: N in {2..64}");
  constexpr int LOG = Log2<N>::value;
#pragma unroll
  for (int i = 0; i < N; ++i) {
    const int j = bitrev(i, LOG);
    if (j > i) {
      const float2 t = v[i];
      v[i] = v[j];
      v[j] = t;
    }
  }
  SparseStage<N, SIGN, nz_bitrev(NZ, LOG), 1>::run(v);
}

// Non-zero mask of a 32-point sequence supported on d in [-H, H] (d mod 32).
__host__ __device__ constexpr uint64_t band_mask32(int H) {
  uint64_t m = 0;
  for (int d = -H; d <= H; ++d) m |= 1ull << (d & 31);
  return m;
}

// ---------------------------------------------------------------------------
// FP64 with every rounding explicit (no FMA contraction), so that decisions
// like "rho <= 1" reproduce numpy's IEEE double arithmetic bit for bit.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ double dsqrt(double a) { return __dsqrt_rn(a); }

// Signed FFT bin k of an N-point grid -> physical frequency, exactly as
// numpy.fft.fftfreq(N, d)[k mod N] = float(k) * (1.0 / (N * d)).
__device__ __forceinline__ double bin_freq(int k, double val) { return dmul((double)k, val); }

// Does signed bin k exist on an N-point FFT grid?
__device__ __forceinline__ bool bin_valid(int k, int n) { return k >= -(n / 2) && k <= (n - 1) / 2; }

__host__ __device__ __forceinline__ int64_t align16(int64_t x) { return (x + 15) & ~int64_t(15); }

// Pitch (float2) of one row group's [kp][b] block (32 x (M + 1)) in the
// transpose-sum stage of the band DFTs (band.cu, rows.cu). A half-warp's
// 8-byte stores span 16 lanes = 16 / Lp row groups (Lp = min(M, 32) lanes
// each); the Lp mod 16 pad starts those groups 2 Lp banks apart, so they
// no longer land on the same banks (a whole multiple of 32 banks apart).
__host__ __device__ constexpr int band_group_pitch(int M) { return 32 * (M + 1) + ((M < 32 ? M : 32) % 16); }

// ---------------------------------------------------------------------------
// TMA bulk copies (cp.async.bulk) completing on shared-memory mbarriers.
// Every wait is bounded by a clock budget; a wait that gives up reports it
// through a status word instead of spinning forever.
// ---------------------------------------------------------------------------
constexpr long long kWaitCycles = 4000000000LL;  // ~2 s at 1.9 GHz

// Clock budget of the waits that make progress (a stage's operands, an MMA's
// accumulator). One copy per translation unit (each .cu is its own device
// module); litho_set_wait_limit() lowers it on the current device so tests
// can make those waits give up. Waits that drain copies or MMAs already in
// flight before a block exits (mbar_wait_drain) always get kWaitCycles.
static __device__ long long g_wait_limit = kWaitCycles;

// Host: set this translation unit's g_wait_limit on the current device.
[[maybe_unused]] static inline cudaError_t set_wait_limit_here(long long cycles) {
  return cudaMemcpyToSymbol(g_wait_limit, &cycles, sizeof(cycles));
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
// Global -> shared bulk copy; dst/src 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// at most N of this thread's bulk groups still reading their shared source
template <int N>
__device__ __forceinline__ void bulk_wait_read() {
  asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(N) : "memory");
}
// at most N of this thread's bulk groups not yet complete
template <int N>
__device__ __forceinline__ void bulk_wait() {
  asm volatile("cp.async.bulk.wait_group %0;" ::"n"(N) : "memory");
}
// orders this thread's generic-proxy shared-memory writes before later
// async-proxy (bulk copy) reads of them
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// true when the phase with this parity completed within `limit` clock cycles.
__device__ __forceinline__ bool mbar_wait_for(uint64_t* bar, uint32_t parity, long long limit) {
  if (mbar_try_wait(bar, parity)) return true;
  const long long t0 = clock64();
  while (clock64() - t0 < limit)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
// A progress wait: within this translation unit's g_wait_limit.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  if (mbar_try_wait(bar, parity)) return true;
  return mbar_wait_for(bar, parity, *(volatile long long*)&g_wait_limit);
}
// A drain wait (copies or MMAs this block already issued, before it exits or
// releases TMEM): the full budget, whatever g_wait_limit says.
__device__ __forceinline__ bool mbar_wait_drain(uint64_t* bar, uint32_t parity) {
  return mbar_wait_for(bar, parity, kWaitCycles);
}
// Order this thread's earlier generic-proxy shared accesses before later
// async-proxy (TMA) accesses to the same buffer.
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Ampere-style asynchronous 8-byte global -> shared copies (LDGSTS), grouped
// and waited on per thread.
__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
// 16 bytes, both addresses 16-byte aligned, bypassing L1 (streamed operands)
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Device twiddle table w[j] = exp(sign * 2 pi i j / n), FP64 evaluated, FP32 stored.
__global__ void k_twiddle_table(float2* w, int n, int sign);

// The shared exp(+2 pi i j / n) table of a power-of-two n <= 8192 on the
// current device (twiddle_cache.cu), or nullptr: then the caller builds its
// own with k_twiddle_table (other sizes, or a stream that is capturing before
// the device's tables exist).
const float2* shared_twiddles(int n, cudaStream_t s);

// `own` filled with exp(+2 pi i j / n) on `s` unless the shared table serves n.
inline const float2* twiddles_for(int n, float2* own, cudaStream_t s) {
  if (const float2* t = shared_twiddles(n, s)) return t;
  k_twiddle_table<<<(n + 255) / 256, 256, 0, s>>>(own, n, +1);
  return own;
}

}  // namespace litho
