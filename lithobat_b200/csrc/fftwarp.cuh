// Warp-per-line transforms of length L = 32 R (R = 4 .. 32) in registers.
//
// Four-step form: with i = p + 32 q (lane p, register q) and k = r + R s,
//     X[k] = sum_p w32^(p s) [ wL^(p r) sum_q x[p + 32 q] wR^(q r) ],
// so each lane runs an R-point FFT over its registers, multiplies by wL^(p r),
// the warp transposes the 32 x 32 block once through shared memory, and each
// lane runs a 32-point FFT. A warp carries 32 / R lines at once (32 complex
// registers per lane whatever L is). Input: x[l R + q] = line l, element
// p + 32 q. Output: lane λ holds line λ / R at indices (λ % R) + R s in x[s].
#pragma once

#include "common.cuh"

namespace litho {

constexpr int kTbLd = 33;  // row pitch of the per-warp transpose buffer (complex)

// The shared twiddle table of warp_fft_lines in lane-major order:
// t[r * 32 + p] = w^(p r), w = exp(+2 pi i / L), for lane p and register r <
// R, so the 32 lanes of a warp read 32 consecutive entries (no bank
// conflicts). src[stride * j] = exp(+2 pi i j / L); p r < L, so no index wraps.
__device__ __forceinline__ void fill_lane_twiddles(float2* t, int L, const float2* __restrict__ src, int stride) {
  for (int i = threadIdx.x; i < L; i += blockDim.x) t[i] = src[stride * ((i & 31) * (i >> 5))];
}

// tb: this warp's 32 x kTbLd complex buffer; tw: fill_lane_twiddles' table.
template <int L, int SIGN>
__device__ __forceinline__ void warp_fft_lines(float2 (&x)[32], float2* tb, const float2* tw) {
  constexpr int R = L / 32, LPW = 32 / R;
  static_assert(R >= 2 && R <= 32 && R * LPW == 32, "warp_fft_lines: L in {64 .. 1024}");
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int l = 0; l < LPW; ++l) {
    float2 y[R];
#pragma unroll
    for (int q = 0; q < R; ++q) y[q] = x[l * R + q];
    fft_reg<R, SIGN>(y);
#pragma unroll
    for (int r = 0; r < R; ++r) {
      if (r == 0) {
        x[l * R] = y[0];
      } else {
        float2 w = tw[r * 32 + lane];  // w^(lane r)
        if (SIGN < 0) w.y = -w.y;
        x[l * R + r] = cmul(y[r], w);
      }
    }
  }
  __syncwarp();
#pragma unroll
  for (int rho = 0; rho < 32; ++rho) tb[rho * kTbLd + lane] = x[rho];
  __syncwarp();
#pragma unroll
  for (int p = 0; p < 32; ++p) x[p] = tb[lane * kTbLd + p];
  __syncwarp();
  fft_reg<32, SIGN>(x);
}

}  // namespace litho
