// Shared-memory radix-2 transforms of many lines at once (plain.cu, wide.cu).
#pragma once

#include "common.cuh"

namespace litho {

// In-place radix-2 DIT over `lines` sequences of length n held in shared
// memory (stride ld), input already bit-reversed. SIGN +1 inverse, -1 forward.
template <int SIGN>
__device__ void block_fft_lines(float2* s, int n, int lines, int ld, const float2* tw) {
  const int halfn = n >> 1;
  for (int half = 1; half < n; half <<= 1) {
    const int tstep = n / (2 * half);
    __syncthreads();
    for (int id = threadIdx.x; id < lines * halfn; id += blockDim.x) {
      const int line = id / halfn, bf = id - line * halfn;
      const int k = bf & (half - 1), i0 = ((bf - k) << 1) + k, i1 = i0 + half;
      float2 w = tw[k * tstep];
      if (SIGN < 0) w.y = -w.y;
      float2* p = s + line * ld;
      const float2 a = p[i0], b = cmul(p[i1], w);
      p[i0] = cadd(a, b);
      p[i1] = csub(a, b);
    }
  }
  __syncthreads();
}

__device__ __forceinline__ int brev(int i, int log2n) { return (int)(__brev((unsigned)i) >> (32 - log2n)); }

}  // namespace litho
