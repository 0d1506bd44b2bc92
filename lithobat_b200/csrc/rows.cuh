// Row engines shared by the Abbe, SOCS and ILT pipelines (rows.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/litho_b200.h"

namespace litho {

// Pair-FFT synthesis of real images from Hermitian band boxes of half-width
// g0: available for power-of-two n in [256, 2048] and g0 <= 31.
bool synth_pairs_ok(int n, int g0);
int synth_pairs_blocks(int n);
cudaError_t launch_synth_pairs(const float2* box, int g0, int n, int n_out, const float2* tw, const LithoNorm* norm,
                               float* image, float* peak, float* blockmax, cudaStream_t s, cudaEvent_t mid,
                               float2* cbuf);
// Bytes of the whole-image column buffer of launch_synth_pairs.
int64_t synth_cols_bytes(int n_out, int n, int g0);

// Tensor-core synthesis (synth_mma.cu): same contract as launch_synth_pairs,
// for power-of-two n in [256, 4096] and g0 <= 31; `planes` holds
// synth_mma_bytes(n_out, n, g0) of workspace, `status` the word a wait that
// gives up sets to LITHO_E_TIMEOUT.
bool synth_mma_ok(int n, int g0);
bool synth_mma_pick(int n_out, int n, int g0);   // ok, and the batch is large enough to gain
int64_t synth_mma_bytes(int n_out, int n, int g0);
cudaError_t launch_synth_mma(const float2* box, int g0, int n, int n_out, const float2* tw, const LithoNorm* norm,
                             float* image, float* peak, float* blockmax, cudaStream_t s, cudaEvent_t mid,
                             void* planes, int* status, int num_sms);

}  // namespace litho
