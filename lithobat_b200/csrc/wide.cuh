// Host-side pieces of the wide-pupil engine (wide.cu) shared with the uneven
// work queue (queue.cu): the workspace layout of one plan, the stages before
// the coherent passes and the stages after them.
#pragma once

#include "common.cuh"

namespace litho {

struct WideLayout {
  int64_t status, twN, twL, u1, mb, table, T, partial, J, F, bbox, spec, blockmax, total;
  int jobs_per_chunk;
};

// t_bytes >= 0 sizes the pass-A buffer T exactly (the queue's ring of
// slots); the default sizes it for chunks of jobs within the engine's budget.
WideLayout wide_layout(const LithoAbbePlan& p, int64_t t_bytes = -1);
bool wide_plan_ok(const LithoAbbePlan& p);

// Status word cleared, then the band boxes of every clip's mask spectrum
// (scaled 1 / N^2) into the workspace's `mb` region.
int wide_prepare(const LithoAbbePlan& p, const void* mask, void* ws, const WideLayout& l, cudaStream_t s,
                 int num_sms);

// From the items' partial intensities on the coarse grid to the images:
// ordered reduction per output, F = FFT_L(J) / L^2, the image band box,
// synthesis and normalisation. transposed: the partials hold J^T.
int wide_finish(const LithoAbbePlan& p, const void* blob, float* image, float* peak, void* ws, const WideLayout& l,
                bool transposed, cudaStream_t s);

}  // namespace litho
