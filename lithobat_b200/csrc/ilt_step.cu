// One ILT iteration of a batch of clips in one call: the loop body of
// opc/ilt.py:run_ilt (:576-596) -- dJ/dtheta, Adam, the beta anneal, mask_of
// -- followed by the objective and its adjoint (opc/ilt.py:_Objective
// :292-360 on socs_fields / socs_gradient :208-266), for callers that drive
// the optimisation from C (no Python host layer).
//
// The gradient travels between iterations as its band box H (the transform
// of dJ/dmask on |f| <= h; dJ/dmask is band-limited to the kernels' band),
// so an iteration is, on the caller's stream:
//   g = synthesis of H                                   (litho_band_synthesis)
//   theta, m1, m2, mask <- Adam on g sigma'(beta theta)  (litho_ilt_update_sched)
//   M = band box of the mask                             (litho_band_spectrum)
//   B = image band box, B(g) = sum_f Tc(f+g, f) M(f+g) M*(f)     (litho_socs_tcc_image)
//   cost, pattern error, S = band box of dJ/dI           (litho_ilt_image_objective_band)
//   H = adjoint band box from S and M                    (litho_socs_tcc_adjoint)
// Every stage is one of the library's own entry points, so the iteration is
// bit for bit the one the Python layer's graph-replayed step takes.
#include "common.cuh"

namespace litho {
namespace {

struct StepLayout {
  int64_t grad, mbox, ibox, sbox, counters, ws_synth, ws_band, ws_obj, total;
  size_t synth_bytes, band_bytes, obj_bytes;
};

int step_layout(int n_clips, int n, int h, StepLayout& l) {
  size_t synth = 0, band = 0, obj = 0;
  int st;
  if ((st = litho_band_synthesis_workspace(n_clips, n, &synth)) != LITHO_OK) return st;
  if ((st = litho_band_spectrum_workspace(n_clips, n, h, &band)) != LITHO_OK) return st;
  if ((st = litho_ilt_image_objective_band_workspace(n_clips, n, 2 * h, 2 * h, &obj)) != LITHO_OK) return st;
  const int64_t side = 2 * h + 1, G = 4 * h + 1;
  int64_t off = 0;
  l.grad = off;     off = align16(off + (int64_t)n_clips * n * n * 4);
  l.mbox = off;     off = align16(off + (int64_t)n_clips * side * side * 8);
  l.ibox = off;     off = align16(off + (int64_t)n_clips * G * G * 8);
  l.sbox = off;     off = align16(off + (int64_t)n_clips * G * G * 8);
  l.counters = off; off = align16(off + (int64_t)n_clips * 4);
  l.ws_synth = off; off = align16(off + (int64_t)synth);
  l.ws_band = off;  off = align16(off + (int64_t)band);
  l.ws_obj = off;   off = align16(off + (int64_t)obj);
  l.total = off;
  l.synth_bytes = synth;
  l.band_bytes = band;
  l.obj_bytes = obj;
  return LITHO_OK;
}

}  // namespace
}  // namespace litho

using namespace litho;

extern "C" int litho_ilt_step_workspace(int n_clips, int n, int h, size_t* bytes) {
  if (!bytes) return LITHO_E_NULL;
  if (n_clips < 1 || n < 2 || h < 0) return LITHO_E_SIZE;
  if (n % 4) return LITHO_E_SIZE;
  StepLayout l{};
  const int st = step_layout(n_clips, n, h, l);
  if (st) return st;
  *bytes = (size_t)l.total;
  return LITHO_OK;
}

extern "C" int litho_ilt_step(const void* tcc_dev, int n_band, int h, int n_clips, int n, const float* target_dev,
                              float* theta_dev, float* m1_dev, float* m2_dev, LithoIltSched* sched_dev,
                              void* grad_box_dev, float* mask_out_dev, float scale, float level, float sign,
                              float steepness_a, float step, float b1, float b2, float eps, double* cost_out_dev,
                              long long* perr_out_dev, void* ws, size_t ws_bytes, cudaStream_t s) {
  if (!tcc_dev || !target_dev || !theta_dev || !m1_dev || !m2_dev || !sched_dev || !grad_box_dev || !mask_out_dev ||
      !cost_out_dev || !perr_out_dev || !ws)
    return LITHO_E_NULL;
  size_t need = 0;
  int st = litho_ilt_step_workspace(n_clips, n, h, &need);
  if (st) return st;
  if (ws_bytes < need) return LITHO_E_WORKSPACE;
  size_t tcc_need = 0;
  if ((st = litho_socs_tcc_bytes(n_band, h, &tcc_need)) != LITHO_OK) return st;
  if (((uintptr_t)ws & 15) || ((uintptr_t)tcc_dev & 15) || ((uintptr_t)grad_box_dev & 7)) return LITHO_E_ALIGN;
  StepLayout l{};
  if ((st = step_layout(n_clips, n, h, l)) != LITHO_OK) return st;
  char* w = static_cast<char*>(ws);
  float* grad = reinterpret_cast<float*>(w + l.grad);
  void* mbox = w + l.mbox;
  void* ibox = w + l.ibox;
  void* sbox = w + l.sbox;
  unsigned int* counters = reinterpret_cast<unsigned int*>(w + l.counters);
  const long long count = (long long)n_clips * n * n;
  const cudaError_t e = cudaMemsetAsync(counters, 0, (size_t)n_clips * 4, s);
  if (e != cudaSuccess) return (int)e;
  if ((st = litho_band_synthesis(grad_box_dev, n_clips, n, h, 0, grad, w + l.ws_synth, l.synth_bytes, s)) != 0)
    return st;
  if ((st = litho_ilt_update_sched(grad, count, sched_dev, step, b1, b2, eps, theta_dev, m1_dev, m2_dev,
                                   mask_out_dev, s)) != 0)
    return st;
  if ((st = litho_band_spectrum(mask_out_dev, 0, n_clips, n, h, 1.0f / ((float)n * (float)n), mbox, w + l.ws_band,
                                l.band_bytes, s)) != 0)
    return st;
  if ((st = litho_socs_tcc_image(tcc_dev, n_band, h, mbox, n_clips, ibox, s)) != 0) return st;
  if ((st = litho_ilt_image_objective_band(ibox, n_clips, n, 2 * h, target_dev, scale, level, sign, steepness_a,
                                           2 * h, scale / ((float)n * (float)n), sbox, counters, cost_out_dev,
                                           perr_out_dev, w + l.ws_obj, l.obj_bytes, s)) != 0)
    return st;
  return litho_socs_tcc_adjoint(tcc_dev, n_band, h, mbox, sbox, n_clips, grad_box_dev, s);
}

extern "C" int litho_ilt_step_status(int n_clips, int n, int h, const void* ws, cudaStream_t s) {
  if (!ws) return LITHO_E_NULL;
  StepLayout l{};
  const int st = step_layout(n_clips, n, h, l);
  if (st) return st;
  int words[3] = {0, 0, 0};
  const char* w = static_cast<const char*>(ws);
  const int64_t offs[3] = {l.ws_synth, l.ws_band, l.ws_obj};
  for (int i = 0; i < 3; ++i) {
    const cudaError_t e = cudaMemcpyAsync(&words[i], w + offs[i], sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e != cudaSuccess) return (int)e;
  }
  const cudaError_t e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return (int)e;
  for (int i = 0; i < 3; ++i)
    if (words[i]) return words[i];
  return LITHO_OK;
}
