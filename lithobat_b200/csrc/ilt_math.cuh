// Per-pixel arithmetic of the ILT objective, shared by the objective kernel
// (ilt.cu) and the synthesis that applies it to the image it makes (rows.cu),
// so both give the same values bit for bit.
#pragma once

#include "common.cuh"

namespace litho {

// sigmoid(s) with s clipped to [-60, 60] (opc/ilt.py:326, 378). The
// correctly rounded reciprocal (rcp.rn) is the IEEE quotient 1 / x itself,
// without the general division's operand scaling and special-case path.
__device__ __forceinline__ float sigmoid_clipped(float s) {
  s = fminf(fmaxf(s, -60.f), 60.f);
  return __frcp_rn(1.0f + expf(-s));
}

// The resist relaxation of the objective, sigmoid(s) clipped as above, with
// the hardware exponential and reciprocal (__expf, __fdividef). The
// exponential's relative error grows with |s| (documented bound 2 +
// 1.173 |s| ulps), so z is a few ulps from the correctly rounded value near
// the threshold, where cost and dJ/dfield take their size, and up to ~70 ulps
// at the clip, where z (1 - z) < 1e-26 and r = z - t is set by the target.
// The mask (sigmoid_clipped), whose value feeds Adam's sign-like first
// steps, keeps the correctly rounded form. 1 + e^60 < 2^126, the bound below
// which __fdividef is a true quotient.
__device__ __forceinline__ float objective_sigmoid(float s) {
  s = fminf(fmaxf(s, -60.f), 60.f);
  return __fdividef(1.0f, 1.0f + __expf(-s));
}

// One pixel of the relaxed resist objective (opc/ilt.py:_Objective, :313-336)
// for image value img and target t: signed = sign (scale img - level),
// z = sigmoid(a signed), r = z - t; accumulates r^2 into cost and the pattern
// error into perr; returns dJ/dfield = sign (2 / npix) r a z (1 - z) (the
// factor 2 / npix as inv_npix2; sign (2 / npix) a is one loop-invariant
// product); *signed_out receives signed.
__device__ __forceinline__ float ilt_objective_pixel(float img, float t, float scale, float level, float sign,
                                                     float a, float inv_npix2, float& cost, unsigned int& perr,
                                                     float* signed_out) {
  const float s = sign * (img * scale - level);
  const float z = objective_sigmoid(a * s);
  const float r = z - t;
  cost = fmaf(r, r, cost);
  perr += ((s > 0.f) != (t > 0.5f)) ? 1u : 0u;
  *signed_out = s;
  return (sign * inv_npix2 * a) * r * (z * (1.0f - z));
}

// Operands of the objective applied inside the image synthesis.
struct SynthObj {
  const float* target;
  float scale, level, sign, a, inv_npix2;
  float* dfield;
  double* cost_part;       // [field][block]
  unsigned int* perr_part;
  unsigned int* counters;  // [field], zero between calls
  double* cost_out;        // [field]: sum / npix
  long long* perr_out;
  // the band form (no dfield): the band rows of dJ/dfield on |k| <= band_half,
  // [field][k + band_half][row], are written instead of dJ/dfield itself
  float2* band_rows = nullptr;
  int band_half = 0;
};

}  // namespace litho
