// Pupil function of one optical state at one frequency, evaluated in FP64.
//
// Restates, for a single in-aperture point:
//   expose/pupil.py:defocus_opd (:155-221), zernike_noll/_radial_poly (:81-141),
//   vector_coefficients (:292-369), and expose/aerial_image.py:_pupil_phase
//   (:142-166): P = exp(i W), W = defocus OPD + 2 pi sum_j c_j Z_j(rho, phi).
// The aperture decision itself (rho <= 1) is made by the caller with the
// exact IEEE operations of the reference; everything here is continuous, so
// FP64 rounding differences against numpy are far below the FP32 result.
#pragma once

#include "common.cuh"

namespace litho {

// Noll index j (1..21) -> radial order n and signed azimuthal order m, the
// standard Noll (1976) ordering; cos(m phi) for m > 0, sin(|m| phi) for m < 0.
__device__ __forceinline__ void noll_nm(int j, int& n, int& m) {
  switch (j) {
    case 1: n = 0; m = 0; break;   case 2: n = 1; m = 1; break;   case 3: n = 1; m = -1; break;
    case 4: n = 2; m = 0; break;   case 5: n = 2; m = -2; break;  case 6: n = 2; m = 2; break;
    case 7: n = 3; m = -1; break;  case 8: n = 3; m = 1; break;   case 9: n = 3; m = -3; break;
    case 10: n = 3; m = 3; break;  case 11: n = 4; m = 0; break;  case 12: n = 4; m = 2; break;
    case 13: n = 4; m = -2; break; case 14: n = 4; m = 4; break;  case 15: n = 4; m = -4; break;
    case 16: n = 5; m = 1; break;  case 17: n = 5; m = -1; break; case 18: n = 5; m = 3; break;
    case 19: n = 5; m = -3; break; case 20: n = 5; m = 5; break;  default: n = 5; m = -5; break;
  }
}

// Zernike radial polynomial R_n^|m|(r), r already clipped to [0, 1].
__device__ __forceinline__ double zernike_radial(int n, int ma, double r) {
  const double r2 = r * r;
  switch (n * 10 + ma) {
    case 0: return 1.0;
    case 11: return r;
    case 20: return 2.0 * r2 - 1.0;
    case 22: return r2;
    case 31: return (3.0 * r2 - 2.0) * r;
    case 33: return r2 * r;
    case 40: return (6.0 * r2 - 6.0) * r2 + 1.0;
    case 42: return (4.0 * r2 - 3.0) * r2;
    case 44: return r2 * r2;
    case 51: return ((10.0 * r2 - 12.0) * r2 + 3.0) * r;
    case 53: return (5.0 * r2 - 4.0) * r2 * r;
    case 55: return r2 * r2 * r;
  }
  return 0.0;
}

// Wavefront phase W [rad] at normalised radius rho and azimuth (cp, sp).
__device__ __forceinline__ double pupil_phase(const LithoPupil& P, double rho, double cp, double sp) {
  double W = 0.0;
  if (P.defocus != 0.0) {
    if (!P.exact_defocus) {
      W = M_PI * P.NA * P.NA * rho * rho * P.defocus / (P.wavelength * P.n_image);
    } else {
      const double s = rho * P.NA / P.n_image;
      const double s2 = fmin(fmax(s * s, 0.0), 1.0);
      W = (2.0 * M_PI / P.wavelength) * (P.n_image * P.defocus * (1.0 - sqrt(1.0 - s2)));
    }
  }
  if (P.has_zernike) {
    const double r = fmin(fmax(rho, 0.0), 1.0);
    // cos(k phi), sin(k phi) for k = 0..5 from the unit phasor (cp, sp).
    double ck[6], sk[6];
    ck[0] = 1.0; sk[0] = 0.0;
#pragma unroll
    for (int k = 1; k < 6; ++k) {
      ck[k] = ck[k - 1] * cp - sk[k - 1] * sp;
      sk[k] = sk[k - 1] * cp + ck[k - 1] * sp;
    }
    double z = 0.0;
    for (int j = 1; j <= 21; ++j) {
      const double c = P.zernike[j - 1];
      if (c == 0.0) continue;
      int n, m;
      noll_nm(j, n, m);
      const int ma = m < 0 ? -m : m;
      const double norm = (m == 0) ? sqrt((double)(n + 1)) : sqrt(2.0 * (n + 1));
      double Z = norm * zernike_radial(n, ma, r);
      if (m > 0) Z *= ck[ma];
      else if (m < 0) Z *= sk[ma];
      z += 2.0 * M_PI * c * Z;
    }
    W += z;
  }
  return W;
}

// (cW, sW): the scalar factor exp(iW) (times the mask blank's reflection in
// the multilayer model); the vector components multiply it.
__device__ __forceinline__ void pupil_components(const LithoPupil& P, double rho, double cp, double sp, double jx,
                                                 double jy, double cW, double sW, float2* out) {
  if (!P.vector) {
    out[0] = make_float2((float)cW, (float)sW);
    return;
  }
  const double stm = P.NA / P.n_image;
  const double s = rho * stm;
  const double s2 = fmin(fmax(s * s, 0.0), 1.0);
  const double ct = sqrt(1.0 - s2), st = sqrt(s2);
  const double es = -jx * sp + jy * cp;
  const double ep = jx * cp + jy * sp;
  double vx = -es * sp + ep * ct * cp;
  double vy = es * cp + ep * ct * sp;
  double vz = -ep * st;
  if (P.obliquity) {
    const double a = sqrt(ct);
    vx *= a; vy *= a; vz *= a;
  }
  out[0] = make_float2((float)(cW * vx), (float)(sW * vx));
  out[1] = make_float2((float)(cW * vy), (float)(sW * vy));
  out[2] = make_float2((float)(cW * vz), (float)(sW * vz));
}

__device__ __forceinline__ void pupil_direction(double fx, double fy, double& cp, double& sp) {
  const double r = sqrt(fx * fx + fy * fy);
  cp = 1.0;
  sp = 0.0;  // atan2(0, 0) = 0
  if (r > 0.0) {
    cp = fx / r;
    sp = fy / r;
  }
}

// Coherent pupil value(s) at an in-aperture point. (fx, fy) is the diffracted
// ray's frequency minus the source offset; rho its normalised radius.
// Scalar: out[0] = exp(iW). Vector: out[c] = exp(iW) * V_c, c = x, y, z.
__device__ __forceinline__ void pupil_values(const LithoPupil& P, double rho, double fx, double fy,
                                             double jx, double jy, float2* out) {
  double cp, sp;
  pupil_direction(fx, fy, cp, sp);
  const double W = pupil_phase(P, rho, cp, sp);
  double sW, cW;
  sincos(W, &sW, &cW);
  pupil_components(P, rho, cp, sp, jx, jy, cW, sW, out);
}

// pupil_values times the complex factor (rr + i ri).
__device__ __forceinline__ void pupil_values_scaled(const LithoPupil& P, double rho, double fx, double fy,
                                                    double jx, double jy, double rr, double ri, float2* out) {
  double cp, sp;
  pupil_direction(fx, fy, cp, sp);
  const double W = pupil_phase(P, rho, cp, sp);
  double sW, cW;
  sincos(W, &sW, &cW);
  pupil_components(P, rho, cp, sp, jx, jy, cW * rr - sW * ri, cW * ri + sW * rr, out);
}

// Exact aperture test of expose/aerial_image.py:_pupil_geometry (:131-138):
// rho = sqrt((FX - fsx)^2 + (FY - fsy)^2) / (NA / lambda) <= 1, with FX the
// numpy fftfreq value of bin kx. Returns rho (> 1 when outside) and the
// offset frequency components.
__device__ __forceinline__ double aperture_rho(int kx, int ky, double val, double fsx, double fsy,
                                               double kmax, double& fx, double& fy) {
  fx = dsub(bin_freq(kx, val), fsx);
  fy = dsub(bin_freq(ky, val), fsy);
  const double r2 = dadd(dmul(fx, fx), dmul(fy, fy));
  return ddiv(dsqrt(r2), kmax);
}

// Reflection of the mask blank for the order at frequency (FX, FY) under
// source offset (fsx, fsy) (expose/m3d/provider.py:252-270): sin theta =
// |(tilt lambda fs / m + chief ray) + lambda F / m|, then |r| and arg r
// interpolated linearly in theta = asin(min(sin theta, 1)) on the ascending
// table, held at its end values outside it; 0 when sin theta > 1.
__device__ __forceinline__ void mirror_reflection(const LithoMirror& M, const double* __restrict__ tab, double FX,
                                                  double FY, double fsx, double fsy, double& re, double& im) {
  const double lam = M.wavelength, m = M.reduction;
  const double sx0 = dadd(ddiv(dmul(dmul(M.tilt_sign, lam), fsx), m), M.sin_cx);
  const double sy0 = dadd(ddiv(dmul(dmul(M.tilt_sign, lam), fsy), m), M.sin_cy);
  const double sx = dadd(sx0, ddiv(dmul(lam, FX), m));
  const double sy = dadd(sy0, ddiv(dmul(lam, FY), m));
  const double st = dsqrt(dadd(dmul(sx, sx), dmul(sy, sy)));
  if (!(st <= 1.0)) {
    re = 0.0;
    im = 0.0;
    return;
  }
  const double th = asin(fmax(st, 0.0));
  const int nt = M.n_theta;
  const double* xp = tab;
  const double* mag = tab + nt;
  const double* ph = tab + 2 * nt;
  double a, p;
  if (th <= xp[0]) {
    a = mag[0];
    p = ph[0];
  } else if (th >= xp[nt - 1]) {
    a = mag[nt - 1];
    p = ph[nt - 1];
  } else {
    // bisection for xp[j] <= th < xp[j + 1]
    int lo = 0, hi = nt - 1;
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (xp[mid] <= th) lo = mid; else hi = mid;
    }
    const double dx = dsub(th, xp[lo]);
    const double span = dsub(xp[lo + 1], xp[lo]);
    a = dadd(dmul(ddiv(dsub(mag[lo + 1], mag[lo]), span), dx), mag[lo]);
    p = dadd(dmul(ddiv(dsub(ph[lo + 1], ph[lo]), span), dx), ph[lo]);
  }
  double sp, cp;
  sincos(p, &sp, &cp);
  re = a * cp;
  im = a * sp;
}

}  // namespace litho
