// Device functions whose float results decide discrete outcomes (occlusion
// masks, tile classes, uv-cell keys).  They are written as the same float
// expressions as the upstream kernels and every translation unit of this
// library is compiled with the upstream flags (-O3 --use_fast_math, FMA
// contraction on), so the compiler lowers them to the same instructions and
// the decisions are bit-identical.  Parity tests pin this against the
// upstream kernels themselves.
#pragma once
#include <cuda_runtime.h>

#include "vb_internal.h"

namespace vb {

// Per-pixel occlusion dot of one endpoint: (l x + m y + n z) * invn.
// Upstream: viss_recon_kernel.cuh:271-272 (stage 1),
// viss_recon_kernel_mirror_tile_vissfast.cuh:1101-1102 (stage 2).
__device__ __forceinline__ float occ_dot(float lp, float mp, float np, float x, float y,
                                         float z, float invn) {
  return (lp * x + mp * y + np * z) * invn;
}

// Tile-cone three-way test of one endpoint direction against a tile cone
// (centre dot `dotc`, cone cosA/sinA), upstream
// viss_recon_kernel_mirror_tile_vissfast.cuh:91-98.
__device__ __forceinline__ void cone_classify(float dotc, float cosA, float sinA, float cosphi,
                                              bool& all_vis, bool& all_hid) {
  dotc = fminf(1.0f, fmaxf(-1.0f, dotc));
  float sind = sqrtf(fmaxf(0.0f, 1.0f - dotc * dotc));
  float lower = dotc * cosA - sind * sinA;
  float upper = dotc * cosA + sind * sinA;
  all_vis = (lower >= cosphi);
  all_hid = (upper < cosphi);
}

// Unit endpoint direction used by the tile test: (x, y, z) * invn, then the
// dot with the tile centre, upstream ..._vissfast.cuh:484-485, 525-526.
__device__ __forceinline__ float cone_dot(float ux, float uy, float uz, float cx, float cy,
                                          float cz) {
  return ux * cx + uy * cy + uz * cz;
}

// Round half away from zero, upstream viss_recon_kernel.cuh:13.
__device__ __forceinline__ int round_half_away(float x) {
  return (x >= 0.0f) ? (int)floorf(x + 0.5f) : (int)ceilf(x - 0.5f);
}

// Full-grid key of one signed baseline, upstream viss_recon_kernel.cuh:303-311.
__device__ __forceinline__ int uv_key_full(float uu, float vv, float inv_du, int RES, int half) {
  int ui = round_half_away(uu * inv_du);
  int vi = round_half_away(vv * inv_du);
  int U = ui + half;
  int V = vi + half;
  if ((unsigned)U >= (unsigned)RES || (unsigned)V >= (unsigned)RES) return 0;
  return U * RES + V + 1;
}

// Half-grid key of one positive half-baseline, upstream
// viss_recon_kernel_mirror_tile_vissfast.cuh:742-748.
__device__ __forceinline__ int uv_key_half(float uu, float vv, float inv_du, int RES, int half) {
  int U = (int)floorf(uu * inv_du + 0.5f) + half;
  int V = (int)floorf(vv * inv_du + 0.5f) + half;
  if (U < 0 || U >= RES || V < 0 || V >= RES) return 0;
  return U * RES + V + 1;
}

// Exact (margin-protected) classification of one endpoint against a cone:
// 1 = every pixel of the tile passes the FP32 test, -1 = every pixel fails,
// 0 = undecided.
//
// With r = endpoint * invn (|r| = 1 to within 1e-6, checked), d = angle(axis, r),
// a = the cone's half-angle and p any pixel direction of the cone, p.r spans
// [cos(min(pi, d + a)), cos(max(0, d - a))].  Against a threshold cos(phi):
//   all pass when d + a <= phi: a <= phi and cos d >= cos(phi - a) = cos phi cos a + sin phi sin a;
//   all fail when d - a >= phi: a <= pi - phi and cos d <= cos(phi + a) = cos phi cos a - sin phi sin a.
// cos d is the FP64 dot of the axis with r (within 1e-6 of the unit-vector
// dot); the thresholds are moved by a margin of 1e-5 with directed rounding
// (cos phi up for "pass", down for "fail"; sin phi rounded up, which only
// tightens both tests), so a decided class holds for the FP32 per-pixel dot,
// whose evaluation error is below 2e-6 for unit vectors.  No FP64 square
// root or division.
__device__ __forceinline__ int exact_class(const ExactCone& c, float x, float y, float z, float invn,
                                           float cosphi) {
  const double rx = (double)x * invn, ry = (double)y * invn, rz = (double)z * invn;
  const double rr = fma(rx, rx, fma(ry, ry, rz * rz));
  if (!(fabs(rr - 1.0) <= 2e-6)) return 0;   // |r| off unit by more than 1e-6 (or NaN): undecided
  const double cd = fma(c.cx, rx, fma(c.cy, ry, c.cz * rz));
  constexpr float kMargin = 1e-5f;
  constexpr double kDotErr = 2e-6;           // |r| - 1 plus FP64 rounding
  const float cv = __fadd_ru(cosphi, kMargin);
  if (cv <= 1.0f && c.cos_a >= (double)cv) {
    const float sv = __fsqrt_ru(fmaxf(0.0f, __fmaf_ru(-cv, cv, 1.0f)));
    if (cd - kDotErr >= fma((double)cv, c.cos_a, (double)sv * c.sin_a)) return 1;
  }
  const float ch = __fsub_rd(cosphi, kMargin);
  if (ch >= -1.0f && c.cos_a >= -(double)ch) {
    const float sh = __fsqrt_ru(fmaxf(0.0f, __fmaf_ru(-ch, ch, 1.0f)));
    if (cd + kDotErr <= fma((double)ch, c.cos_a, -(double)sh * c.sin_a)) return -1;
  }
  return 0;
}

// The same classification in FP64 with the exact endpoint norm (two square
// roots and a division per call; the FP32 evaluation error of the per-pixel
// test is < 2e-6 for unit vectors, the margin 1e-5).  Stage 1 calls this form
// from its out-of-line sub-tile test: with exact_class there, the persistent
// stage-1 kernel ran 8 % slower on the nside-1024 day (1332 against 1231 ms)
// with identical decisions, a code-generation effect around the call.
__device__ __forceinline__ int exact_class_fp64(const ExactCone& c, float x, float y, float z, float invn,
                                                float cosphi) {
  double rx = (double)x * invn, ry = (double)y * invn, rz = (double)z * invn;
  double rn = sqrt(rx * rx + ry * ry + rz * rz);
  double cd = (c.cx * rx + c.cy * ry + c.cz * rz) / rn;
  cd = fmin(1.0, fmax(-1.0, cd));
  // d = angle(axis, endpoint), a = half-angle: the cone's dots with the
  // endpoint span [cos(d + a), cos(d - a)], clamped at d + a >= pi and d <= a;
  // cos(d -/+ a) = cos d cos a +/- sin d sin a with sin d = sqrt(1 - cos^2 d)
  const double sd = sqrt(fmax(0.0, 1.0 - cd * cd));
  double lo = (cd <= -c.cos_a) ? -1.0 : cd * c.cos_a - sd * c.sin_a;
  double hi = (cd >= c.cos_a) ? 1.0 : cd * c.cos_a + sd * c.sin_a;
  // scale by the endpoint norm (|r invn| = 1 +- 3e-7) conservatively
  const double margin = 1e-5;
  if (lo * rn - margin >= (double)cosphi && lo - margin >= (double)cosphi) return 1;
  if (hi * rn + margin < (double)cosphi && hi + margin < (double)cosphi) return -1;
  return 0;
}

}  // namespace vb
