// Stage 2: segmented short-time 2-D reconstruction, all segments of a day in
// one device-only batch (no host round trips, graph capturable).
//
//  per segment s (one CTA each): no-intercept plane fit w ~ fa u + fb v over
//    the segment's signed baselines in double-double (upstream: long double on
//    the host, viss_recon_kernel.cuh:673-701), RES / half / du
//    (main_recon_online.cu:377-383, IEEE float steps as the host code);
//  keys: uv cell of every keyed baseline (full grid: signed set, round half
//    away, viss_recon_kernel.cuh:295-312; mirror: positive half set,
//    floor(x+0.5), ..._vissfast.cuh:730-749), composite (segment << 32 | key);
//  one stable radix sort of (composite key, index) for all segments, run
//    flags + scan -> groups, representative idx_sorted[s0 + (L>>1)]
//    (..._vissfast.cuh:869-879), dense group records;
//  reconstruction: persistent CTAs over (pixel block x group chunk):
//    acc += Re(V_q exp(+2 pi i (ugu l' + vgu m'))), l' = l + fa n, m' = m + fb n,
//    W += 1 per visible group (viss_recon_kernel.cuh:521-639,
//    ..._vissfast.cuh:1039-1286); FP32 sums per staged sub-chunk, FP64 totals;
//  finalize: C = sum C / sum W (blockage=1) or C / sum nuniq (blockage=0).
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <cmath>
#include <type_traits>

#include "vb_common.cuh"
#include "vb_geom.cuh"
#include "vb_internal.h"

namespace vb {

constexpr int S2_THREADS = 256;
constexpr int S2_STAGE = S2_THREADS;     // group records staged per step (one per thread)
constexpr double kMagic2 = 805306368.0;  // 1.5 * 2^29: 2^-23-turn ulp, see stage 1
constexpr float kTwoPiF2 = 6.28318530717958647692f;
constexpr float kAngScale2 = 6.28318530717958647692f * 1.1920928955078125e-7f;

struct GroupRec {         // 96 bytes
  double a, b, c;         // t = a l + b m + c n  (a = ugu, b = vgu, c = ugu fa + vgu fb)
  float vx, vy;           // representative / averaged visibility
  float fa, fb;
  float cp1, cp2;         // horizon cosines of the representative endpoints
  float4 p1, p2;          // (x, y, z, invn) of the representative endpoints
  float chi, clo;         // c split into two floats (double-single phase)
  int key, flags;         // flags: bit0 = skip (key 0 / nothing to add), bit1 = non-finite V,
                          // bits 2.. = segment
};
struct GroupMeta {        // members of a group (member-sampling path)
  int s0, L, seg, pad;
};

// --- double-double helpers (Dekker/Knuth two-sum and fma two-product) ------
struct dd { double hi, lo; };
__device__ __forceinline__ dd dd_add(dd a, dd b) {
  double s = a.hi + b.hi;
  double bb = s - a.hi;
  double e = (a.hi - (s - bb)) + (b.hi - bb);
  e += a.lo + b.lo;
  double hi = s + e;
  return {hi, e - (hi - s)};
}
__device__ __forceinline__ dd dd_from_prod(double a, double b) {
  double p = a * b;
  return {p, fma(a, b, -p)};
}
__device__ __forceinline__ dd dd_mul(dd a, dd b) {
  double p = a.hi * b.hi;
  double e = fma(a.hi, b.hi, -p);
  e += a.hi * b.lo + a.lo * b.hi;
  double hi = p + e;
  return {hi, e - (hi - p)};
}
__device__ __forceinline__ dd dd_neg(dd a) { return {-a.hi, -a.lo}; }
__device__ __forceinline__ dd dd_div(dd a, dd b) {
  double q1 = a.hi / b.hi;
  dd r = dd_add(a, dd_neg(dd_mul({q1, 0.0}, b)));
  double q2 = r.hi / b.hi;
  r = dd_add(r, dd_neg(dd_mul({q2, 0.0}, b)));
  double q3 = r.hi / b.hi;
  dd q = dd_add({q1, 0.0}, {q2, 0.0});
  return dd_add(q, {q3, 0.0});
}
// Correctly rounded float of a double-double value.
__device__ __forceinline__ float dd_to_float(dd a) {
  float f = __double2float_rn(a.hi);
  double r = a.hi - (double)f;   // exact
  double up = (double)nextafterf(f, INFINITY) - (double)f;
  double dn = (double)f - (double)nextafterf(f, -INFINITY);
  double rr = r + a.lo;
  if (rr > 0.5 * up || (rr == 0.5 * up && (__float_as_int(f) & 1))) return nextafterf(f, INFINITY);
  if (-rr > 0.5 * dn || (-rr == 0.5 * dn && (__float_as_int(f) & 1))) return nextafterf(f, -INFINITY);
  return f;
}

// --- per-segment fit ---------------------------------------------------------
__global__ void __launch_bounds__(256) k_seg_fit(const float* __restrict__ u, const float* __restrict__ v,
                                                 const float* __restrict__ w, int nbl, const int* __restrict__ seg_t0,
                                                 const int* __restrict__ seg_tlen, float bl_max, float lambda,
                                                 int grid_res, int mirror, vb_seg_params* __restrict__ out) {
  __shared__ dd red[5][256];
  const int s = blockIdx.x;
  const int i0 = 2 * nbl * seg_t0[s];
  const int n = 2 * nbl * seg_tlen[s];
  dd a[5];
  for (int k = 0; k < 5; ++k) a[k] = {0.0, 0.0};
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    double uu = u[i0 + i], vv = v[i0 + i], ww = w[i0 + i];
    a[0] = dd_add(a[0], dd_from_prod(uu, uu));
    a[1] = dd_add(a[1], dd_from_prod(vv, vv));
    a[2] = dd_add(a[2], dd_from_prod(uu, vv));
    a[3] = dd_add(a[3], dd_from_prod(uu, ww));
    a[4] = dd_add(a[4], dd_from_prod(vv, ww));
  }
  for (int k = 0; k < 5; ++k) red[k][threadIdx.x] = a[k];
  __syncthreads();
  for (int off = 128; off > 0; off >>= 1) {
    if (threadIdx.x < off)
      for (int k = 0; k < 5; ++k) red[k][threadIdx.x] = dd_add(red[k][threadIdx.x], red[k][threadIdx.x + off]);
    __syncthreads();
  }
  if (threadIdx.x != 0) return;
  dd su2 = red[0][0], sv2 = red[1][0], suv = red[2][0], suw = red[3][0], svw = red[4][0];
  dd p = dd_mul(su2, sv2);
  dd denom = dd_add(p, dd_neg(dd_mul(suv, suv)));
  vb_seg_params q;
  q.denom = denom.hi;
  dd scale = (p.hi > 0.0) ? p : dd{1.0, 0.0};
  double eps = 1e-24 * scale.hi;
  if (!isfinite(denom.hi) || fabs(denom.hi) < eps) {
    double sign = (denom.hi >= 0.0) ? 1.0 : -1.0;
    denom = {sign * eps, 0.0};
  }
  dd na = dd_add(dd_mul(sv2, suw), dd_neg(dd_mul(suv, svw)));
  dd nb = dd_add(dd_mul(su2, svw), dd_neg(dd_mul(suv, suw)));
  dd A = dd_div(na, denom), Bq = dd_div(nb, denom);
  float fa = 0.f, fb = 0.f;
  if (isfinite(A.hi) && isfinite(Bq.hi)) {
    fa = dd_to_float(A);
    fb = dd_to_float(Bq);
  }
  q.fa = fa;
  q.fb = fb;
  // RES / half / du: IEEE float steps of main_recon_online.cu:377-383
  int RES;
  const float span = __fdiv_rn(__fmul_rn(2.0f, bl_max), lambda);
  if (grid_res > 0) {
    RES = (grid_res % 2 == 0) ? grid_res + 1 : grid_res;
  } else {
    float lmax = __fsqrt_rn(__fadd_rn(1.0f, __fmul_rn(fa, fa)));
    float mmax = __fsqrt_rn(__fadd_rn(1.0f, __fmul_rn(fb, fb)));
    float lmmax = fmaxf(lmax, mmax);
    float temp_res = ceilf(__fmul_rn(__fmul_rn(span, 2.0f), lmmax));
    float r = __fsub_rn(__fadd_rn(__fadd_rn(temp_res, 2.0f), 1.0f), fmodf(temp_res, 2.0f));
    RES = (int)r;
  }
  q.RES = RES;
  q.half = (RES - 1) / 2;
  q.du = __fdiv_rn(span, (float)(RES - 1));
  q.inv_du = __fdiv_rn(1.0f, q.du);
  q.nuniq = 0;
  q.group_start = 0;
  q.n_keyed = mirror ? nbl * seg_tlen[s] : 2 * nbl * seg_tlen[s];
  q.pad = 0;
  out[s] = q;
}

__device__ __forceinline__ int seg_of_step(int step, const int* __restrict__ seg_t0, int nseg) {
  int lo = 0, hi = nseg - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (seg_t0[mid] <= step) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// Composite keys for the keyed set (mirror: half indices, full: signed indices).
__global__ void k_keys(const float* __restrict__ u, const float* __restrict__ v, int n_keyed, int nbl, int mirror,
                       const int* __restrict__ seg_t0, int nseg, const vb_seg_params* __restrict__ sp,
                       unsigned long long* __restrict__ keys, int* __restrict__ vals, int* __restrict__ raw_keys) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_keyed; i += gridDim.x * blockDim.x) {
    const int step = mirror ? i / nbl : i / (2 * nbl);
    const int s = seg_of_step(step, seg_t0, nseg);
    const vb_seg_params q = sp[s];
    int key;
    if (mirror) {
      const int f = half_to_full_pos(i, nbl);
      key = uv_key_half(u[f], v[f], q.inv_du, q.RES, q.half);
    } else {
      key = uv_key_full(u[i], v[i], q.inv_du, q.RES, q.half);
    }
    keys[i] = ((unsigned long long)(unsigned)s << 32) | (unsigned)key;
    vals[i] = i;
    if (raw_keys) raw_keys[i] = key;
  }
}

__global__ void k_run_flags(const unsigned long long* __restrict__ k, int n, int* __restrict__ flags) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    flags[i] = (i == 0 || k[i] != k[i - 1]) ? 1 : 0;
}

// gid = inclusive scan of flags: run starts, group count, per-segment ranges.
__global__ void k_group_starts(const int* __restrict__ flags, const int* __restrict__ gid, int n,
                               const unsigned long long* __restrict__ k, int* __restrict__ start,
                               int* __restrict__ ngroups, vb_seg_params* __restrict__ sp) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (flags[i]) {
      const int g = gid[i] - 1;
      start[g] = i;
      const int seg = (int)(k[i] >> 32);
      if (i == 0 || (int)(k[i - 1] >> 32) != seg) sp[seg].group_start = g;
      atomicAdd(&sp[seg].nuniq, 1);
    }
    if (i == n - 1) {
      *ngroups = gid[i];
      start[gid[i]] = n;
    }
  }
}

struct RecArgs {
  const unsigned long long* skeys;
  const int* svals;
  const int* start;
  const int* ngroups;
  const vb_seg_params* sp;
  const float *V;       // mirror: V_half (2 floats per half index); full: V_full
  const float *x1, *y1, *z1, *in1, *x2, *y2, *z2, *in2, *cp1, *cp2;
  float cosphi;
  int nbl, mirror, blockage, occ_mode;
  GroupRec* rec;
  GroupMeta* meta;
  unsigned* err;
};

__global__ void k_group_records(const RecArgs r, int max_groups) {
  const int ng = *r.ngroups;
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < ng && g < max_groups; g += gridDim.x * blockDim.x) {
    const int s0 = r.start[g];
    const int L = r.start[g + 1] - s0;
    const unsigned long long ck = r.skeys[s0];
    const int seg = (int)(ck >> 32);
    const int key = (int)(unsigned)(ck & 0xffffffffull);
    const vb_seg_params q = r.sp[seg];
    GroupRec o;
    o.key = key;
    o.flags = ((key == 0) ? 1 : 0) | (seg << 2);
    float ugu = 0.f, vgu = 0.f;
    if (key != 0) {
      int tmp = key - 1;
      int U = tmp / q.RES;
      int Vc = tmp - U * q.RES;
      int ui = U - q.half;
      int vi = Vc - q.half;
      ugu = ui * q.du;
      vgu = vi * q.du;
    }
    o.a = (double)ugu;
    o.b = (double)vgu;
    o.c = (double)ugu * (double)q.fa + (double)vgu * (double)q.fb;
    o.chi = (float)o.c;
    o.clo = (float)(o.c - (double)o.chi);
    o.fa = q.fa;
    o.fb = q.fb;
    // the F32X phase needs |a l + b m + c n| < 2^28 turns (kMagic2)
    if (fabs(o.a) + fabs(o.b) + fabs(o.c) >= 268435456.0) atomicOr(r.err, ERR_PHASE_RANGE);
    o.vx = o.vy = 0.f;
    o.cp1 = o.cp2 = r.cosphi;
    o.p1 = o.p2 = make_float4(0.f, 0.f, 0.f, 0.f);
    if (!r.blockage) {
      // group average of V (upstream: CUB ReduceByKey float2 sum / count)
      double sx = 0.0, sy = 0.0;
      for (int j = 0; j < L; ++j) {
        const int idx = r.svals[s0 + j];
        sx += (double)r.V[2 * idx];
        sy += (double)r.V[2 * idx + 1];
      }
      o.vx = (float)(sx / L);
      o.vy = (float)(sy / L);
    } else if (r.occ_mode == 2) {
      const int rep = r.svals[s0 + (L >> 1)];
      const int f = r.mirror ? half_to_full_pos(rep, r.nbl) : rep;
      o.vx = r.V[2 * rep];
      o.vy = r.V[2 * rep + 1];
      o.p1 = make_float4(r.x1[f], r.y1[f], r.z1[f], r.in1[f]);
      o.p2 = make_float4(r.x2[f], r.y2[f], r.z2[f], r.in2[f]);
      if (r.cp1) { o.cp1 = r.cp1[f]; o.cp2 = r.cp2[f]; }
      // full-grid path tests finiteness of V before use (viss_recon_kernel.cuh:595)
      if (!r.mirror && !(isfinite(o.vx) && isfinite(o.vy))) o.flags |= 2;
    }
    r.rec[g] = o;
    if (r.meta) r.meta[g] = GroupMeta{s0, L, seg, 0};
  }
}

// --- reconstruction ------------------------------------------------------------
// Groups per work-queue chunk for ng groups split into at most nchunk_target
// chunks (a multiple of the staging width): ceil(ng / result) <= nchunk_target.
__host__ __device__ inline int group_chunk(int ng, int nchunk_target) {
  int g = (ng + nchunk_target - 1) / nchunk_target;
  g = (g + S2_STAGE - 1) / S2_STAGE * S2_STAGE;
  return g < S2_STAGE ? S2_STAGE : g;
}

struct ReconArgs {
  const float *l, *m, *n;    // the sky's direction cosines (FP64 phases take their exact doubles)
  int64_t npix;
  int block_pix, nblocks, nchunk_target;
  const int* ngroups;
  const GroupRec* rec;
  const GroupMeta* meta;
  const vb_seg_params* sp;   // per segment: fa, fb, first group, group count
  const int* svals;
  const float* V;
  const float *x1, *y1, *z1, *in1, *x2, *y2, *z2, *in2, *cp1, *cp2;
  float cosphi;
  int nbl, mirror, blockage, occ_mode, cull, finite_check;
  const ExactCone* cones;    // one per pixel block (cull == VB_CULL_EXACT)
  int* queue;
  double* Cpart;             // [group chunk][npix]
  unsigned* Wpart;
  unsigned long long* counters;
  unsigned* err;
};

template <int MODE>
__device__ __forceinline__ void recon_phase(const GroupRec& g, double ld, double md, double nd, float lf, float mf,
                                            float nf, float& s, float& c, double& sd, double& cd) {
  if constexpr (MODE == VB_PREC_FP32_FP64PH) {
    double t = fma(g.a, ld, fma(g.b, md, fma(g.c, nd, kMagic2)));
    unsigned lo = (unsigned)__double2loint(t);
    unsigned kb = (lo & 0x7FFFFFu) | 0x4B000000u;
    float ang = __fmaf_rn(__uint_as_float(kb), kAngScale2, -kTwoPiF2);
    __sincosf(ang, &s, &c);
  } else if constexpr (MODE == VB_PREC_FP32_DSPH) {
    const float af = (float)g.a, bf = (float)g.b;
    float p1 = __fmul_rn(af, lf), e1 = __fmaf_rn(af, lf, -p1);
    float p2 = __fmul_rn(bf, mf), e2 = __fmaf_rn(bf, mf, -p2);
    float p3 = __fmul_rn(g.chi, nf), e3 = __fmaf_rn(g.chi, nf, -p3);
    auto rn = [](float x) { return __fsub_rn(__fadd_rn(x, 12582912.0f), 12582912.0f); };
    float fr = __fadd_rn(__fadd_rn(__fsub_rn(p1, rn(p1)), __fsub_rn(p2, rn(p2))), __fsub_rn(p3, rn(p3)));
    float er = __fadd_rn(__fadd_rn(e1, e2), __fmaf_rn(g.clo, nf, e3));
    float t = __fadd_rn(fr, er);
    t = __fsub_rn(t, rn(t));
    t = (t < 0.f) ? __fadd_rn(t, 1.0f) : t;
    __sincosf(__fmul_rn(t, kTwoPiF2), &s, &c);
  } else if constexpr (MODE == VB_PREC_REF32) {
    const float TWO_PI = 6.2831853071795864769f;
    float lp = lf + g.fa * nf;
    float mp = mf + g.fb * nf;
    float ugu = (float)g.a, vgu = (float)g.b;
    float phase = TWO_PI * (ugu * lp + vgu * mp);
    __sincosf(phase, &s, &c);
  } else {
    double t = g.a * (ld + (double)g.fa * nd) + g.b * (md + (double)g.fb * nd);
    sincos(6.283185307179586476925286766559 * t, &sd, &cd);
  }
}

// Per-group data read by the term loop of k_recon_rec, 32 bytes in every mode.
// vx, nvy = Re V, -Im V of the group's visibility (times -1 in the odd slots
// of a dithered mode, see rec_term).
template <int MODE>
struct TermRec {          // FP64, FP32 with FP64 phase: t = a l + b m + c n
  double a, b, c;
  float vx, nvy;
};
template <>
struct TermRec<VB_PREC_FP32_DSPH> {   // double-single phase: a, b and c = chi + clo as floats
  float af, bf, chi, clo, vx, nvy, pad0, pad1;
};
template <>
struct TermRec<VB_PREC_REF32> {       // upstream FP32 arithmetic: (ugu, vgu, fa, fb)
  float ugu, vgu, fa, fb, vx, nvy, pad0, pad1;
};
struct OccRec {           // occlusion data of a mixed group
  float4 p1, p2;
  float cp1, cp2;
};

// Half-turn dithering.  MUFU sin/cos carry a small mean error over the angle
// range, and a term-by-term sum of ~1e4-1e6 terms would add it coherently.  In
// the FP32 modes the odd slot of every pair of staged groups is evaluated half
// a turn further on (exp(i(t + pi)) = -exp(i t)) with its visibility negated,
// so the products are unchanged and the two slots' mean errors cancel.
template <int MODE>
__device__ constexpr bool rec_dither() {
  return MODE == VB_PREC_FP32_FP64PH || MODE == VB_PREC_FP32_DSPH;
}

template <int MODE>
__device__ __forceinline__ TermRec<MODE> make_term(const GroupRec& g, bool odd) {
  TermRec<MODE> t;
  const float sg = (rec_dither<MODE>() && odd) ? -1.0f : 1.0f;
  if constexpr (MODE == VB_PREC_FP32_DSPH) {
    t.af = (float)g.a; t.bf = (float)g.b; t.chi = g.chi; t.clo = g.clo; t.pad0 = t.pad1 = 0.f;
  } else if constexpr (MODE == VB_PREC_REF32) {
    t.ugu = (float)g.a; t.vgu = (float)g.b; t.fa = g.fa; t.fb = g.fb; t.pad0 = t.pad1 = 0.f;
  } else {
    t.a = g.a; t.b = g.b; t.c = g.c;
  }
  t.vx = sg * g.vx;
  t.nvy = -(sg * g.vy);
  return t;
}

template <int MODE>
__device__ __forceinline__ TermRec<MODE> zero_term() {
  return TermRec<MODE>{};
}

// Pixel coordinates of one reconstruction pixel.
struct RecPix {
  double ld, md, nd;
  float lf, mf, nf;
};

// Re(V exp(+2 pi i t)) of one (group, pixel) term accumulated into acc.
// PAR = 1 adds the half turn of the odd dither slot.
template <int MODE, int PAR, class Acc>
__device__ __forceinline__ void rec_term(const TermRec<MODE>& r, const RecPix& p, Acc& acc) {
  if constexpr (MODE == VB_PREC_FP32_FP64PH) {
    constexpr double K = kMagic2 + (PAR ? 0.5 : 0.0);
    const double t = fma(r.a, p.ld, fma(r.b, p.md, fma(r.c, p.nd, K)));
    const unsigned lo = (unsigned)__double2loint(t);
    const unsigned kb = (lo & 0x7FFFFFu) | 0x4B000000u;
    const float ang = __fmaf_rn(__uint_as_float(kb), kAngScale2, -kTwoPiF2);
    float s, c;
    __sincosf(ang, &s, &c);
    acc = fmaf(r.vx, c, acc);
    acc = fmaf(r.nvy, s, acc);
  } else if constexpr (MODE == VB_PREC_FP32_DSPH) {
    auto rn = [](float x) { return __fsub_rn(__fadd_rn(x, 12582912.0f), 12582912.0f); };
    const float p1 = __fmul_rn(r.af, p.lf), e1 = __fmaf_rn(r.af, p.lf, -p1);
    const float p2 = __fmul_rn(r.bf, p.mf), e2 = __fmaf_rn(r.bf, p.mf, -p2);
    const float p3 = __fmul_rn(r.chi, p.nf), e3 = __fmaf_rn(r.chi, p.nf, -p3);
    const float fr = __fadd_rn(__fadd_rn(__fsub_rn(p1, rn(p1)), __fsub_rn(p2, rn(p2))), __fsub_rn(p3, rn(p3)));
    const float er = __fadd_rn(__fadd_rn(e1, e2), __fmaf_rn(r.clo, p.nf, e3));
    float t = __fadd_rn(fr, er);
    t = __fsub_rn(t, rn(t));
    if constexpr (PAR) {
      t = __fadd_rn(t, 0.5f);
      t = __fsub_rn(t, rn(t));
    }
    t = (t < 0.f) ? __fadd_rn(t, 1.0f) : t;   // angle in [0, 2 pi), as stage 1
    float s, c;
    __sincosf(__fmul_rn(t, kTwoPiF2), &s, &c);
    acc = fmaf(r.vx, c, acc);
    acc = fmaf(r.nvy, s, acc);
  } else if constexpr (MODE == VB_PREC_REF32) {
    // upstream: phase = 2 pi (ugu (l + fa n) + vgu (m + fb n)) in FP32
    // (viss_recon_kernel.cuh:620-626, ..._vissfast.cuh:1270-1276)
    const float TWO_PI = 6.2831853071795864769f;
    const float lp = p.lf + r.fa * p.nf;
    const float mp = p.mf + r.fb * p.nf;
    const float phase = TWO_PI * (r.ugu * lp + r.vgu * mp);
    float s, c;
    __sincosf(phase, &s, &c);
    acc += fmaf(r.vx, c, r.nvy * s);
  } else {
    const double t = fma(r.a, p.ld, fma(r.b, p.md, r.c * p.nd));
    double s, c;
    sincospi(2.0 * t, &s, &c);
    acc = fma((double)r.vx, c, acc);
    acc = fma((double)r.nvy, s, acc);
  }
}

// FP32 with FP64 phase, and FP64: the phase of a (group, pixel) term is
// a l' + b m' with the segment's l' = l + fa n, m' = m + fb n (the upstream
// form, viss_recon_kernel.cuh:620-626), formed in FP64 once per pixel per stage
// because the stages of k_recon_rec hold the groups of one segment: two FP64
// products per term instead of three.  Two groups share a 48-byte record (the
// dither pair): three shared loads per two groups.
template <int MODE>
__device__ constexpr bool rec_pairs() {
  return MODE == VB_PREC_FP32_FP64PH || MODE == VB_PREC_FP64;
}
struct PairRec {
  double2 ab0, ab1;   // (a, b) of the even and of the odd slot
  float4 v;           // (vx, -vy) of the even slot, then of the odd slot (dither signs applied)
};

template <int MODE, int PAR, class Acc>
__device__ __forceinline__ void pair_term(const double2 ab, const float vx, const float nvy, const double lp,
                                          const double mp, Acc& acc) {
  if constexpr (MODE == VB_PREC_FP32_FP64PH) {
    constexpr double K = kMagic2 + (PAR ? 0.5 : 0.0);
    const double t = fma(ab.x, lp, fma(ab.y, mp, K));
    const unsigned lo = (unsigned)__double2loint(t);
    const unsigned kb = (lo & 0x7FFFFFu) | 0x4B000000u;
    const float ang = __fmaf_rn(__uint_as_float(kb), kAngScale2, -kTwoPiF2);
    float s, c;
    __sincosf(ang, &s, &c);
    acc = fmaf(vx, c, acc);
    acc = fmaf(nvy, s, acc);
  } else {
    const double t = fma(ab.x, lp, ab.y * mp);
    double s, c;
    sincospi(2.0 * t, &s, &c);
    acc = fma((double)vx, c, acc);
    acc = fma((double)nvy, s, acc);
  }
}

// Writes group record g into slot k of a stage list (pair records or term records).
template <int MODE, class L>
__device__ __forceinline__ void put_term(L* list, int k, const GroupRec& g) {
  const TermRec<MODE> t = make_term<MODE>(g, k & 1);
  if constexpr (rec_pairs<MODE>()) {
    PairRec& pr = list[k >> 1];
    if (k & 1) { pr.ab1 = make_double2(t.a, t.b); pr.v.z = t.vx; pr.v.w = t.nvy; }
    else { pr.ab0 = make_double2(t.a, t.b); pr.v.x = t.vx; pr.v.y = t.nvy; }
  } else {
    list[k] = t;
  }
}
template <int MODE, class L>
__device__ __forceinline__ void put_zero(L* list, int k) {
  if constexpr (rec_pairs<MODE>()) {
    PairRec& pr = list[k >> 1];
    if (k & 1) { pr.ab1 = make_double2(0.0, 0.0); pr.v.z = 0.f; pr.v.w = 0.f; }
    else { pr.ab0 = make_double2(0.0, 0.0); pr.v.x = 0.f; pr.v.y = 0.f; }
  } else {
    list[k] = zero_term<MODE>();
  }
}

// Exact-cone class of a representative against a pixel block (0 hidden,
// 1 visible, 2 mixed).  Out of line: it runs once per (group, block) and would
// otherwise take registers from the term loop.  The square-root-free test
// (exact_class) is 1.2 % faster here than the FP64 form on the nside-1024 day
// (390.9 against 395.8 ms) with the same decisions.
__device__ __noinline__ int exact_group_class(const ExactCone* cone, float4 p1, float cp1, float4 p2, float cp2) {
  const ExactCone c = *cone;
  const int e1 = exact_class(c, p1.x, p1.y, p1.z, p1.w, cp1);
  const int e2 = exact_class(c, p2.x, p2.y, p2.z, p2.w, cp2);
  return (e1 < 0 || e2 < 0) ? 0 : ((e1 > 0 && e2 > 0) ? 1 : 2);
}

// occ_mode 2 (representative) and blockage=0 (group averages) paths.
//
// Work item = (pixel block of PPT * 256 pixels, chunk of groups).  Each thread
// owns PPT pixels.  The chunk is walked in stages of up to 256 groups that
// belong to one segment; per stage the CTA classifies every group against the
// block (hidden / visible / mixed; exact cones with VB_CULL_EXACT, otherwise
// mixed) and compacts the visible and the mixed ones into two lists in shared
// memory; the term loop then runs without branches over the visible list and
// with the per-pixel occlusion test over the mixed list, two groups (the
// dither pair) by PPT pixels per step.
template <int MODE, int PPT>
__global__ void __launch_bounds__(S2_THREADS, 2) k_recon_rec(const ReconArgs a) {
  constexpr int NW = S2_THREADS / 32;
  constexpr bool kPairs = rec_pairs<MODE>();
  using ListT = typename std::conditional<kPairs, PairRec, TermRec<MODE>>::type;
  constexpr int kListLen = kPairs ? (S2_STAGE / 2 + 1) : (S2_STAGE + 1);
  __shared__ ListT s_vis[kListLen];
  __shared__ ListT s_mix[kListLen];
  __shared__ OccRec s_occ[S2_STAGE + 1];
  __shared__ int s_wv[NW], s_wm[NW];
  __shared__ int s_item;
  __shared__ ExactCone s_cone;
  constexpr bool kDouble = (MODE == VB_PREC_FP64);
  using Acc = typename std::conditional<kDouble, double, float>::type;
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int ng = *a.ngroups;
  const int gchunk = group_chunk(ng, a.nchunk_target);
  const int nchunk = (ng + gchunk - 1) / gchunk;
  const int n_items = nchunk * a.nblocks;
  unsigned long long c_fast = 0, c_mask = 0, c_hid = 0, c_all = 0;

  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) s_item = atomicAdd(a.queue, 1);
    __syncthreads();
    const int item = s_item;
    if (item >= n_items) break;
    const int gc = item / a.nblocks;
    const int blk = item - gc * a.nblocks;
    if (a.cull == VB_CULL_EXACT && threadIdx.x == 0) s_cone = a.cones[blk];
    const int64_t pix0 = (int64_t)blk * a.block_pix;
    const int npx_blk = (int)min((int64_t)a.block_pix, a.npix - pix0);

    RecPix px[PPT];
    bool act[PPT];
#pragma unroll
    for (int q = 0; q < PPT; ++q) {
      const int64_t pix = pix0 + q * S2_THREADS + threadIdx.x;
      act[q] = pix < a.npix;
      px[q] = RecPix{0.0, 0.0, 0.0, 0.f, 0.f, 0.f};
      if (act[q]) {
        px[q].lf = a.l[pix]; px[q].mf = a.m[pix]; px[q].nf = a.n[pix];
        px[q].ld = px[q].lf; px[q].md = px[q].mf; px[q].nd = px[q].nf;
      }
    }
    double totC[PPT];
    float kc[PPT];
    unsigned totW[PPT];
#pragma unroll
    for (int q = 0; q < PPT; ++q) { totC[q] = 0.0; kc[q] = 0.f; totW[q] = 0u; }

    const int g_begin = gc * gchunk;
    const int g_end = min(ng, g_begin + gchunk);
    int gs = g_begin;
    while (gs < g_end) {
      // this stage: up to 256 groups of the segment that group gs belongs to
      // (every thread reads the same words)
      const int seg = a.rec[gs].flags >> 2;
      const int seg_end = a.sp[seg].group_start + a.sp[seg].nuniq;
      const int nst = min(S2_STAGE, min(g_end, seg_end) - gs);
      __syncthreads();   // previous stage's lists fully read; s_cone visible
      // --- classify this stage's groups and compact them ---------------------
      int cls = 0;
      GroupRec r;
      if ((int)threadIdx.x < nst) {
        r = a.rec[gs + threadIdx.x];
        if (r.flags & 3) cls = 0;              // key 0, or non-finite V: neither summed nor counted
        else if (!a.blockage) cls = 1;
        else if (a.cull == VB_CULL_EXACT) {
          cls = exact_group_class(&s_cone, r.p1, r.cp1, r.p2, r.cp2);
        } else {
          cls = 2;
        }
      }
      const unsigned bv = __ballot_sync(0xffffffffu, cls == 1);
      const unsigned bm = __ballot_sync(0xffffffffu, cls == 2);
      if (lane == 0) { s_wv[warp] = __popc(bv); s_wm[warp] = __popc(bm); }
      __syncthreads();
      int ov = 0, om = 0, nv = 0, nm = 0;
#pragma unroll
      for (int w = 0; w < NW; ++w) {
        const int cv = s_wv[w], cm = s_wm[w];
        if (w < warp) { ov += cv; om += cm; }
        nv += cv;
        nm += cm;
      }
      const unsigned below = (1u << lane) - 1u;
      if (cls == 1) {
        put_term<MODE>(s_vis, ov + __popc(bv & below), r);
      } else if (cls == 2) {
        const int k = om + __popc(bm & below);
        put_term<MODE>(s_mix, k, r);
        s_occ[k] = OccRec{r.p1, r.p2, r.cp1, r.cp2};
      }
      if (threadIdx.x == 0) {
        // pad odd lists with a record that adds nothing (and fails the test)
        if (nv & 1) put_zero<MODE>(s_vis, nv);
        if (nm & 1) {
          put_zero<MODE>(s_mix, nm);
          s_occ[nm] = OccRec{make_float4(0.f, 0.f, 0.f, 0.f), make_float4(0.f, 0.f, 0.f, 0.f), INFINITY, INFINITY};
        }
        c_fast += (unsigned long long)nv * npx_blk;
        c_mask += (unsigned long long)nm * npx_blk;
        c_hid += (unsigned long long)(nst - nv - nm) * npx_blk;
        c_all += (unsigned long long)nst * npx_blk;
      }
      // the segment's coordinates l' = l + fa n, m' = m + fb n of this thread's pixels
      double lp[PPT], mp[PPT];
      if constexpr (kPairs) {
        const double fa = (double)a.sp[seg].fa, fb = (double)a.sp[seg].fb;
#pragma unroll
        for (int q = 0; q < PPT; ++q) {
          lp[q] = mp[q] = 0.0;
          if (act[q]) {
            // the exact doubles of the float coordinates (the float registers
            // stay for the occlusion test)
            const double nd = (double)px[q].nf;
            lp[q] = fma(fa, nd, (double)px[q].lf);
            mp[q] = fma(fb, nd, (double)px[q].mf);
          }
        }
      }
      __syncthreads();

      // --- visible groups: no test ---------------------------------------------
      Acc e[PPT], o[PPT];
#pragma unroll
      for (int q = 0; q < PPT; ++q) { e[q] = Acc(0); o[q] = Acc(0); }
      if constexpr (kPairs) {
        for (int k2 = 0; k2 < nv; k2 += 2) {
          const PairRec pr = s_vis[k2 >> 1];
#pragma unroll
          for (int q = 0; q < PPT; ++q) {
            pair_term<MODE, 0>(pr.ab0, pr.v.x, pr.v.y, lp[q], mp[q], e[q]);
            pair_term<MODE, 1>(pr.ab1, pr.v.z, pr.v.w, lp[q], mp[q], o[q]);
          }
        }
      } else {
        for (int k = 0; k < nv; k += 2) {
          const TermRec<MODE> r0 = s_vis[k];
          const TermRec<MODE> r1 = s_vis[k + 1];
#pragma unroll
          for (int q = 0; q < PPT; ++q) {
            rec_term<MODE, 0>(r0, px[q], e[q]);
            rec_term<MODE, 1>(r1, px[q], o[q]);
          }
        }
      }
      if (a.blockage) {
#pragma unroll
        for (int q = 0; q < PPT; ++q) totW[q] += (unsigned)nv;
      }
      // --- mixed groups: per-pixel occlusion test ------------------------------
      for (int k = 0; k < nm; k += 2) {
        const OccRec c0 = s_occ[k];
        const OccRec c1 = s_occ[k + 1];
        PairRec pr;
        TermRec<MODE> r0, r1;
        if constexpr (kPairs) {
          pr = s_mix[k >> 1];
        } else {
          r0 = s_mix[k];
          r1 = s_mix[k + 1];
        }
#pragma unroll
        for (int q = 0; q < PPT; ++q) {
          const RecPix& p = px[q];
          const bool in0 = occ_dot(p.lf, p.mf, p.nf, c0.p1.x, c0.p1.y, c0.p1.z, c0.p1.w) >= c0.cp1 &&
                           occ_dot(p.lf, p.mf, p.nf, c0.p2.x, c0.p2.y, c0.p2.z, c0.p2.w) >= c0.cp2;
          const bool in1 = occ_dot(p.lf, p.mf, p.nf, c1.p1.x, c1.p1.y, c1.p1.z, c1.p1.w) >= c1.cp1 &&
                           occ_dot(p.lf, p.mf, p.nf, c1.p2.x, c1.p2.y, c1.p2.z, c1.p2.w) >= c1.cp2;
          Acc t0 = Acc(0), t1 = Acc(0);
          if constexpr (kPairs) {
            pair_term<MODE, 0>(pr.ab0, pr.v.x, pr.v.y, lp[q], mp[q], t0);
            pair_term<MODE, 1>(pr.ab1, pr.v.z, pr.v.w, lp[q], mp[q], t1);
          } else {
            rec_term<MODE, 0>(r0, p, t0);
            rec_term<MODE, 1>(r1, p, t1);
          }
          e[q] += in0 ? t0 : Acc(0);
          o[q] += in1 ? t1 : Acc(0);
          totW[q] += (in0 ? 1u : 0u) + (in1 ? 1u : 0u);
        }
      }
      // --- fold the stage sums into the totals -------------------------------
#pragma unroll
      for (int q = 0; q < PPT; ++q) {
        if constexpr (kDouble) {
          totC[q] += e[q] + o[q];
        } else if constexpr (MODE == VB_PREC_FP32_DSPH) {
          const float x = __fadd_rn(e[q], o[q]);
          const float sr = (float)totC[q];
          const float y = __fsub_rn(x, kc[q]);
          const float t = __fadd_rn(sr, y);
          kc[q] = __fsub_rn(__fsub_rn(t, sr), y);
          totC[q] = t;
        } else {
          totC[q] += (double)e[q] + (double)o[q];
        }
      }
      gs += nst;
    }
#pragma unroll
    for (int q = 0; q < PPT; ++q) {
      if (act[q]) {
        const int64_t pix = pix0 + q * S2_THREADS + threadIdx.x;
        a.Cpart[(int64_t)gc * a.npix + pix] = totC[q];
        a.Wpart[(int64_t)gc * a.npix + pix] = totW[q];
      }
    }
  }
  if (a.counters && threadIdx.x == 0) {
    atomicAdd(&a.counters[0], c_fast);
    atomicAdd(&a.counters[1], c_mask);
    atomicAdd(&a.counters[2], c_hid);
    atomicAdd(&a.counters[3], c_all);
  }
}

// occ_mode 0 / 1 / other: per pixel, sample members, average the visible V.
template <int MODE>
__global__ void __launch_bounds__(S2_THREADS) k_recon_members(const ReconArgs a) {
  __shared__ GroupRec s_rec[S2_STAGE];
  __shared__ GroupMeta s_meta[S2_STAGE];
  __shared__ int s_item;
  constexpr bool kDouble = (MODE == VB_PREC_FP64);
  const int ng = *a.ngroups;
  const int gchunk = group_chunk(ng, a.nchunk_target);
  const int nchunk = (ng + gchunk - 1) / gchunk;
  const int n_items = nchunk * a.nblocks;
  unsigned long long c_all = 0;
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) s_item = atomicAdd(a.queue, 1);
    __syncthreads();
    const int item = s_item;
    if (item >= n_items) break;
    const int gc = item / a.nblocks;
    const int blk = item - gc * a.nblocks;
    const int64_t pix = (int64_t)blk * a.block_pix + threadIdx.x;
    const bool active = pix < a.npix;
    float lf = 0.f, mf = 0.f, nf = 0.f;
    double ld = 0.0, md = 0.0, nd = 0.0;
    if (active) {
      lf = a.l[pix]; mf = a.m[pix]; nf = a.n[pix];
      ld = lf; md = mf; nd = nf;
    }
    const int npx_blk = (int)min((int64_t)a.block_pix, a.npix - (int64_t)blk * a.block_pix);
    double totC = 0.0;
    unsigned totW = 0;
    const int g_begin = gc * gchunk;
    const int g_end = min(ng, g_begin + gchunk);
    for (int gs = g_begin; gs < g_end; gs += S2_STAGE) {
      const int nst = min(S2_STAGE, g_end - gs);
      __syncthreads();
      for (int j = threadIdx.x; j < nst; j += S2_THREADS) {
        s_rec[j] = a.rec[gs + j];
        s_meta[j] = a.meta[gs + j];
      }
      __syncthreads();
      double accd = 0.0;
      float accf = 0.f;
      for (int j = 0; j < nst; ++j) {
        const GroupRec& r = s_rec[j];
        if (r.flags & 1) continue;
        const GroupMeta mt = s_meta[j];
        const int L = mt.L;
        if (L <= 0) continue;
        float sx = 0.f, sy = 0.f;
        int cnt = 0;
        auto handle = [&](int pos) {
          const int idx = a.svals[pos];
          const int f = a.mirror ? half_to_full_pos(idx, a.nbl) : idx;
          const float o1 = occ_dot(lf, mf, nf, a.x1[f], a.y1[f], a.z1[f], a.in1[f]);
          const float o2 = occ_dot(lf, mf, nf, a.x2[f], a.y2[f], a.z2[f], a.in2[f]);
          const float c1 = a.cp1 ? a.cp1[f] : a.cosphi;
          const float c2 = a.cp2 ? a.cp2[f] : a.cosphi;
          if (o1 >= c1 && o2 >= c2) {
            const float vx = a.V[2 * idx], vy = a.V[2 * idx + 1];
            if (isfinite(vx) && isfinite(vy)) { sx += vx; sy += vy; ++cnt; }
          }
        };
        const int s0 = mt.s0, s1 = mt.s0 + L;
        if (a.occ_mode == 0) {
          for (int pos = s0; pos < s1; ++pos) handle(pos);
        } else if (a.occ_mode == 1) {
          handle(s0);
        } else {
          handle(s0);
          handle(s0 + (L / 3));
          handle(s0 + (2 * L / 3));
          handle(s1 - 1);
        }
        if (cnt > 0 && active) {
          const float invc = 1.0f / (float)cnt;
          const float vx = sx * invc, vy = sy * invc;
          float s, c;
          double sd, cd;
          recon_phase<MODE>(r, ld, md, nd, lf, mf, nf, s, c, sd, cd);
          if constexpr (kDouble) accd += (double)vx * cd - (double)vy * sd;
          else accf += fmaf(vx, c, -vy * s);
          totW += 1;
        }
      }
      totC += kDouble ? accd : (double)accf;
    }
    if (threadIdx.x == 0) c_all += (int64_t)npx_blk * (g_end - g_begin);
    if (active) {
      a.Cpart[(int64_t)gc * a.npix + pix] = totC;
      a.Wpart[(int64_t)gc * a.npix + pix] = totW;
    }
  }
  if (a.counters && threadIdx.x == 0) {
    atomicAdd(&a.counters[1], c_all);
    atomicAdd(&a.counters[3], c_all);
  }
}

__global__ void k_finalize(const double* __restrict__ Cpart, const unsigned* __restrict__ Wpart,
                           const int* __restrict__ ngroups, int nchunk_target, int64_t npix, int blockage,
                           float* __restrict__ C, uint32_t* __restrict__ W, double* __restrict__ wsum_out) {
  const int ng = *ngroups;
  const int gchunk = group_chunk(ng, nchunk_target);
  const int nchunk = (ng + gchunk - 1) / gchunk;
  if (blockIdx.x == 0 && threadIdx.x == 0 && wsum_out) *wsum_out = (double)ng;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < npix; p += stride) {
    double c = 0.0;
    unsigned w = 0;
    for (int k = 0; k < nchunk; ++k) {
      c += Cpart[(int64_t)k * npix + p];
      w += Wpart[(int64_t)k * npix + p];
    }
    float out;
    if (blockage) out = (w > 0) ? (float)(c / (double)w) : 0.0f;
    else out = (ng > 0) ? (float)(c / (double)ng) : 0.0f;
    C[p] = out;
    if (W) W[p] = w;
  }
}

// ---------------------------------------------------------------------------
int stage2_plan(int n_half_total, int nseg, int64_t npix, const vb_stage2_opts* o, Stage2Plan* p) {
  if (!o || !p) return fail(VB_ERR_INVALID, "stage 2: null argument");
  if (n_half_total < 0 || nseg <= 0 || npix <= 0)
    return fail(VB_ERR_INVALID, "stage 2: n_half_total=%d nseg=%d npix=%lld", n_half_total, nseg, (long long)npix);
  if (o->precision < VB_PREC_REF32 || o->precision > VB_PREC_FP32_DSPH)
    return fail(VB_ERR_INVALID, "stage 2: precision=%d", o->precision);
  if (!(o->lambda > 0.f) || !(o->bl_max > 0.f)) return fail(VB_ERR_INVALID, "stage 2: lambda/bl_max must be > 0");
  Stage2Plan q{};
  q.mirror = o->mirror ? 1 : 0;
  q.blockage = o->blockage ? 1 : 0;
  q.occ_mode = o->occ_mode;
  q.precision = o->precision;
  q.cull = (o->cull == VB_CULL_EXACT && q.blockage && q.occ_mode == 2) ? VB_CULL_EXACT : VB_CULL_NONE;
  q.grid_res = o->grid_res;
  // pixels per thread of the representative / average path (the member path
  // keeps one): by default 4 with the FP64 phase in FP32 (its pair records are
  // read once per 4 pixels; 0.835 against 0.772 of the SFU peak at nside 1024),
  // 2 in the other modes (whose registers do not hold 4); 1, 2 or 4 on request
  if (o->ppt != 0 && o->ppt != 1 && o->ppt != 2 && o->ppt != 4)
    return fail(VB_ERR_INVALID, "stage 2: ppt=%d (0, 1, 2 or 4)", o->ppt);
  const bool members = q.blockage && q.occ_mode != 2;
  const int ppt_auto = (o->precision == VB_PREC_FP32_FP64PH) ? 4 : 2;
  q.ppt = members ? 1 : (o->ppt == 0 ? ppt_auto : o->ppt);
  q.bl_max = o->bl_max;
  q.lambda = o->lambda;
  q.n_half_total = n_half_total;
  q.n_keyed_total = q.mirror ? n_half_total : 2 * n_half_total;
  q.nseg = nseg;
  q.npix = npix;
  q.block_pix = S2_THREADS * q.ppt;
  q.nblocks = (int)ceil_div(npix, q.block_pix);
  if (o->items_per_cta < 0) return fail(VB_ERR_INVALID, "stage 2: items_per_cta=%d", o->items_per_cta);
  const int capacity = sm_count() * 2;
  // enough items per CTA that the dynamic queue's tail (one item) stays short
  const int64_t want_items = (int64_t)capacity * (o->items_per_cta > 0 ? o->items_per_cta : 24);
  int64_t nchunks = ceil_div(want_items, q.nblocks);
  if (nchunks < 1) nchunks = 1;
  // the group count is known on the device only: the kernels split it into at
  // most nchunk_target chunks (group_chunk), which sizes the partial buffers
  const int64_t max_useful = ceil_div(q.n_keyed_total > 0 ? q.n_keyed_total : 1, S2_STAGE);
  if (nchunks > max_useful) nchunks = max_useful;
  q.nchunk_target = (int)nchunks;
  if ((int64_t)q.nblocks * q.nchunk_target > INT32_MAX) return fail(VB_ERR_UNSUPPORTED, "stage 2: too many work items");
  // CUB temporary storage for the largest batch
  size_t sort_bytes = 0, scan_bytes = 0;
  int n = q.n_keyed_total > 0 ? q.n_keyed_total : 1;
  cub::DoubleBuffer<unsigned long long> dk(nullptr, nullptr);
  cub::DoubleBuffer<int> dv(nullptr, nullptr);
  if (cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, dk, dv, n, 0, 64) != cudaSuccess)
    return fail(VB_ERR_CUDA, "stage 2: CUB sort size query failed");
  if (cub::DeviceScan::InclusiveSum(nullptr, scan_bytes, (int*)nullptr, (int*)nullptr, n) != cudaSuccess)
    return fail(VB_ERR_CUDA, "stage 2: CUB scan size query failed");
  q.cub_sort_bytes = sort_bytes;
  q.cub_scan_bytes = scan_bytes;
  *p = q;
  return VB_OK;
}

struct S2Slices {
  vb_seg_params* sp;
  unsigned long long *k0, *k1;
  int *v0, *v1, *flags, *gid, *start, *ngroups, *queue;
  unsigned* err;
  GroupRec* rec;
  GroupMeta* meta;
  double* Cpart;
  unsigned* Wpart;
  ExactCone* cones;
  float* Vfull;
  void* cub_sort;
  void* cub_scan;
  double* wsum;
};

static size_t carve2(const Stage2Plan& p, void* ws, size_t cap, S2Slices* s) {
  Carve c(ws, cap);
  S2Slices x{};
  x.err = c.take<unsigned>(4);   // first: vb_workspace_error_flags reads it at offset 0
  const size_t n = (size_t)(p.n_keyed_total > 0 ? p.n_keyed_total : 1);
  x.sp = c.take<vb_seg_params>(p.nseg);
  x.k0 = c.take<unsigned long long>(n);
  x.k1 = c.take<unsigned long long>(n);
  x.v0 = c.take<int>(n);
  x.v1 = c.take<int>(n);
  x.flags = c.take<int>(n);
  x.gid = c.take<int>(n);
  x.start = c.take<int>(n + 1);
  x.ngroups = c.take<int>(4);
  x.queue = c.take<int>(4);
  x.wsum = c.take<double>(2);
  x.rec = c.take<GroupRec>(n);
  x.meta = c.take<GroupMeta>(n);
  x.Cpart = c.take<double>((size_t)p.nchunk_target * (size_t)p.npix);
  x.Wpart = c.take<unsigned>((size_t)p.nchunk_target * (size_t)p.npix);
  x.cones = c.take<ExactCone>(p.nblocks);
  x.Vfull = p.mirror ? nullptr : c.take<float>((size_t)4 * (p.n_half_total > 0 ? p.n_half_total : 1));
  x.cub_sort = c.take<char>(p.cub_sort_bytes);
  x.cub_scan = c.take<char>(p.cub_scan_bytes);
  if (s) *s = x;
  if (ws && !c.ok) return 0;
  return c.used();
}

int stage2_prepare_cones(const vb_sky* sky, const Stage2Plan& p, void* ws, size_t cap, cudaStream_t st) {
  if (p.cull != VB_CULL_EXACT) return VB_OK;
  S2Slices x;
  if (!carve2(p, ws, cap, &x)) return fail(VB_ERR_NOMEM, "stage 2: workspace too small (%zu bytes)", cap);
  return geom_exact_cones(p.block_pix, sky->l, sky->m, sky->n, p.npix, x.cones, st);
}

size_t stage2_workspace(const Stage2Plan& p, void* ws, size_t cap, void** slices) {
  S2Slices s;
  size_t r = carve2(p, ws, cap, &s);
  (void)slices;
  return r;
}

template <class K>
static int launch_persistent(K kern, const ReconArgs& a, cudaStream_t s) {
  int occ = 0;
  VB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, S2_THREADS, 0));
  if (occ < 1) occ = 1;
  kern<<<sm_count() * occ, S2_THREADS, 0, s>>>(a);
  VB_LAUNCH_CHECK();
  return VB_OK;
}

template <int MODE>
static int launch_recon(const ReconArgs& a, bool members, int ppt, cudaStream_t s) {
  if (members) return launch_persistent(k_recon_members<MODE>, a, s);
  switch (ppt) {
    case 1: return launch_persistent(k_recon_rec<MODE, 1>, a, s);
    case 4: return launch_persistent(k_recon_rec<MODE, 4>, a, s);
    default: return launch_persistent(k_recon_rec<MODE, 2>, a, s);
  }
}

__global__ void k_expand_half(const float* __restrict__ Vh, int n_half, int nbl, float* __restrict__ Vf) {
  for (int ih = blockIdx.x * blockDim.x + threadIdx.x; ih < n_half; ih += gridDim.x * blockDim.x) {
    const int ip = half_to_full_pos(ih, nbl);
    const float re = Vh[2 * ih], im = Vh[2 * ih + 1];
    Vf[2 * ip] = re;
    Vf[2 * ip + 1] = im;
    Vf[2 * (ip + nbl)] = re;
    Vf[2 * (ip + nbl) + 1] = -im;
  }
}

// Steps 1-4 read only the baselines (u, v and the segment table), so a caller
// may run them on a second stream concurrently with stage 1; the sort's
// double-buffer choice is known at enqueue time and handed to stage2_finish.
int stage2_group(const vb_baselines* bl, int nseg, const int* seg_t0, const int* seg_tlen, const Stage2Plan& p,
                 void* ws, size_t cap, cudaStream_t st, Stage2Groups* out) {
  S2Slices x;
  if (!carve2(p, ws, cap, &x)) return fail(VB_ERR_NOMEM, "stage 2: workspace too small (%zu bytes)", cap);
  const int n = p.n_keyed_total;
  const int nbl = bl->nbl;
  out->sorted_keys_alt = 0;
  out->sorted_vals_alt = 0;
  VB_CUDA(cudaMemsetAsync(x.err, 0, sizeof(unsigned), st));
  VB_CUDA(cudaMemsetAsync(x.ngroups, 0, sizeof(int), st));
  VB_CUDA(cudaMemsetAsync(x.wsum, 0, sizeof(double), st));
  int g = (int)ceil_div(n > 0 ? n : 1, 256);
  if (g > sm_count() * 16) g = sm_count() * 16;
  // 1. per-segment fit
  k_seg_fit<<<nseg, 256, 0, st>>>(bl->u, bl->v, bl->w, nbl, seg_t0, seg_tlen, p.bl_max, p.lambda, p.grid_res,
                                  p.mirror, x.sp);
  VB_LAUNCH_CHECK();
  if (n > 0) {
    // 2. keys
    k_keys<<<g, 256, 0, st>>>(bl->u, bl->v, n, nbl, p.mirror, seg_t0, nseg, x.sp, x.k0, x.v0, nullptr);
    VB_LAUNCH_CHECK();
    // 3. stable sort of (segment, key) with the keyed index as payload
    int seg_bits = 1;
    while ((1 << seg_bits) < nseg) ++seg_bits;
    cub::DoubleBuffer<unsigned long long> dk(x.k0, x.k1);
    cub::DoubleBuffer<int> dv(x.v0, x.v1);
    size_t sb = p.cub_sort_bytes;
    VB_CUDA(cub::DeviceRadixSort::SortPairs(x.cub_sort, sb, dk, dv, n, 0, 32 + seg_bits, st));
    const unsigned long long* sk = dk.Current();
    out->sorted_keys_alt = dk.selector;
    out->sorted_vals_alt = dv.selector;
    // 4. runs -> groups
    k_run_flags<<<g, 256, 0, st>>>(sk, n, x.flags);
    VB_LAUNCH_CHECK();
    size_t scb = p.cub_scan_bytes;
    VB_CUDA(cub::DeviceScan::InclusiveSum(x.cub_scan, scb, x.flags, x.gid, n, st));
    k_group_starts<<<g, 256, 0, st>>>(x.flags, x.gid, n, sk, x.start, x.ngroups, x.sp);
    VB_LAUNCH_CHECK();
  }
  return VB_OK;
}

// Steps 5-9, after stage2_group (same workspace, ordered after it on st).
int stage2_finish(const vb_sky* sky, const vb_baselines* bl, const float* V_half, int nseg, const Stage2Plan& p,
                  void* ws, size_t cap, const Stage2Groups& gr, float* C, uint32_t* W, vb_seg_params* seg_params_out,
                  unsigned long long* counters, double* w_scalar_total, cudaStream_t st, const Stage2Pixels* pre,
                  cudaEvent_t kbeg, cudaEvent_t kend) {
  S2Slices x;
  if (!carve2(p, ws, cap, &x)) return fail(VB_ERR_NOMEM, "stage 2: workspace too small (%zu bytes)", cap);
  const int n = p.n_keyed_total;
  const int nbl = bl->nbl;
  int g = (int)ceil_div(n > 0 ? n : 1, 256);
  if (g > sm_count() * 16) g = sm_count() * 16;
  const int* sv = nullptr;
  const float* Vk = V_half;
  if (n > 0) {
    const unsigned long long* sk = gr.sorted_keys_alt ? x.k1 : x.k0;
    sv = gr.sorted_vals_alt ? x.v1 : x.v0;
    // 5. V in the keyed layout (full grid: conjugate-completed signed set)
    if (!p.mirror) {
      k_expand_half<<<g, 256, 0, st>>>(V_half, p.n_half_total, nbl, x.Vfull);
      VB_LAUNCH_CHECK();
      Vk = x.Vfull;
    }
    // 6. group records
    RecArgs r{};
    r.skeys = sk; r.svals = sv; r.start = x.start; r.ngroups = x.ngroups; r.sp = x.sp; r.V = Vk;
    r.x1 = bl->x1; r.y1 = bl->y1; r.z1 = bl->z1; r.in1 = bl->invn1;
    r.x2 = bl->x2; r.y2 = bl->y2; r.z2 = bl->z2; r.in2 = bl->invn2;
    r.cp1 = bl->cosphi1; r.cp2 = bl->cosphi2; r.cosphi = bl->cosphi;
    r.nbl = nbl; r.mirror = p.mirror; r.blockage = p.blockage; r.occ_mode = p.occ_mode;
    r.rec = x.rec; r.meta = x.meta; r.err = x.err;
    k_group_records<<<g, 256, 0, st>>>(r, n);
    VB_LAUNCH_CHECK();
  }
  // 7. block cones (unless the caller already holds them)
  if (p.cull == VB_CULL_EXACT && !(pre && pre->cones_ready))
    VB_TRY(geom_exact_cones(p.block_pix, sky->l, sky->m, sky->n, p.npix, x.cones, st));
  // 8. reconstruction over (pixel block x group chunk)
  if (n > 0) {
    ReconArgs ra{};
    ra.l = sky->l; ra.m = sky->m; ra.n = sky->n; ra.npix = p.npix;
    ra.block_pix = p.block_pix; ra.nblocks = p.nblocks; ra.nchunk_target = p.nchunk_target;
    ra.ngroups = x.ngroups; ra.rec = x.rec; ra.meta = x.meta; ra.sp = x.sp; ra.svals = sv; ra.V = Vk;
    ra.x1 = bl->x1; ra.y1 = bl->y1; ra.z1 = bl->z1; ra.in1 = bl->invn1;
    ra.x2 = bl->x2; ra.y2 = bl->y2; ra.z2 = bl->z2; ra.in2 = bl->invn2;
    ra.cp1 = bl->cosphi1; ra.cp2 = bl->cosphi2; ra.cosphi = bl->cosphi;
    ra.nbl = nbl; ra.mirror = p.mirror; ra.blockage = p.blockage; ra.occ_mode = p.occ_mode; ra.cull = p.cull;
    ra.finite_check = p.mirror ? 0 : 1;
    ra.cones = x.cones; ra.queue = x.queue; ra.Cpart = x.Cpart; ra.Wpart = x.Wpart;
    ra.counters = counters; ra.err = x.err;
    const bool members = p.blockage && p.occ_mode != 2;
    VB_CUDA(cudaMemsetAsync(x.queue, 0, sizeof(int), st));
    if (kbeg) VB_CUDA(record_event(kbeg, st));
    switch (p.precision) {
      case VB_PREC_REF32: VB_TRY(launch_recon<VB_PREC_REF32>(ra, members, p.ppt, st)); break;
      case VB_PREC_FP64: VB_TRY(launch_recon<VB_PREC_FP64>(ra, members, p.ppt, st)); break;
      case VB_PREC_FP32_FP64PH: VB_TRY(launch_recon<VB_PREC_FP32_FP64PH>(ra, members, p.ppt, st)); break;
      default: VB_TRY(launch_recon<VB_PREC_FP32_DSPH>(ra, members, p.ppt, st)); break;
    }
    if (kend) VB_CUDA(record_event(kend, st));
  } else if (kbeg) {
    VB_CUDA(record_event(kbeg, st));
    VB_CUDA(record_event(kend, st));
  }
  // 9. finalize: sum the group-chunk partials, normalise
  int gf = (int)ceil_div(p.npix, 256);
  if (gf > sm_count() * 16) gf = sm_count() * 16;
  k_finalize<<<gf, 256, 0, st>>>(x.Cpart, x.Wpart, x.ngroups, p.nchunk_target, p.npix, p.blockage, C, W, x.wsum);
  VB_LAUNCH_CHECK();
  if (seg_params_out)
    VB_CUDA(cudaMemcpyAsync(seg_params_out, x.sp, nseg * sizeof(vb_seg_params), cudaMemcpyDeviceToDevice, st));
  if (w_scalar_total) VB_CUDA(cudaMemcpyAsync(w_scalar_total, x.wsum, sizeof(double), cudaMemcpyDeviceToDevice, st));
  return VB_OK;
}

int stage2_run(const vb_sky* sky, const vb_baselines* bl, const float* V_half, int nseg, const int* seg_t0,
               const int* seg_tlen, const Stage2Plan& p, void* ws, size_t cap, float* C, uint32_t* W,
               vb_seg_params* seg_params_out, unsigned long long* counters, double* w_scalar_total, cudaStream_t st,
               const Stage2Pixels* pre, cudaEvent_t kbeg, cudaEvent_t kend) {
  Stage2Groups gr;
  VB_TRY(stage2_group(bl, nseg, seg_t0, seg_tlen, p, ws, cap, st, &gr));
  return stage2_finish(sky, bl, V_half, nseg, p, ws, cap, gr, C, W, seg_params_out, counters, w_scalar_total, st,
                       pre, kbeg, kend);
}

}  // namespace vb

using namespace vb;

extern "C" int vb_fa_fb_host(const float* u, const float* v, const float* w, int n, float* fa, float* fb,
                             double* denom_out) {
  if (n < 0 || (n > 0 && (!u || !v || !w)) || !fa || !fb) return fail(VB_ERR_INVALID, "vb_fa_fb_host: bad args");
  // long double sums as viss_recon_kernel.cuh:673-701
  long double su2 = 0, sv2 = 0, suv = 0, suw = 0, svw = 0;
  for (int i = 0; i < n; i++) {
    long double uu = (long double)u[i];
    long double vv = (long double)v[i];
    long double ww = (long double)w[i];
    su2 += uu * uu;
    sv2 += vv * vv;
    suv += uu * vv;
    suw += uu * ww;
    svw += vv * ww;
  }
  long double denom = su2 * sv2 - suv * suv;
  if (denom_out) *denom_out = (double)denom;
  long double scale = (su2 * sv2 > 0) ? (su2 * sv2) : 1.0L;
  long double eps = 1e-24L * scale;
  if (!std::isfinite((double)denom) || fabsl(denom) < eps) {
    long double sign = (denom >= 0) ? 1.0L : -1.0L;
    denom = sign * eps;
  }
  long double a = (sv2 * suw - suv * svw) / denom;
  long double b = (su2 * svw - suv * suw) / denom;
  if (!std::isfinite((double)a) || !std::isfinite((double)b)) { a = 0; b = 0; }
  *fa = (float)a;
  *fb = (float)b;
  return VB_OK;
}

extern "C" int vb_grid_params(float fa, float fb, float bl_max, float lambda, int grid_res, int* RES_out,
                              int* half_out, float* du_out) {
  if (!(lambda > 0.f) || !(bl_max > 0.f)) return fail(VB_ERR_INVALID, "vb_grid_params: lambda/bl_max must be > 0");
  int RES;
  if (grid_res > 0) {
    RES = (grid_res % 2 == 0) ? grid_res + 1 : grid_res;
  } else {
    volatile float lmax = std::sqrt(1.0f + fa * fa);
    volatile float mmax = std::sqrt(1.0f + fb * fb);
    float lmmax = std::max((float)lmax, (float)mmax);
    volatile float temp_res = std::ceil(2.0f * bl_max / lambda * 2.0f * lmmax);
    RES = (int)(temp_res + 2 + 1 - std::fmod((float)temp_res, 2.0f));
  }
  if (RES < 3) return fail(VB_ERR_INVALID, "vb_grid_params: RES=%d", RES);
  if (RES_out) *RES_out = RES;
  if (half_out) *half_out = (RES - 1) / 2;
  if (du_out) *du_out = 2.0f * bl_max / lambda / (RES - 1);
  return VB_OK;
}

__global__ void k_keys_plain(const float* __restrict__ u, const float* __restrict__ v, int n, int nbl, int mirror,
                             float inv_du, int RES, int half, int* __restrict__ keys) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (mirror) {
      const int f = half_to_full_pos(i, nbl);
      keys[i] = uv_key_half(u[f], v[f], inv_du, RES, half);
    } else {
      keys[i] = uv_key_full(u[i], v[i], inv_du, RES, half);
    }
  }
}

extern "C" int vb_build_keys(const float* u_full, const float* v_full, int n, int nbl, int mirror, float inv_du,
                             int RES, int half, int* keys, void* stream) {
  if (n < 0 || nbl <= 0 || RES <= 0) return fail(VB_ERR_INVALID, "vb_build_keys: n=%d nbl=%d RES=%d", n, nbl, RES);
  if (n == 0) return VB_OK;
  if (!u_full || !v_full || !keys) return fail(VB_ERR_INVALID, "vb_build_keys: null pointer");
  int g = (int)ceil_div(n, 256);
  if (g > sm_count() * 16) g = sm_count() * 16;
  k_keys_plain<<<g, 256, 0, as_stream(stream)>>>(u_full, v_full, n, nbl, mirror ? 1 : 0, inv_du, RES, half, keys);
  VB_LAUNCH_CHECK();
  return VB_OK;
}

extern "C" size_t vb_stage2_workspace_bytes(int n_half_total, int nseg, int64_t npix, const vb_stage2_opts* o) {
  Stage2Plan p{};
  if (stage2_plan(n_half_total, nseg, npix, o, &p) != VB_OK) return 0;
  return stage2_workspace(p, nullptr, 0, nullptr);
}

extern "C" int vb_recon_batched(const vb_sky* sky, const vb_baselines* bl, const float* V_half, int nseg,
                                const int* seg_t0, const int* seg_tlen, const vb_stage2_opts* o, void* workspace,
                                size_t ws_bytes, float* C, uint32_t* W, vb_seg_params* seg_params,
                                unsigned long long* term_counters, void* stream) {
  if (!sky || !bl || !o) return fail(VB_ERR_INVALID, "vb_recon_batched: null argument");
  if (bl->nbl <= 0 || bl->n_full % (2 * bl->nbl) != 0) return fail(VB_ERR_INVALID, "vb_recon_batched: n_full/nbl");
  if (!C || !V_half || !seg_t0 || !seg_tlen) return fail(VB_ERR_INVALID, "vb_recon_batched: null buffer");
  Stage2Plan p{};
  VB_TRY(stage2_plan(bl->n_full / 2, nseg, sky->npix, o, &p));
  size_t need = stage2_workspace(p, nullptr, 0, nullptr);
  if (!workspace || ws_bytes < need) return fail(VB_ERR_NOMEM, "vb_recon_batched: workspace %zu < %zu", ws_bytes, need);
  if (reinterpret_cast<uintptr_t>(workspace) % 256 != 0)
    return fail(VB_ERR_INVALID, "vb_recon_batched: workspace %p is not 256-byte aligned", workspace);
  return stage2_run(sky, bl, V_half, nseg, seg_t0, seg_tlen, p, workspace, ws_bytes, C, W, seg_params, term_counters,
                    nullptr, as_stream(stream), nullptr);
}

extern "C" int vb_stage2(const vb_sky* sky, const vb_baselines* bl, const float* V_half, int nseg,
                         const int* seg_t0, const int* seg_tlen, const vb_stage2_opts* o, void* workspace,
                         size_t ws_bytes, float* C, uint32_t* W, void* stream) {
  return vb_recon_batched(sky, bl, V_half, nseg, seg_t0, seg_tlen, o, workspace, ws_bytes, C, W, nullptr,
                          nullptr, stream);
}
