// Stage 1: half-conjugate visibility sum
//   V[ih] = sum_p B_p * occ_a(p) * occ_b(p) * exp(-2 pi i t(ih, p)),
//   t = u l + v m + w (n - 1)        (phase_corrected = 0, as the upstream kernel)
//   t = u l + v m + w n              (phase_corrected = 1, = upstream V after
//                                     phase_correct_viss_halfsym_host)
// Upstream: viss_partial_all_halfsym<256,true> (viss_recon_kernel.cuh:200-287)
// and viss_partial_all_halfsym_tilecone<TILE,true>
// (viss_recon_kernel_mirror_tile_vissfast.cuh:437-561).
//
// B200 design: persistent CTAs pull (baseline tile x pixel chunk) items from a
// device counter; each thread owns BPT half-baselines; pixels are staged in
// shared memory as FP64 (l, m), (n, B) and FP32 (l, m, n, B) records and read
// as warp-broadcasts.  Per pixel tile each warp takes one of three paths
// (skip / unmasked / masked) from its lanes' tile classes, so the hot loop is
// warp-uniform.  Partial sums per chunk are reduced in a fixed order
// (deterministic).
//
// Precision modes (the `MODE` template argument):
//   REF32  : FP32 phase (upstream arithmetic), FP32 sincos, FP32 stage sums.
//   FP64   : FP64 phase, FP64 sincos, FP64 sums (the plain FP64 direct sum).
//   F32X   : phase formed in FP64 with a magic-constant range reduction: the
//            turn fraction lands in the low 23 bits of the double and becomes
//            an exact FP32 angle in [0, 2pi); FP32 sincos; FP32
//            sums per staged tile (<= 1024 terms), FP64 across tiles.
//   DS     : each product split exactly (p = fl(a b), e = fma(a, b, -p)),
//            fractions p - rint(p) exact in FP32; FP32 sincos; Kahan sums
//            across tiles.
#include <cmath>
#include <algorithm>
#include <type_traits>

#include "vb_common.cuh"
#include "vb_geom.cuh"
#include "vb_internal.h"

namespace vb {

constexpr int S1_THREADS = 256;
constexpr int kClsHid = 0, kClsVis = 1, kClsMix = 2;
// Kernel-internal cull variant: tile-cone culling whose visible tiles still take
// the per-pixel test (vb_stage1_opts.mask_visible_tiles).  A template value of
// its own, so that the default tile-cone kernel carries no extra test.
constexpr int kCullTileconeMV = 3;
template <int CULL>
__host__ __device__ constexpr bool is_tilecone() { return CULL == VB_CULL_TILECONE || CULL == kCullTileconeMV; }

// F32X phase reduction: magic = 1.5 * 2^29 keeps every partial sum of the FMA
// chain in [2^29, 2^30) (|u| + |v| + |w| < 2^28); the double's ulp is then
// 2^-23 turns, so each FMA rounds to nearest on the 2^-23-turn grid the FP32
// angle is built on, and the low 23 bits of the double are the turn fraction:
// one LOP3 turns them into the exact float 2^23 + k.
constexpr double kMagic = 805306368.0;              // 1.5 * 2^29
constexpr float kTwoPiF = 6.28318530717958647692f;
constexpr float kAngScale = 6.28318530717958647692f * 1.1920928955078125e-7f;  // fl(2pi) * 2^-23
constexpr double kMaxUvwF32X = 67108864.0;         // 2^26: 3 * 2^26 < 2^28

struct S1Args {
  const PixRec* __restrict__ px;   // stage-1 pixel records (interleaved, one per pixel)
  int64_t npix;
  int cull, cull_tile, stage_pix, chunk_pix, nchunk, n_btile, n_items;
  const float *tcx, *tcy, *tcz, *tcosA, *tsinA;   // VB_CULL_TILECONE
  const ExactCone* cones;                          // VB_CULL_EXACT
  const ExactCone* subcones;                       // tile-cone refinement: cones of refine_pix sub-tiles
  int refine_pix;                                  // 0: no refinement
  int mask_visible;                                // tile-cone: visible tiles take the per-pixel test
  const float *u, *v, *w, *x1, *y1, *z1, *in1, *x2, *y2, *z2, *in2, *cp1, *cp2;
  float cosphi;
  int n_half, nbl, blockage, phase_corrected;
  int* queue;
  double2* partial;
  unsigned long long* counters;
  unsigned* err;
};


struct Baseline {
  double U, V, W, C;
  float uf, vf, wf, fw;   // FP32 copies; fw = -frac(w) (raw phase, DS)
  float ku, kv, kw;       // REF32: -2 pi * (u, v, w)
  float x1, y1, z1, i1, x2, y2, z2, i2, c1, c2;
  float t1, t2;   // occ_threshold of (i1, c1), (i2, c2)
  float ux1, uy1, uz1, ux2, uy2, uz2;
  int cls;    // class the pixel loop uses (tile class, or the sub-tile class when refined)
  int tcls;   // tile class (decides whether the staged partials are kept)
  bool active;
};

__device__ __forceinline__ float rint_magic(float x) {
  return __fsub_rn(__fadd_rn(x, 12582912.0f), 12582912.0f);
}

// VB_CULL_EXACT class of one baseline for one tile.  Kept out of line: the
// FP64 cone test runs once per (baseline, tile), and inlining it into the
// persistent kernel costs the pixel loop registers in every cull mode.  It
// uses the FP64 form of the test: with the square-root-free form the kernel
// ran 8 % slower (out of line) or 15 % slower (inlined) with the same
// decisions.
__device__ __noinline__ int exact_tile_class(const ExactCone* cone, float x1, float y1, float z1, float i1, float c1,
                                             float x2, float y2, float z2, float i2, float c2) {
  const ExactCone c = *cone;
  const int e1 = exact_class_fp64(c, x1, y1, z1, i1, c1);
  const int e2 = exact_class_fp64(c, x2, y2, z2, i2, c2);
  return (e1 < 0 || e2 < 0) ? kClsHid : ((e1 > 0 && e2 > 0) ? kClsVis : kClsMix);
}

// Tile class of one baseline for one cull tile (0 hidden, 1 visible, 2 mixed).
// Upstream decision: ..._vissfast.cuh:519-531 (tile cone), per-pixel mask
// everywhere for the plain kernel (viss_recon_kernel.cuh:270-274).  The cull
// mode is a template argument so that each mode's kernel carries only its own
// test.
template <int CULL>
__device__ __forceinline__ int tile_class(const S1Args& a, const Baseline& b, int tile_id) {
  if (!b.active) return kClsHid;
  if (!a.blockage) return kClsVis;
  if constexpr (is_tilecone<CULL>()) {
    const float cx = a.tcx[tile_id], cy = a.tcy[tile_id], cz = a.tcz[tile_id];
    const float cA = a.tcosA[tile_id], sA = a.tsinA[tile_id];
    bool vis1, hid1, vis2, hid2;
    cone_classify(cone_dot(b.ux1, b.uy1, b.uz1, cx, cy, cz), cA, sA, b.c1, vis1, hid1);
    cone_classify(cone_dot(b.ux2, b.uy2, b.uz2, cx, cy, cz), cA, sA, b.c2, vis2, hid2);
    return (hid1 || hid2) ? kClsHid : ((vis1 && vis2 && CULL != kCullTileconeMV) ? kClsVis : kClsMix);
  } else if constexpr (CULL == VB_CULL_EXACT) {
    return exact_tile_class(a.cones + tile_id, b.x1, b.y1, b.z1, b.i1, b.c1, b.x2, b.y2, b.z2, b.i2, b.c2);
  } else {
    return kClsMix;
  }
}

__device__ __forceinline__ int tile_class_rt(const S1Args& a, const Baseline& b, int tile_id) {
  if (a.cull == VB_CULL_TILECONE)
    return a.mask_visible ? tile_class<kCullTileconeMV>(a, b, tile_id) : tile_class<VB_CULL_TILECONE>(a, b, tile_id);
  if (a.cull == VB_CULL_EXACT) return tile_class<VB_CULL_EXACT>(a, b, tile_id);
  return tile_class<VB_CULL_NONE>(a, b, tile_id);
}

// Loads half-baseline ih into registers (upstream: viss_recon_kernel.cuh:231-240,
// ..._vissfast.cuh:476-497).

// Per-endpoint threshold of the per-pixel occlusion test: the test
// "fl(d * invn) < cosphi" (d the FP32 dot of pixel and endpoint, rounded as
// occ_dot rounds it) holds exactly when d < t, t being the smallest float with
// fl(t * invn) >= cosphi: fl(d * invn) does not decrease as d grows (invn > 0).
// The masked path then compares d with t instead of multiplying first, with
// the same masks (two multiplies fewer per masked term: 1217.7 -> 1206.1 ms on
// the nside-1024 day, 9.66 -> 9.64 ms at nside 256).
__device__ __noinline__ float occ_threshold(float invn, float c) {
  if (c != c || invn != invn) return -INFINITY;                  // the test never fails
  if (invn == 0.0f) return c > 0.0f ? INFINITY : -INFINITY;      // fl(d * 0) = 0 against c
  if (isinf(invn)) return 0.0f;                                  // d * inf: fails exactly for d < 0
  float t = c / invn;                                            // within a few ulps; fixed below
  for (int k = 0; k < 16 && !(t * invn >= c); ++k) t = nextafterf(t, INFINITY);
  for (int k = 0; k < 16; ++k) {
    const float p = nextafterf(t, -INFINITY);
    if (p * invn >= c) t = p; else break;
  }
  return t;
}

__device__ __forceinline__ void load_baseline(const S1Args& a, int ih, bool raw, Baseline& b) {
  b.active = ih < a.n_half;
  const int i = b.active ? half_to_full_pos(ih, a.nbl) : 0;
  float uu = b.active ? a.u[i] : 0.f, vv = b.active ? a.v[i] : 0.f, ww = b.active ? a.w[i] : 0.f;
  b.uf = uu; b.vf = vv; b.wf = ww;
  b.U = uu; b.V = vv; b.W = ww;
  b.C = kMagic - (raw ? (double)ww : 0.0);
  b.fw = raw ? -__fsub_rn(ww, rint_magic(ww)) : 0.0f;
  const float kk = -2.0f * 3.14159265358979323846f;
  b.ku = kk * uu; b.kv = kk * vv; b.kw = kk * ww;
  if (a.blockage && b.active) {
    b.x1 = a.x1[i]; b.y1 = a.y1[i]; b.z1 = a.z1[i]; b.i1 = a.in1[i];
    b.x2 = a.x2[i]; b.y2 = a.y2[i]; b.z2 = a.z2[i]; b.i2 = a.in2[i];
    b.c1 = a.cp1 ? a.cp1[i] : a.cosphi;
    b.c2 = a.cp2 ? a.cp2[i] : a.cosphi;
  } else {
    b.x1 = b.y1 = b.z1 = b.i1 = b.x2 = b.y2 = b.z2 = b.i2 = 0.f;
    b.c1 = b.c2 = a.cosphi;
  }
  b.t1 = occ_threshold(b.i1, b.c1);
  b.t2 = occ_threshold(b.i2, b.c2);
  b.ux1 = b.x1 * b.i1; b.uy1 = b.y1 * b.i1; b.uz1 = b.z1 * b.i1;
  b.ux2 = b.x2 * b.i2; b.uy2 = b.y2 * b.i2; b.uz2 = b.z2 * b.i2;
  b.cls = b.tcls = kClsHid;
}

// Half-turn dithering (FP32 modes): MUFU sin/cos carry a small mean error over
// the angle range, which a sum over ~1e6 pixels would add coherently.  Odd
// pixels are evaluated half a turn further on and their partial sums are
// subtracted (exp(i(t + pi)) = -exp(i t)), so the two parities' mean errors
// cancel.  PAR = 1 selects the shifted evaluation.
template <int MODE>
__device__ constexpr bool pixel_dither() {
  return MODE == VB_PREC_FP32_FP64PH || MODE == VB_PREC_FP32_DSPH;
}

template <int MODE, int PAR>
__device__ __forceinline__ void phase_sincos(const Baseline& b, const double2 lm, const double nd,
                                             const float4 f, const float nm1, float& s, float& c,
                                             double& sd, double& cd, bool raw) {
  if constexpr (MODE == VB_PREC_FP32_FP64PH) {
    double t = fma(b.U, lm.x, fma(b.V, lm.y, fma(b.W, nd, b.C)));
    const unsigned lo = (unsigned)__double2loint(t);
    // (lo & M) has no bits above 22: OR with the exponent bits is an XOR, and
    // the odd pixels' half turn (bit 22) folds into the same constant
    const unsigned kb = (lo & 0x7FFFFFu) ^ (PAR ? 0x4B400000u : 0x4B000000u);
    float ang = __fmaf_rn(__uint_as_float(kb), kAngScale, -kTwoPiF);
    __sincosf(ang, &s, &c);
  } else if constexpr (MODE == VB_PREC_FP32_DSPH) {
    float p1 = __fmul_rn(b.uf, f.x), e1 = __fmaf_rn(b.uf, f.x, -p1);
    float p2 = __fmul_rn(b.vf, f.y), e2 = __fmaf_rn(b.vf, f.y, -p2);
    float p3 = __fmul_rn(b.wf, f.z), e3 = __fmaf_rn(b.wf, f.z, -p3);
    float f1 = __fsub_rn(p1, rint_magic(p1));
    float f2 = __fsub_rn(p2, rint_magic(p2));
    float f3 = __fsub_rn(p3, rint_magic(p3));
    float sfr = __fadd_rn(__fadd_rn(f1, f2), __fadd_rn(f3, b.fw));
    float efr = __fadd_rn(__fadd_rn(e1, e2), e3);
    float t = __fadd_rn(sfr, efr);
    t = __fsub_rn(t, rint_magic(t));
    if constexpr (PAR) {
      t = __fadd_rn(t, 0.5f);
      t = __fsub_rn(t, rint_magic(t));
    }
    // angle in [0, 2 pi) as in F32X: at |uvw| ~ 2e5 this halves the C error
    // against an angle in [-pi, pi) (measured; the phase itself is exact to ~1e-8 turns)
    t = (t < 0.f) ? __fadd_rn(t, 1.0f) : t;
    __sincosf(__fmul_rn(t, kTwoPiF), &s, &c);
  } else if constexpr (MODE == VB_PREC_REF32) {
    float ang = raw ? fmaf(b.kw, nm1, fmaf(b.kv, f.y, b.ku * f.x))
                    : fmaf(b.kw, f.z, fmaf(b.kv, f.y, b.ku * f.x));
    __sincosf(ang, &s, &c);
  } else {  // FP64
    double t = fma(b.U, lm.x, fma(b.V, lm.y, b.W * (raw ? (nd - 1.0) : nd)));
    sincos(-6.283185307179586476925286766559 * t, &sd, &cd);
  }
}

// Imaginary-part sign of the accumulated sums: F32X/DS accumulate sin(+2 pi t).
template <int MODE>
__device__ constexpr float imag_sign() {
  return (MODE == VB_PREC_FP32_FP64PH || MODE == VB_PREC_FP32_DSPH) ? -1.0f : 1.0f;
}

// --- bulk-copy staging --------------------------------------------------------
// One thread copies a stage's records (a contiguous range of the interleaved
// global array) into this CTA's own shared memory with cp.async.bulk, which
// signals an mbarrier when the bytes have landed; the other buffer is filled
// while the CTA computes on this one.  No cluster multicast: the source is
// always this GPU's own memory and the destination this CTA's shared memory.
// (Measured on one B200 against the cooperative loads it replaced, which
// staged through registers between two barriers per stage: 1231 against 1248
// ms on the nside-1024 day, 9.72 against 9.80 ms at nside 256.)
__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void bulk_stage_issue(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
  // shared memory the threads read before the preceding barrier is written by
  // the async proxy next: order the two proxies
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_addr(dst)),
               "l"(src), "r"(bytes), "r"(smem_addr(bar))
               : "memory");
}
// Waits for the phase `parity` of the barrier to complete, at most kBulkWaitTries
// polls; a wait that runs out sets ERR_WAIT_TIMEOUT (the outputs of the call
// are then not to be trusted) and returns.
constexpr int kBulkWaitTries = 1 << 22;
__device__ __forceinline__ void bulk_stage_wait(unsigned long long* bar, unsigned parity, unsigned* err) {
  for (int i = 0; i < kBulkWaitTries; ++i) {
    unsigned done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    if (done) return;
  }
  atomicOr(err, ERR_WAIT_TIMEOUT);
}

// Register budget per thread: 80 for 3 resident CTAs of 256 threads; 120 for
// 2 (measured: 120 beats the full 128 the 2-CTA budget allows by ~2 % on the
// nside-256 workload, 112 and below lose more to the extra scheduling limits).
template <int MODE, int BPT, int MINB, int CULL>
__global__ void __maxnreg__(MINB == 3 ? 80 : 120) k_stage1(const S1Args a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  PixRec* s_px = reinterpret_cast<PixRec*>(smem_raw);
  __shared__ int s_item;
  __shared__ unsigned long long s_cnt[4];
  __shared__ unsigned long long s_bar[2];   // one mbarrier per staging buffer

  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const bool raw = (a.phase_corrected == 0);
  constexpr bool kDoubleAcc = (MODE == VB_PREC_FP64);

  if (threadIdx.x < 4) s_cnt[threadIdx.x] = 0ull;
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&s_bar[0])) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&s_bar[1])) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  // Staging state; every thread keeps its own copy and takes the same
  // (CTA-uniform) decisions, thread 0 alone issues the copies.  Each issued
  // copy is waited for exactly once, so the parity bits stay in step with the
  // barriers' phases.
  unsigned bar_parity = 0;   // bit b: parity of the next completion of buffer b's barrier
  auto stage_wait = [&](int b) {
    bulk_stage_wait(&s_bar[b], (bar_parity >> b) & 1u, a.err);
    bar_parity ^= 1u << b;
  };
  auto stage_issue = [&](int b, int64_t p0, int64_t p1) {   // records [p0, min(p0 + stage, p1)) into buffer b
    if (threadIdx.x == 0) {
      const int ns = (int)((p1 - p0) < a.stage_pix ? (p1 - p0) : a.stage_pix);
      bulk_stage_issue(s_px + (size_t)b * a.stage_pix, a.px + p0, (unsigned)(ns * sizeof(PixRec)), &s_bar[b]);
    }
  };

  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) s_item = atomicAdd(a.queue, 1);
    __syncthreads();
    const int item = s_item;
    if (item >= a.n_items) break;
    // chunk-major order: the CTAs running at one time share a pixel chunk,
    // which then stays in L2 while they stage it
    const int chunk = item / a.n_btile;
    const int btile = item - chunk * a.n_btile;

    // --- per-thread baselines -------------------------------------------------
    Baseline bl[BPT];
#pragma unroll
    for (int k = 0; k < BPT; ++k) {
      Baseline& b = bl[k];
      const int ih = btile * (S1_THREADS * BPT) + warp * (32 * BPT) + k * 32 + lane;
      load_baseline(a, ih, raw, b);
      const float uu = b.uf, vv = b.vf, ww = b.wf;
      if (MODE == VB_PREC_FP32_FP64PH && b.active &&
          (fabsf(uu) >= (float)kMaxUvwF32X || fabsf(vv) >= (float)kMaxUvwF32X ||
           fabsf(ww) >= (float)kMaxUvwF32X))
        atomicOr(a.err, ERR_PHASE_RANGE);
    }

    double accR[BPT], accI[BPT];
    float kcR[BPT], kcI[BPT];   // Kahan compensation (DS)
#pragma unroll
    for (int k = 0; k < BPT; ++k) { accR[k] = 0.0; accI[k] = 0.0; kcR[k] = 0.f; kcI[k] = 0.f; }

    unsigned long long cnt_fast = 0, cnt_mask = 0, cnt_hid = 0, cnt_all = 0;
    int nact = 0;
#pragma unroll
    for (int k = 0; k < BPT; ++k) nact += __popc(__ballot_sync(0xffffffffu, bl[k].active));

    const int64_t p_begin = (int64_t)chunk * a.chunk_pix;
    int64_t p_end = p_begin + a.chunk_pix;
    if (p_end > a.npix) p_end = a.npix;

    for (int64_t t0 = p_begin; t0 < p_end; t0 += a.cull_tile) {
      int64_t t1 = t0 + a.cull_tile;
      if (t1 > p_end) t1 = p_end;
      const int tile_id = (int)(t0 / a.cull_tile);

      // --- tile classes of this thread's baselines ----------------------------
      bool any_live = false, any_mix = false;
#pragma unroll
      for (int k = 0; k < BPT; ++k) {
        Baseline& b = bl[k];
        const int cls = tile_class<CULL>(a, b, tile_id);
        b.cls = b.tcls = cls;
        any_live |= (cls != kClsHid);
        any_mix |= (cls == kClsMix);
      }
      const bool warp_live = __any_sync(0xffffffffu, any_live);
      const bool warp_mix = __any_sync(0xffffffffu, any_mix);
      // mixed tiles refined into exact sub-tiles count their terms per sub-tile
      const bool refine = is_tilecone<CULL>() && warp_mix && a.refine_pix > 0;
      const int64_t tile_terms = (int64_t)nact * (t1 - t0);
      cnt_all += tile_terms;
      if (!warp_live) cnt_hid += tile_terms;
      else if (!warp_mix) cnt_fast += tile_terms;
      else if (!refine) cnt_mask += tile_terms;

      // (a CTA-wide barrier: every thread is done with the staged records of
      // the previous tile, so both buffers are free)
      if (!__syncthreads_or(warp_live ? 1 : 0)) continue;
      stage_issue(0, t0, t1);

      int si = 0;   // stage si of the tile sits in buffer si & 1
      for (int64_t s0 = t0; s0 < t1; s0 += a.stage_pix, ++si) {
        const int ns = (int)((t1 - s0) < a.stage_pix ? (t1 - s0) : a.stage_pix);
        const int b = si & 1;
        // every thread is done with the other buffer (the previous stage); the
        // next stage of the tile goes there while this one is computed
        if (si > 0) __syncthreads();
        const int64_t s1 = s0 + a.stage_pix;
        if (s1 < t1) stage_issue(b ^ 1, s1, t1);
        stage_wait(b);
        const PixRec* sp = s_px + (size_t)b * a.stage_pix;
        if (!warp_live) continue;

        // two interleaved FP32 partial sums per baseline (even / odd pixels)
        float pR0[BPT], pI0[BPT], pR1[BPT], pI1[BPT];
        double dR[BPT], dI[BPT];
#pragma unroll
        for (int k = 0; k < BPT; ++k) {
          pR0[k] = pI0[k] = pR1[k] = pI1[k] = 0.f;
          dR[k] = dI[k] = 0.0;
        }

        // one pixel.  PATH 0: every baseline of the warp is included; 1: each
        // baseline by its class (visible or hidden, no per-pixel test); 2: the
        // per-pixel occlusion test for mixed baselines (visible ones included
        // unconditionally, hidden excluded)
        float e1[BPT], e2[BPT];   // thresholds with the class folded in (masked path)
        auto pixel = [&](const int j, float (&aR)[BPT], float (&aI)[BPT], auto path_tag, auto par_tag) {
          constexpr int PATH = decltype(path_tag)::value;
          constexpr bool MASKED = (PATH == 2);
          constexpr int PAR = decltype(par_tag)::value;
          const PixRec* rp = sp + j;
          const double2 lm = rp->lm;
          const float4 nb = rp->nb;
          const double nd = __hiloint2double(__float_as_int(nb.y), __float_as_int(nb.x));
          float4 f;
          if constexpr (MASKED || MODE == VB_PREC_FP32_DSPH || MODE == VB_PREC_REF32) f = rp->f4;
          else f = make_float4(0.f, 0.f, 0.f, nb.z);
          const float Bp = nb.z;
#pragma unroll
          for (int k = 0; k < BPT; ++k) {
            const Baseline& b = bl[k];
            bool inc = true;
            if constexpr (MASKED) {
              const float d1 = f.x * b.x1 + f.y * b.y1 + f.z * b.z1;
              const float d2 = f.x * b.x2 + f.y * b.y2 + f.z * b.z2;
              inc = !(d1 < e1[k] || d2 < e2[k]);
            } else if constexpr (PATH == 1) {
              inc = (b.cls != kClsHid);
            }
            float sn, cs;
            double sd, cd;
            phase_sincos<MODE, PAR>(b, lm, nd, f, nb.w, sn, cs, sd, cd, raw);
            if constexpr (kDoubleAcc) {
              const double Bw = inc ? (double)Bp : 0.0;
              dR[k] = fma(Bw, cd, dR[k]);
              dI[k] = fma(Bw, sd, dI[k]);
            } else {
              const float Bw = inc ? Bp : 0.0f;
              aR[k] = fmaf(Bw, cs, aR[k]);
              aI[k] = fmaf(Bw, sn, aI[k]);
            }
          }
        };
        using Unmasked = std::integral_constant<int, 0>;
        using Select = std::integral_constant<int, 1>;
        using Masked = std::integral_constant<int, 2>;
        using Even = std::integral_constant<int, 0>;
        using Odd = std::integral_constant<int, pixel_dither<MODE>() ? 1 : 0>;

        // pixels [j0, j1) of the staged tile (j0 even: pixel parity = index parity)
        auto run = [&](const int j0, const int j1, auto path_tag) {
          if constexpr (decltype(path_tag)::value == 2) {
            // masked path: fold each baseline's class into its thresholds, so
            // that inclusion is one pair of comparisons (visible: -inf, always
            // in; hidden: +inf, never in for a finite dot; a hidden class comes
            // only from cone tests on finite endpoints, whose dots are finite)
#pragma unroll
            for (int k = 0; k < BPT; ++k) {
              const int c = bl[k].cls;
              e1[k] = c == kClsMix ? bl[k].t1 : (c == kClsVis ? -INFINITY : INFINITY);
              e2[k] = c == kClsMix ? bl[k].t2 : (c == kClsVis ? -INFINITY : INFINITY);
            }
          }
          int j = j0;
          // two pixel pairs per trip: 0.5 % faster than the compiler's choice
          // (no unroll 1: +5 %, unroll 3 / 4: +5-6 %)
#pragma unroll 2
          for (; j + 1 < j1; j += 2) {
            pixel(j, pR0, pI0, path_tag, Even{});
            pixel(j + 1, pR1, pI1, path_tag, Odd{});
          }
          if (j < j1) pixel(j, pR0, pI0, path_tag, Even{});
        };

        if (!warp_mix) {
          run(0, ns, Unmasked{});
        } else if (refine) {
          // exact sub-tiles of a mixed tile: baselines the tile cone left mixed
          // are classified again per sub-tile, and each sub-tile takes the
          // cheapest path its warp allows; a term is included exactly when the
          // per-pixel test would include it, so the sums are unchanged
          for (int r0 = 0; r0 < ns; r0 += a.refine_pix) {
            const int r1 = (ns - r0) < a.refine_pix ? ns : r0 + a.refine_pix;
            const int sub_id = (int)((s0 + r0) / a.refine_pix);
            bool l_live = false, l_mix = false, l_newhid = false;
#pragma unroll
            for (int k = 0; k < BPT; ++k) {
              Baseline& b = bl[k];
              int e = b.tcls;
              if (e == kClsMix)
                e = exact_tile_class(a.subcones + sub_id, b.x1, b.y1, b.z1, b.i1, b.c1, b.x2, b.y2, b.z2, b.i2, b.c2);
              b.cls = e;
              l_live |= (e != kClsHid);
              l_mix |= (e == kClsMix);
              l_newhid |= (e == kClsHid && b.tcls != kClsHid);
            }
            const bool w_live = __any_sync(0xffffffffu, l_live);
            const bool w_mix = __any_sync(0xffffffffu, l_mix);
            const bool w_newhid = __any_sync(0xffffffffu, l_newhid);
            const int64_t sub_terms = (int64_t)nact * (r1 - r0);
            if (!w_live) cnt_hid += sub_terms;
            else if (w_mix) cnt_mask += sub_terms;
            else cnt_fast += sub_terms;
            if (!w_live) continue;
            if (w_mix) run(r0, r1, Masked{});
            else if (w_newhid) run(r0, r1, Select{});
            else run(r0, r1, Unmasked{});
          }
        } else {
          run(0, ns, Masked{});
        }
        // the odd-pixel sums were taken half a turn on: subtract them
        constexpr float kOddSign = pixel_dither<MODE>() ? -1.0f : 1.0f;

        // fold the staged-tile partials into the running totals
#pragma unroll
        for (int k = 0; k < BPT; ++k) {
          if (bl[k].tcls == kClsHid) continue;
          if constexpr (kDoubleAcc) {
            accR[k] += dR[k];
            accI[k] += dI[k];
          } else if constexpr (MODE == VB_PREC_FP32_DSPH) {
            // Kahan summation in FP32 across staged tiles
            float xr = __fmaf_rn(kOddSign, pR1[k], pR0[k]);
            float xi = __fmaf_rn(kOddSign, pI1[k], pI0[k]);
            float sr = (float)accR[k], si = (float)accI[k];
            float yr = __fsub_rn(xr, kcR[k]);
            float tr = __fadd_rn(sr, yr);
            kcR[k] = __fsub_rn(__fsub_rn(tr, sr), yr);
            float yi = __fsub_rn(xi, kcI[k]);
            float ti = __fadd_rn(si, yi);
            kcI[k] = __fsub_rn(__fsub_rn(ti, si), yi);
            accR[k] = tr;
            accI[k] = ti;
          } else {
            accR[k] += (double)pR0[k] + (double)kOddSign * (double)pR1[k];
            accI[k] += (double)pI0[k] + (double)kOddSign * (double)pI1[k];
          }
        }
      }
    }
#pragma unroll
    for (int k = 0; k < BPT; ++k) {
      const int ih = btile * (S1_THREADS * BPT) + warp * (32 * BPT) + k * 32 + lane;
      if (ih < a.n_half)
        a.partial[(int64_t)chunk * a.n_half + ih] =
            make_double2(accR[k], (double)imag_sign<MODE>() * accI[k]);
    }
    if (a.counters && lane == 0) {
      atomicAdd(&s_cnt[0], cnt_fast);
      atomicAdd(&s_cnt[1], cnt_mask);
      atomicAdd(&s_cnt[2], cnt_hid);
      atomicAdd(&s_cnt[3], cnt_all);
    }
  }
  __syncthreads();
  if (a.counters && threadIdx.x < 4) atomicAdd(&a.counters[threadIdx.x], s_cnt[threadIdx.x]);
}

// V[ih] = sum over chunks of the partials, in chunk order (accumulate: V += that sum).
__global__ void k_reduce_partials(const double2* __restrict__ partial, int nchunk, int n_half,
                                  double* __restrict__ V, int accumulate) {
  for (int ih = blockIdx.x * blockDim.x + threadIdx.x; ih < n_half; ih += gridDim.x * blockDim.x) {
    double r = 0.0, im = 0.0;
    for (int c = 0; c < nchunk; ++c) {
      double2 p = partial[(int64_t)c * n_half + ih];
      r += p.x;
      im += p.y;
    }
    if (accumulate) {
      V[2 * ih] += r;
      V[2 * ih + 1] += im;
    } else {
      V[2 * ih] = r;
      V[2 * ih + 1] = im;
    }
  }
}

// V *= exp(-2 pi i w) in FP64 with the exact turn fraction of w, then FP32
// half and conjugate-completed full layouts (common.hpp:255-277).
__global__ void k_phase_correct_expand(const double* __restrict__ Vr, const float* __restrict__ w,
                                       int n_half, int nbl, int already, float* __restrict__ Vh,
                                       float* __restrict__ Vf) {
  for (int ih = blockIdx.x * blockDim.x + threadIdx.x; ih < n_half; ih += gridDim.x * blockDim.x) {
    const int ip = half_to_full_pos(ih, nbl);
    double re = Vr[2 * ih], im = Vr[2 * ih + 1];
    if (!already) {
      double ww = (double)w[ip];
      double fr = ww - rint(ww);
      double s, c;
      sincospi(-2.0 * fr, &s, &c);
      double nr = re * c - im * s;
      double ni = re * s + im * c;
      re = nr;
      im = ni;
    }
    float fr_ = (float)re, fi_ = (float)im;
    if (Vh) { Vh[2 * ih] = fr_; Vh[2 * ih + 1] = fi_; }
    if (Vf) {
      Vf[2 * ip] = fr_;
      Vf[2 * ip + 1] = fi_;
      Vf[2 * (ip + nbl)] = fr_;
      Vf[2 * (ip + nbl) + 1] = -fi_;
    }
  }
}

// ---------------------------------------------------------------------------
// Kernel variants: precision x cull mode x baselines per thread x the
// resident-CTA count the register budget is built for (3 CTAs/SM = 80
// registers, only with BPT <= 2).
template <int MODE, int CULL>
static void* stage1_kernel(int bpt, int minb) {
  if (bpt == 1) return minb == 3 ? (void*)k_stage1<MODE, 1, 3, CULL> : (void*)k_stage1<MODE, 1, 2, CULL>;
  if (bpt == 2) return minb == 3 ? (void*)k_stage1<MODE, 2, 3, CULL> : (void*)k_stage1<MODE, 2, 2, CULL>;
  return (void*)k_stage1<MODE, 4, 2, CULL>;
}

template <int MODE>
static void* stage1_kernel_cull(int bpt, int minb, int cull) {
  if (cull == VB_CULL_TILECONE) return stage1_kernel<MODE, VB_CULL_TILECONE>(bpt, minb);
  if (cull == kCullTileconeMV) return stage1_kernel<MODE, kCullTileconeMV>(bpt, minb);
  if (cull == VB_CULL_EXACT) return stage1_kernel<MODE, VB_CULL_EXACT>(bpt, minb);
  return stage1_kernel<MODE, VB_CULL_NONE>(bpt, minb);
}

static void* stage1_kernel_of(int mode, int bpt, int minb, int cull) {
  switch (mode) {
    case VB_PREC_REF32: return stage1_kernel_cull<VB_PREC_REF32>(bpt, minb, cull);
    case VB_PREC_FP64: return stage1_kernel_cull<VB_PREC_FP64>(bpt, minb, cull);
    case VB_PREC_FP32_FP64PH: return stage1_kernel_cull<VB_PREC_FP32_FP64PH>(bpt, minb, cull);
    default: return stage1_kernel_cull<VB_PREC_FP32_DSPH>(bpt, minb, cull);
  }
}

static int occupancy(int mode, int bpt, int minb, int cull, size_t smem) {
  int n = 0;
  const void* kern = stage1_kernel_of(mode, bpt, minb, cull);
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return 1;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, S1_THREADS, smem) != cudaSuccess) return 1;
  return n < 1 ? 1 : n;
}

static bool is_pow2(int x) { return x > 0 && (x & (x - 1)) == 0; }

int stage1_plan(const vb_sky* sky, const vb_baselines* bl, const vb_stage1_opts* o, Stage1Plan* p) {
  if (!sky || !bl || !o || !p) return fail(VB_ERR_INVALID, "stage 1: null argument");
  if (sky->npix <= 0) return fail(VB_ERR_INVALID, "stage 1: npix=%lld", (long long)sky->npix);
  if (bl->nbl <= 0 || bl->n_full < 0 || bl->n_full % (2 * bl->nbl) != 0)
    return fail(VB_ERR_INVALID, "stage 1: n_full=%d must be a multiple of 2*nbl=%d", bl->n_full, 2 * bl->nbl);
  if (o->precision < VB_PREC_REF32 || o->precision > VB_PREC_FP32_DSPH)
    return fail(VB_ERR_INVALID, "stage 1: precision=%d", o->precision);
  if (o->cull < VB_CULL_NONE || o->cull > VB_CULL_EXACT) return fail(VB_ERR_INVALID, "stage 1: cull=%d", o->cull);
  Stage1Plan q{};
  q.precision = o->precision;
  q.cull = o->blockage ? o->cull : VB_CULL_NONE;
  q.phase_corrected = o->phase_corrected ? 1 : 0;
  q.blockage = o->blockage ? 1 : 0;
  q.bpt = o->bpt > 0 ? o->bpt : 2;
  if (q.bpt != 1 && q.bpt != 2 && q.bpt != 4) return fail(VB_ERR_INVALID, "stage 1: bpt=%d", q.bpt);
  q.minb = o->ctas_per_sm > 0 ? o->ctas_per_sm : 2;
  if (q.minb != 2 && !(q.minb == 3 && q.bpt <= 2))
    return fail(VB_ERR_INVALID, "stage 1: ctas_per_sm=%d (2, or 3 with bpt <= 2)", o->ctas_per_sm);
  if (o->items_per_cta < 0) return fail(VB_ERR_INVALID, "stage 1: items_per_cta=%d", o->items_per_cta);
  q.npix = sky->npix;
  q.n_half = bl->n_full / 2;
  q.nbl = bl->nbl;

  int stage = o->stage_pix > 0 ? o->stage_pix : 1024;
  if (!is_pow2(stage) || stage < 32 || stage > 2048)
    return fail(VB_ERR_INVALID, "stage 1: stage_pix=%d (power of two in [32, 2048])", stage);
  if (q.cull == VB_CULL_TILECONE) {
    if (!is_pow2(sky->tile_pix)) return fail(VB_ERR_INVALID, "stage 1: tile_pix=%d must be a power of two", sky->tile_pix);
    if (!sky->cx || !sky->cy || !sky->cz || !sky->cosA || !sky->sinA)
      return fail(VB_ERR_INVALID, "stage 1: tile-cone culling needs the tile meta arrays");
    q.cull_tile = sky->tile_pix;
    if (stage > q.cull_tile) stage = q.cull_tile;
  } else if (q.cull == VB_CULL_EXACT) {
    int et = o->exact_tile_pix > 0 ? o->exact_tile_pix : 1024;
    if (!is_pow2(et) || et < 32) return fail(VB_ERR_INVALID, "stage 1: exact_tile_pix=%d", et);
    q.cull_tile = et;
    if (stage > et) stage = et;
  } else {
    q.cull_tile = stage;
  }
  q.stage_pix = stage;
  q.ntile_cull = (int)ceil_div(q.npix, q.cull_tile);
  // tile-cone culling: exact sub-tiles inside mixed tiles (0 = automatic,
  // < 0 = off; on the nside-256 workload 128-pixel sub-tiles cut the masked
  // terms from 2.77e9 to 1.44e9 and the kernel time by 6 %).  Automatic: 256
  // pixels on cull tiles of 4096 and more, else 128 (measured on one B200,
  // 256 against 128: 1220.6 / 1231.9 ms on 16384-pixel tiles, 355.7 / 357.0 ms
  // on 4096, 9.76 / 9.72 ms and 23.62 / 23.55 ms on 1024)
  q.refine_pix = 0;
  q.mask_visible = (q.cull == VB_CULL_TILECONE && o->mask_visible_tiles) ? 1 : 0;
  if (q.cull == VB_CULL_TILECONE && o->refine_pix >= 0) {
    int r = o->refine_pix > 0 ? o->refine_pix : (q.cull_tile >= 4096 ? 256 : 128);
    if (!is_pow2(r) || r < 32) return fail(VB_ERR_INVALID, "stage 1: refine_pix=%d (power of two >= 32)", r);
    if (r < q.cull_tile && r <= q.stage_pix) q.refine_pix = r;
  }

  const int per_tile = S1_THREADS * q.bpt;
  q.n_btile = (int)ceil_div(q.n_half, per_tile);
  size_t smem = 2 * (size_t)stage * sizeof(PixRec);   // two staging buffers
  int occ = occupancy(q.precision, q.bpt, q.minb, q.mask_visible ? kCullTileconeMV : q.cull, smem);
  int capacity = sm_count() * occ;
  q.grid = capacity;
  // enough items per CTA that the dynamic queue's tail (one item) stays short
  // (96 per CTA measured against 48 / 24: 9.69 / 9.71 / 9.76 ms at nside 256,
  // 1219 / 1221 / 1237 ms at nside 1024)
  int64_t target_items = (int64_t)capacity * (o->items_per_cta > 0 ? o->items_per_cta : 96);
  int64_t nchunk = q.n_btile > 0 ? ceil_div(target_items, q.n_btile) : 1;
  int64_t max_chunks = ceil_div(q.npix, q.cull_tile);
  if (nchunk > max_chunks) nchunk = max_chunks;
  if (nchunk < 1) nchunk = 1;
  int64_t chunk = ceil_div(ceil_div(q.npix, nchunk), q.cull_tile) * q.cull_tile;
  if (o->chunk_pix > 0) {
    if (o->chunk_pix % q.cull_tile != 0)
      return fail(VB_ERR_INVALID, "stage 1: chunk_pix=%d must be a multiple of the cull tile %d", o->chunk_pix,
                  q.cull_tile);
    chunk = o->chunk_pix;
  }
  if (chunk > INT32_MAX) chunk = (INT32_MAX / q.cull_tile) * (int64_t)q.cull_tile;
  q.chunk_pix = (int)chunk;
  q.nchunk = (int)ceil_div(q.npix, q.chunk_pix);
  int64_t items = (int64_t)q.n_btile * q.nchunk;
  if (items > INT32_MAX) return fail(VB_ERR_UNSUPPORTED, "stage 1: too many work items");
  q.n_items = (int)items;
  if (q.grid > q.n_items) q.grid = q.n_items > 0 ? q.n_items : 1;
  *p = q;
  return VB_OK;
}

size_t stage1_carve(const Stage1Plan& p, void* ws, size_t cap, Stage1Buffers* b, bool pack_pixels) {
  Carve c(ws, cap);
  Stage1Buffers x;
  x.err = c.take<unsigned>(4);   // first: vb_workspace_error_flags reads it at offset 0
  if (pack_pixels) {
    x.px = c.take<PixRec>(p.npix);
    if (p.cull == VB_CULL_EXACT) x.cones = c.take<ExactCone>(p.ntile_cull);
    if (p.refine_pix > 0) x.subcones = c.take<ExactCone>((size_t)ceil_div(p.npix, p.refine_pix));
  }
  x.partial = c.take<double2>((size_t)p.nchunk * (size_t)p.n_half);
  x.queue = c.take<int>(4);
  if (b) *b = x;
  if (ws && !c.ok) return 0;
  return c.used();
}

int stage1_prepare_pixels(const vb_sky* sky, const Stage1Plan& p, const Stage1Buffers& b, cudaStream_t s) {
  VB_TRY(geom_pack_pixels(sky->B, sky->l, sky->m, sky->n, p.npix, b.px, s));
  if (p.cull == VB_CULL_EXACT) VB_TRY(geom_exact_cones(p.cull_tile, sky->l, sky->m, sky->n, p.npix, b.cones, s));
  if (p.refine_pix > 0) VB_TRY(geom_exact_cones(p.refine_pix, sky->l, sky->m, sky->n, p.npix, b.subcones, s));
  return VB_OK;
}

int stage1_run(const vb_sky* sky, const vb_baselines* bl, const Stage1Plan& p, const Stage1Buffers& b,
               bool pixels_ready, double* V_half, unsigned long long* counters, cudaStream_t s, cudaEvent_t kbeg,
               cudaEvent_t kend, bool accumulate) {
  if (p.n_half == 0) return VB_OK;
  if (!pixels_ready) VB_TRY(stage1_prepare_pixels(sky, p, b, s));
  S1Args a{};
  a.px = b.px;
  a.npix = p.npix;
  a.cull = p.cull; a.cull_tile = p.cull_tile; a.stage_pix = p.stage_pix; a.chunk_pix = p.chunk_pix;
  a.nchunk = p.nchunk; a.n_btile = p.n_btile; a.n_items = p.n_items;
  a.tcx = sky->cx; a.tcy = sky->cy; a.tcz = sky->cz; a.tcosA = sky->cosA; a.tsinA = sky->sinA;
  a.cones = b.cones;
  a.subcones = b.subcones;
  a.refine_pix = p.refine_pix;
  a.mask_visible = p.mask_visible;
  a.u = bl->u; a.v = bl->v; a.w = bl->w;
  a.x1 = bl->x1; a.y1 = bl->y1; a.z1 = bl->z1; a.in1 = bl->invn1;
  a.x2 = bl->x2; a.y2 = bl->y2; a.z2 = bl->z2; a.in2 = bl->invn2;
  a.cp1 = bl->cosphi1; a.cp2 = bl->cosphi2; a.cosphi = bl->cosphi;
  a.n_half = p.n_half; a.nbl = p.nbl; a.blockage = p.blockage; a.phase_corrected = p.phase_corrected;
  a.queue = b.queue; a.partial = b.partial; a.counters = counters; a.err = b.err;
  VB_CUDA(cudaMemsetAsync(b.queue, 0, sizeof(int), s));
  size_t smem = 2 * (size_t)p.stage_pix * sizeof(PixRec);
  const void* kern = stage1_kernel_of(p.precision, p.bpt, p.minb, p.mask_visible ? kCullTileconeMV : p.cull);
  VB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  void* args[] = {&a};
  if (kbeg) VB_CUDA(record_event(kbeg, s));
  VB_CUDA(cudaLaunchKernel(kern, dim3(p.grid), dim3(S1_THREADS), args, smem, s));
  if (kend) VB_CUDA(record_event(kend, s));
  int rg = (int)ceil_div(p.n_half, 256);
  if (rg > sm_count() * 16) rg = sm_count() * 16;
  k_reduce_partials<<<rg, 256, 0, s>>>(b.partial, p.nchunk, p.n_half, V_half, accumulate ? 1 : 0);
  VB_LAUNCH_CHECK();
  return VB_OK;
}

int phase_correct_expand_async(const double* Vraw, const float* w_full, int n_half, int nbl, int already,
                               float* Vh, float* Vf, cudaStream_t s) {
  if (n_half <= 0) return VB_OK;
  int g = (int)ceil_div(n_half, 256);
  if (g > sm_count() * 16) g = sm_count() * 16;
  k_phase_correct_expand<<<g, 256, 0, s>>>(Vraw, w_full, n_half, nbl, already, Vh, Vf);
  VB_LAUNCH_CHECK();
  return VB_OK;
}

}  // namespace vb

using namespace vb;

extern "C" size_t vb_stage1_workspace_bytes(const vb_sky* sky, const vb_baselines* bl, const vb_stage1_opts* o) {
  Stage1Plan p{};
  if (stage1_plan(sky, bl, o, &p) != VB_OK) return 0;
  return stage1_carve(p, nullptr, 0, nullptr, true);
}

extern "C" int vb_viss_halfsym(const vb_sky* sky, const vb_baselines* bl, const vb_stage1_opts* o, void* workspace,
                               size_t ws_bytes, double* V_half, unsigned long long* term_counters, void* stream) {
  Stage1Plan p{};
  VB_TRY(stage1_plan(sky, bl, o, &p));
  if (p.n_half == 0) return VB_OK;
  if (!V_half) return fail(VB_ERR_INVALID, "vb_viss_halfsym: V_half is NULL");
  if (!sky->B || !sky->l || !sky->m || !sky->n) return fail(VB_ERR_INVALID, "vb_viss_halfsym: sky arrays missing");
  if (!bl->u || !bl->v || !bl->w) return fail(VB_ERR_INVALID, "vb_viss_halfsym: u/v/w missing");
  if (p.blockage && (!bl->x1 || !bl->y1 || !bl->z1 || !bl->invn1 || !bl->x2 || !bl->y2 || !bl->z2 || !bl->invn2))
    return fail(VB_ERR_INVALID, "vb_viss_halfsym: endpoint arrays missing");
  Stage1Buffers b;
  size_t need = stage1_carve(p, nullptr, 0, nullptr, true);
  if (!workspace || ws_bytes < need)
    return fail(VB_ERR_NOMEM, "vb_viss_halfsym: workspace %zu bytes < %zu", ws_bytes, need);
  if (reinterpret_cast<uintptr_t>(workspace) % 256 != 0)
    return fail(VB_ERR_INVALID, "vb_viss_halfsym: workspace %p is not 256-byte aligned", workspace);
  stage1_carve(p, workspace, ws_bytes, &b, true);
  cudaStream_t s = as_stream(stream);
  VB_CUDA(cudaMemsetAsync(b.err, 0, sizeof(unsigned), s));
  return stage1_run(sky, bl, p, b, false, V_half, term_counters, s);
}

extern "C" int vb_phase_correct_expand(const double* V_half_raw, const float* w_full, int n_half, int nbl,
                                       int already_corrected, float* V_half_out, float* V_full_out, void* stream) {
  if (n_half < 0 || nbl <= 0 || n_half % nbl != 0)
    return fail(VB_ERR_INVALID, "vb_phase_correct_expand: n_half=%d nbl=%d", n_half, nbl);
  if (n_half == 0) return VB_OK;
  if (!V_half_raw || (!already_corrected && !w_full)) return fail(VB_ERR_INVALID, "vb_phase_correct_expand: null input");
  return phase_correct_expand_async(V_half_raw, w_full, n_half, nbl, already_corrected, V_half_out, V_full_out,
                                    as_stream(stream));
}

namespace vb {
__global__ void k_tile_classes(const S1Args a, int ntile, uint8_t* __restrict__ cls) {
  const bool raw = (a.phase_corrected == 0);
  const int64_t total = (int64_t)a.n_half * ntile;
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < total; q += (int64_t)gridDim.x * blockDim.x) {
    const int ih = (int)(q / ntile);
    const int t = (int)(q - (int64_t)ih * ntile);
    Baseline b;
    load_baseline(a, ih, raw, b);
    cls[q] = (uint8_t)tile_class_rt(a, b, t);
  }
}
}  // namespace vb

extern "C" int vb_stage1_tile_classes(const vb_sky* sky, const vb_baselines* bl, const vb_stage1_opts* o,
                                      void* workspace, size_t ws_bytes, uint8_t* cls, int* ntile_out, void* stream) {
  Stage1Plan p{};
  VB_TRY(stage1_plan(sky, bl, o, &p));
  if (ntile_out) *ntile_out = p.ntile_cull;
  if (p.n_half == 0) return VB_OK;
  if (!cls) return fail(VB_ERR_INVALID, "vb_stage1_tile_classes: cls is NULL");
  {
    // the classes are written by a kernel: refuse a host buffer up front
    cudaPointerAttributes at{};
    if (cudaPointerGetAttributes(&at, cls) != cudaSuccess ||
        (at.type != cudaMemoryTypeDevice && at.type != cudaMemoryTypeManaged)) {
      cudaGetLastError();
      return fail(VB_ERR_INVALID, "vb_stage1_tile_classes: cls %p is not device memory", (void*)cls);
    }
  }
  Stage1Buffers b;
  size_t need = stage1_carve(p, nullptr, 0, nullptr, true);
  if (!workspace || ws_bytes < need)
    return fail(VB_ERR_NOMEM, "vb_stage1_tile_classes: workspace %zu bytes < %zu", ws_bytes, need);
  if (reinterpret_cast<uintptr_t>(workspace) % 256 != 0)
    return fail(VB_ERR_INVALID, "vb_stage1_tile_classes: workspace %p is not 256-byte aligned", workspace);
  stage1_carve(p, workspace, ws_bytes, &b, true);
  cudaStream_t s = as_stream(stream);
  if (p.cull == VB_CULL_EXACT)
    VB_TRY(geom_exact_cones(p.cull_tile, sky->l, sky->m, sky->n, p.npix, b.cones, s));
  S1Args a{};
  a.npix = p.npix;
  a.cull = p.cull; a.cull_tile = p.cull_tile;
  a.tcx = sky->cx; a.tcy = sky->cy; a.tcz = sky->cz; a.tcosA = sky->cosA; a.tsinA = sky->sinA;
  a.cones = b.cones;
  a.u = bl->u; a.v = bl->v; a.w = bl->w;
  a.x1 = bl->x1; a.y1 = bl->y1; a.z1 = bl->z1; a.in1 = bl->invn1;
  a.x2 = bl->x2; a.y2 = bl->y2; a.z2 = bl->z2; a.in2 = bl->invn2;
  a.cp1 = bl->cosphi1; a.cp2 = bl->cosphi2; a.cosphi = bl->cosphi;
  a.n_half = p.n_half; a.nbl = p.nbl; a.blockage = p.blockage; a.phase_corrected = p.phase_corrected;
  a.mask_visible = p.mask_visible;
  int64_t total = (int64_t)p.n_half * p.ntile_cull;
  int g = (int)std::min<int64_t>(ceil_div(total, 256), (int64_t)sm_count() * 16);
  k_tile_classes<<<g, 256, 0, s>>>(a, p.ntile_cull, cls);
  VB_LAUNCH_CHECK();
  return VB_OK;
}

extern "C" int vb_stage1(const vb_sky* sky, const vb_baselines* bl, const vb_stage1_opts* o, void* workspace,
                         size_t ws_bytes, double* V_half, void* stream) {
  return vb_viss_halfsym(sky, bl, o, workspace, ws_bytes, V_half, nullptr, stream);
}
