// Vectorised CPU baseline of the upstream FP32 arithmetic -- test
// infrastructure only: the timed CPU leg of bench.py (cpu_baseline and the
// --impl reference arm).  Nothing in the product links or calls it, and no
// parity test uses it (the scalar restatement in vb_oracle.cpp is the one the
// golden fixtures pin).
//
// Per term it evaluates the same float expressions as the upstream kernels:
//   stage 1 (viss_recon_kernel.cuh:262-281): occlusion dots of both endpoints
//     against the horizon cosine, phase = -2 pi (u l + v m + w n) in FP32,
//     B cos(phase), B sin(phase) summed in FP32;
//   stage 2 (viss_recon_kernel_mirror_tile_vissfast.cuh:1096-1110): the
//     representative's occlusion test, phase = 2 pi (ugu (l + fa n) +
//     vgu (m + fb n)), Re(V exp(i phase)) summed in FP32, W counted.
// Unlike the scalar restatement, the loops are branch-free and vectorised
// (#pragma omp simd, glibc's libmvec sinf/cosf under -ffast-math, one clone
// each for AVX-512, AVX2 and baseline x86-64), so a masked term costs as much
// as a visible one and the FP32 sums run in vector lanes.  It is the fastest
// plain restatement of the method on the host cores, not a checker.
#include <omp.h>

#include <cmath>
#include <cstdint>
#include <vector>

#include "vb_oracle.h"

namespace {

inline int half_to_full_simd(int ih, int nbl) {
  const int step = ih / nbl;
  return step * 2 * nbl + (ih - step * nbl);
}

// One half-baseline over all pixels.
__attribute__((target_clones("avx512f", "avx2", "default")))
void stage1_row(int64_t npix, const float* __restrict B, const float* __restrict l, const float* __restrict m,
                const float* __restrict n, float uu, float vv, float ww, float a1, float b1, float c1, float d1,
                float a2, float b2, float c2, float d2, float q1, float q2, float* re, float* im) {
  const float kf = -2.0f * 3.14159265358979323846f;
  float fR = 0.f, fI = 0.f;
#pragma omp simd reduction(+ : fR, fI)
  for (int64_t p = 0; p < npix; ++p) {
    const float lp = l[p], mp = m[p], np_ = n[p];
    const float o1 = (lp * a1 + mp * b1 + np_ * c1) * d1;
    const float o2 = (lp * a2 + mp * b2 + np_ * c2) * d2;
    const float wgt = (o1 < q1 || o2 < q2) ? 0.0f : B[p];
    const float ang = kf * (uu * lp + vv * mp + ww * np_);
    fR += wgt * cosf(ang);
    fI += wgt * sinf(ang);
  }
  *re = fR;
  *im = fI;
}

// Representative groups of one pixel: SoA over all groups of all segments.
struct Reps {
  std::vector<float> ugu, vgu, vx, vy, fa, fb, px, py, pz, pi, qx, qy, qz, qi, cp, cq;
  void push(float u, float v, float x, float y, float a, float b, const float* p1, const float* p2, float c1,
            float c2) {
    ugu.push_back(u); vgu.push_back(v); vx.push_back(x); vy.push_back(y); fa.push_back(a); fb.push_back(b);
    px.push_back(p1[0]); py.push_back(p1[1]); pz.push_back(p1[2]); pi.push_back(p1[3]);
    qx.push_back(p2[0]); qy.push_back(p2[1]); qz.push_back(p2[2]); qi.push_back(p2[3]);
    cp.push_back(c1); cq.push_back(c2);
  }
};

constexpr int kPixBlock = 256;

// A block of up to kPixBlock pixels against every group: SIMD lanes are
// pixels, each group's data is broadcast (the group arrays are streamed once
// per block, not once per pixel).
__attribute__((target_clones("avx512f", "avx2", "default")))
void stage2_block(int ng, const Reps& r, int np, const float* __restrict lb, const float* __restrict mb,
                  const float* __restrict nb, float* __restrict acc, int* __restrict wc) {
  const float two_pi = 6.2831853071795864769f;
  for (int j = 0; j < np; ++j) { acc[j] = 0.f; wc[j] = 0; }
  for (int q = 0; q < ng; ++q) {
    const float px = r.px[q], py = r.py[q], pz = r.pz[q], pi = r.pi[q];
    const float qx = r.qx[q], qy = r.qy[q], qz = r.qz[q], qi = r.qi[q];
    const float cp = r.cp[q], cq = r.cq[q], fa = r.fa[q], fb = r.fb[q];
    const float ugu = r.ugu[q], vgu = r.vgu[q], vx = r.vx[q], vy = r.vy[q];
#pragma omp simd
    for (int j = 0; j < np; ++j) {
      const float lp = lb[j], mp = mb[j], np_ = nb[j];
      const float o1 = (lp * px + mp * py + np_ * pz) * pi;
      const float o2 = (lp * qx + mp * qy + np_ * qz) * qi;
      const bool vis = (o1 >= cp) && (o2 >= cq);
      const float l2 = lp + fa * np_, m2 = mp + fb * np_;
      const float ph = two_pi * (ugu * l2 + vgu * m2);
      const float t = vx * cosf(ph) - vy * sinf(ph);
      acc[j] += vis ? t : 0.0f;
      wc[j] += vis ? 1 : 0;
    }
  }
}

}  // namespace

extern "C" {

void or_stage1_subset_simd(int64_t npix, const float* B, const float* l, const float* m, const float* n, int nbl,
                           const float* u, const float* v, const float* w, const float* x1, const float* y1,
                           const float* z1, const float* in1, const float* x2, const float* y2, const float* z2,
                           const float* in2, const float* cp1, const float* cp2, float cosphi, int nsub,
                           const int* ih_list, double* V) {
#pragma omp parallel for schedule(dynamic, 1)
  for (int k = 0; k < nsub; ++k) {
    const int i = half_to_full_simd(ih_list[k], nbl);
    float re = 0.f, im = 0.f;
    stage1_row(npix, B, l, m, n, u[i], v[i], w[i], x1[i], y1[i], z1[i], in1[i], x2[i], y2[i], z2[i], in2[i],
               cp1 ? cp1[i] : cosphi, cp2 ? cp2[i] : cosphi, &re, &im);
    V[2 * k] = re;
    V[2 * k + 1] = im;
  }
}

// Mirror half grid, occ_mode 2 (representative = sorted index s0 + (L >> 1)),
// over the sampled pixels `pix`; groups of every segment are built first (plane
// fit, keys, stable grouping: the exact restatements of vb_oracle.cpp).
// Returns the number of gridded groups; t_group_s (nullable) receives the time
// the grouping took (a once-per-day cost, whatever the number of pixels).
int or_stage2_subset_simd(int64_t npix, const float* l, const float* m, const float* n, int nbl, int nseg,
                          const int* seg_t0, const int* seg_tlen, const float* u, const float* v, const float* w,
                          const float* x1, const float* y1, const float* z1, const float* in1, const float* x2,
                          const float* y2, const float* z2, const float* in2, const float* cp1, const float* cp2,
                          float cosphi, const float* V_half, float bl_max, float lambda, int grid_res, int npx,
                          const int64_t* pix, double* Cout, uint32_t* Wout, double* t_group_s) {
  (void)npix;
  const double tg0 = omp_get_wtime();
  Reps reps;
  for (int s = 0; s < nseg; ++s) {
    const int i0 = 2 * nbl * seg_t0[s];
    const int segN = 2 * nbl * seg_tlen[s], segNh = nbl * seg_tlen[s];
    float fa, fb, du;
    double denom;
    int RES, half;
    or_fa_fb(u + i0, v + i0, w + i0, segN, &fa, &fb, &denom);
    or_grid_params(fa, fb, bl_max, lambda, grid_res, &RES, &half, &du);
    const float inv_du = 1.0f / du;
    std::vector<int> keys(segNh), order(segNh), uniq(segNh), offs(segNh + 1);
    or_keys(u + i0, v + i0, segNh, nbl, 1, inv_du, RES, half, 0, keys.data());
    const int nu = or_groups(keys.data(), segNh, order.data(), uniq.data(), offs.data());
    for (int q = 0; q < nu; ++q) {
      if (!uniq[q]) continue;
      const int L = offs[q + 1] - offs[q];
      const int j = order[offs[q] + (L >> 1)];
      const int gh = nbl * seg_t0[s] + j;
      const int f = half_to_full_simd(gh, nbl);
      const int tmp = uniq[q] - 1, U = tmp / RES, Vc = tmp - U * RES;
      const float p1[4] = {x1[f], y1[f], z1[f], in1[f]}, p2[4] = {x2[f], y2[f], z2[f], in2[f]};
      reps.push((float)(U - half) * du, (float)(Vc - half) * du, V_half[2 * gh], V_half[2 * gh + 1], fa, fb, p1,
                p2, cp1 ? cp1[f] : cosphi, cp2 ? cp2[f] : cosphi);
    }
  }
  const int ng = (int)reps.ugu.size();
  if (t_group_s) *t_group_s = omp_get_wtime() - tg0;
  const int nblk = (npx + kPixBlock - 1) / kPixBlock;
#pragma omp parallel for schedule(dynamic, 1)
  for (int b = 0; b < nblk; ++b) {
    float lb[kPixBlock], mb[kPixBlock], nb[kPixBlock], acc[kPixBlock];
    int wc[kPixBlock];
    const int k0 = b * kPixBlock, np = (npx - k0) < kPixBlock ? npx - k0 : kPixBlock;
    for (int j = 0; j < np; ++j) {
      const int64_t p = pix[k0 + j];
      lb[j] = l[p]; mb[j] = m[p]; nb[j] = n[p];
    }
    stage2_block(ng, reps, np, lb, mb, nb, acc, wc);
    for (int j = 0; j < np; ++j) {
      Cout[k0 + j] = wc[j] > 0 ? (double)acc[j] / wc[j] : 0.0;
      if (Wout) Wout[k0 + j] = (uint32_t)wc[j];
    }
  }
  return ng;
}

}  // extern "C"
