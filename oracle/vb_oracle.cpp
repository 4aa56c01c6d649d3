// CPU restatement of the upstream two-stage path; test infrastructure only
// (see vb_oracle.h).  Parity of this file is pinned by tests/golden/ fixtures
// produced by the upstream kernels themselves (tests/golden/make_golden.py).
#include "vb_oracle.h"

#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <random>
#include <vector>

namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr int kFaceRow[12] = {2, 2, 2, 2, 3, 3, 3, 3, 4, 4, 4, 4};
constexpr int kFaceCol[12] = {1, 3, 5, 7, 0, 2, 4, 6, 1, 3, 5, 7};

inline int half_to_full(int ih, int nbl) {
  int step = ih / nbl;
  return step * 2 * nbl + (ih - step * nbl);
}

// Exact occlusion dot in FP32 (device contraction, see or_occlusion_mask).
inline float occ_dot(float l, float m, float n, float x, float y, float z, float invn, int variant) {
  float d = variant == 0 ? std::fmaf(n, z, std::fmaf(l, x, m * y)) : std::fmaf(n, z, std::fmaf(m, y, l * x));
  return d * invn;
}

// Turn fraction of t and exp(-2 pi i t) in FP64.
inline void cis_turns(double t, double sign, double* c, double* s) {
  double fr = t - std::nearbyint(t);
  double a = sign * 2.0 * kPi * fr;
  *c = std::cos(a);
  *s = std::sin(a);
}

inline int round_half_away(float x) { return (x >= 0.0f) ? (int)std::floor(x + 0.5f) : (int)std::ceil(x - 0.5f); }

void ring_of(int nside, int64_t ipix, int& face, int& ix, int& iy, int& jr, int& nr, int& kshift, int& jp) {
  int64_t npface = (int64_t)nside * nside;
  face = (int)(ipix / npface);
  int64_t ipf = ipix - (int64_t)face * npface;
  ix = 0;
  iy = 0;
  for (int b = 0; b < 31; ++b) {
    ix |= (int)((ipf >> (2 * b)) & 1) << b;
    iy |= (int)((ipf >> (2 * b + 1)) & 1) << b;
  }
  int jrt = ix + iy, jpt = ix - iy, nl4 = 4 * nside;
  jr = kFaceRow[face] * nside - jrt - 1;
  if (jr < nside) { nr = jr; kshift = 0; }
  else if (jr <= 3 * nside) { nr = nside; kshift = (jr - nside) & 1; }
  else { nr = nl4 - jr; kshift = 0; }
  jp = (kFaceCol[face] * nr + jpt + 1 + kshift) >> 1;
  if (jp > nl4) jp -= nl4;
  if (jp < 1) jp += nl4;
}

}  // namespace

extern "C" {

int or_num_threads(void) { return omp_get_max_threads(); }
void or_set_threads(int n) {
  if (n > 0) omp_set_num_threads(n);
}

void or_nest_ints(int nside, int64_t first, int64_t count, int* face, int* ix, int* iy, int* jr, int* nr,
                  int* kshift, int* jp) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < count; ++i) {
    int f, x, y, r, q, k, p;
    ring_of(nside, first + i, f, x, y, r, q, k, p);
    face[i] = f; ix[i] = x; iy[i] = y; jr[i] = r; nr[i] = q; kshift[i] = k; jp[i] = p;
  }
}

void or_nest_lmn_f64(int nside, int64_t first, int64_t count, double* l, double* m, double* n) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < count; ++i) {
    int f, x, y, jr, nr, ks, jp;
    ring_of(nside, first + i, f, x, y, jr, nr, ks, jp);
    double z;
    if (jr < nside) z = 1.0 - (double)nr * nr / (3.0 * nside * nside);
    else if (jr <= 3 * nside) z = (2.0 * nside - jr) * 2.0 / (3.0 * nside);
    else z = -1.0 + (double)nr * nr / (3.0 * nside * nside);
    z = std::min(1.0, std::max(-1.0, z));
    double theta = std::acos(z);
    double phi = (0.5 * kPi) * ((double)jp - 0.5 * (ks + 1)) / (double)nr;
    if (phi < 0) phi += 2 * kPi;
    double th = 0.5 * kPi - theta;
    if (phi > kPi) phi -= 2 * kPi;
    phi = -phi;
    l[i] = std::cos(th) * std::cos(phi);
    m[i] = std::cos(th) * std::sin(phi);
    n[i] = std::sin(th);
  }
}

void or_occlusion_mask(int64_t npix, const float* l, const float* m, const float* n, int nend, const float* x,
                       const float* y, const float* z, const float* invn, const float* cpe, float cosphi,
                       int variant, uint8_t* mask) {
#pragma omp parallel for schedule(static)
  for (int e = 0; e < nend; ++e) {
    const float cp = cpe ? cpe[e] : cosphi;
    for (int64_t p = 0; p < npix; ++p)
      mask[(int64_t)e * npix + p] = occ_dot(l[p], m[p], n[p], x[e], y[e], z[e], invn[e], variant) >= cp ? 1 : 0;
  }
}

static void stage1_one(int64_t npix, const float* B, const float* l, const float* m, const float* n, int nbl,
                       const float* u, const float* v, const float* w, const float* x1, const float* y1,
                       const float* z1, const float* in1, const float* x2, const float* y2, const float* z2,
                       const float* in2, const float* cp1, const float* cp2, float cosphi, int blockage,
                       int phase_corrected, int tile_pix, const uint8_t* cls_row, int precision, int variant,
                       int ih, double* out2) {
  const int i = half_to_full(ih, nbl);
  const float uu = u[i], vv = v[i], ww = w[i];
  const float a1 = blockage ? x1[i] : 0, b1 = blockage ? y1[i] : 0, c1 = blockage ? z1[i] : 0;
  const float d1 = blockage ? in1[i] : 0;
  const float a2 = blockage ? x2[i] : 0, b2 = blockage ? y2[i] : 0, c2 = blockage ? z2[i] : 0;
  const float d2 = blockage ? in2[i] : 0;
  const float q1 = cp1 ? cp1[i] : cosphi, q2 = cp2 ? cp2[i] : cosphi;
  double accR = 0, accI = 0;
  float fR = 0.f, fI = 0.f;
  const float kf = -2.0f * (float)kPi;
  for (int64_t p = 0; p < npix; ++p) {
    if (blockage) {
      int cls = 2;
      if (cls_row) cls = cls_row[p / tile_pix];
      if (cls == 0) continue;
      if (cls == 2) {
        const float o1 = occ_dot(l[p], m[p], n[p], a1, b1, c1, d1, variant);
        const float o2 = occ_dot(l[p], m[p], n[p], a2, b2, c2, d2, variant);
        if (o1 < q1 || o2 < q2) continue;
      }
    }
    if (precision == 1) {
      const double nn = phase_corrected ? (double)n[p] : (double)n[p] - 1.0;
      const double t = (double)uu * l[p] + (double)vv * m[p] + (double)ww * nn;
      double c, s;
      cis_turns(t, -1.0, &c, &s);
      accR += (double)B[p] * c;
      accI += (double)B[p] * s;
    } else {
      const float nn = phase_corrected ? n[p] : n[p] - 1.0f;
      const float phase = uu * l[p] + vv * m[p] + ww * nn;
      const float ang = kf * phase;
      fR += B[p] * std::cos(ang);
      fI += B[p] * std::sin(ang);
    }
  }
  if (precision == 1) { out2[0] = accR; out2[1] = accI; }
  else { out2[0] = fR; out2[1] = fI; }
}

void or_stage1(int64_t npix, const float* B, const float* l, const float* m, const float* n, int n_full, int nbl,
               const float* u, const float* v, const float* w, const float* x1, const float* y1, const float* z1,
               const float* in1, const float* x2, const float* y2, const float* z2, const float* in2,
               const float* cp1, const float* cp2, float cosphi, int blockage, int phase_corrected, int tile_pix,
               const uint8_t* tile_cls, int precision, int mask_variant, double* V) {
  const int n_half = n_full / 2;
  const int64_t ntile = tile_pix > 0 ? (npix + tile_pix - 1) / tile_pix : 0;
#pragma omp parallel for schedule(dynamic, 4)
  for (int ih = 0; ih < n_half; ++ih)
    stage1_one(npix, B, l, m, n, nbl, u, v, w, x1, y1, z1, in1, x2, y2, z2, in2, cp1, cp2, cosphi, blockage,
               phase_corrected, tile_pix, tile_cls ? tile_cls + (int64_t)ih * ntile : nullptr, precision,
               mask_variant, ih, V + 2 * (int64_t)ih);
}

void or_stage1_subset(int64_t npix, const float* B, const float* l, const float* m, const float* n, int nbl,
                      const float* u, const float* v, const float* w, const float* x1, const float* y1,
                      const float* z1, const float* in1, const float* x2, const float* y2, const float* z2,
                      const float* in2, float cosphi, int precision, int nsub, const int* ih_list, double* V) {
#pragma omp parallel for schedule(dynamic, 1)
  for (int k = 0; k < nsub; ++k)
    stage1_one(npix, B, l, m, n, nbl, u, v, w, x1, y1, z1, in1, x2, y2, z2, in2, nullptr, nullptr, cosphi, 1, 1,
               0, nullptr, precision, 0, ih_list[k], V + 2 * (int64_t)k);
}

void or_phase_correct_expand(const double* V, const float* w_full, int n_half, int nbl, int already, double* Vh,
                             double* Vf) {
#pragma omp parallel for schedule(static)
  for (int ih = 0; ih < n_half; ++ih) {
    const int ip = half_to_full(ih, nbl);
    double re = V[2 * ih], im = V[2 * ih + 1];
    if (!already) {
      double c, s;
      cis_turns((double)w_full[ip], -1.0, &c, &s);
      double nr = re * c - im * s, ni = re * s + im * c;
      re = nr;
      im = ni;
    }
    if (Vh) { Vh[2 * ih] = re; Vh[2 * ih + 1] = im; }
    if (Vf) {
      Vf[2 * ip] = re; Vf[2 * ip + 1] = im;
      Vf[2 * (ip + nbl)] = re; Vf[2 * (ip + nbl) + 1] = -im;
    }
  }
}

void or_fa_fb(const float* u, const float* v, const float* w, int n, float* fa, float* fb, double* denom_out) {
  long double su2 = 0, sv2 = 0, suv = 0, suw = 0, svw = 0;
  for (int i = 0; i < n; i++) {
    long double uu = (long double)u[i], vv = (long double)v[i], ww = (long double)w[i];
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
  if (!std::isfinite((double)denom) || std::fabs(denom) < eps) denom = ((denom >= 0) ? 1.0L : -1.0L) * eps;
  long double a = (sv2 * suw - suv * svw) / denom;
  long double b = (su2 * svw - suv * suw) / denom;
  if (!std::isfinite((double)a) || !std::isfinite((double)b)) { a = 0; b = 0; }
  *fa = (float)a;
  *fb = (float)b;
}

void or_grid_params(float fa, float fb, float bl_max, float lambda, int grid_res, int* RES, int* half, float* du) {
  int r;
  if (grid_res > 0) {
    r = (grid_res % 2 == 0) ? grid_res + 1 : grid_res;
  } else {
    float lmax = std::sqrt(1.0f + fa * fa);
    float mmax = std::sqrt(1.0f + fb * fb);
    float lmmax = std::max(lmax, mmax);
    float temp_res = std::ceil(2.0f * bl_max / lambda * 2.0f * lmmax);
    r = (int)(temp_res + 2 + 1 - std::fmod(temp_res, 2.0f));
  }
  *RES = r;
  *half = (r - 1) / 2;
  *du = 2.0f * bl_max / lambda / (r - 1);
}

void or_keys(const float* u, const float* v, int n, int nbl, int mirror, float inv_du, int RES, int half,
             int variant, int* keys) {
  for (int i = 0; i < n; ++i) {
    int U, V;
    if (mirror) {
      const int f = half_to_full(i, nbl);
      if (variant == 0) {
        U = (int)std::floor(std::fmaf(u[f], inv_du, 0.5f)) + half;
        V = (int)std::floor(std::fmaf(v[f], inv_du, 0.5f)) + half;
      } else {
        U = (int)std::floor(u[f] * inv_du + 0.5f) + half;
        V = (int)std::floor(v[f] * inv_du + 0.5f) + half;
      }
      keys[i] = (U < 0 || U >= RES || V < 0 || V >= RES) ? 0 : U * RES + V + 1;
    } else {
      float xu = u[i] * inv_du, xv = v[i] * inv_du;
      int ui, vi;
      if (variant == 0) {
        ui = (xu >= 0.0f) ? (int)std::floor(std::fmaf(u[i], inv_du, 0.5f)) : (int)std::ceil(std::fmaf(u[i], inv_du, -0.5f));
        vi = (xv >= 0.0f) ? (int)std::floor(std::fmaf(v[i], inv_du, 0.5f)) : (int)std::ceil(std::fmaf(v[i], inv_du, -0.5f));
      } else {
        ui = round_half_away(xu);
        vi = round_half_away(xv);
      }
      U = ui + half;
      V = vi + half;
      keys[i] = ((unsigned)U >= (unsigned)RES || (unsigned)V >= (unsigned)RES) ? 0 : U * RES + V + 1;
    }
  }
}

int or_groups(const int* keys, int n, int* order, int* uniq, int* offsets) {
  std::iota(order, order + n, 0);
  std::stable_sort(order, order + n, [&](int a, int b) { return keys[a] < keys[b]; });
  int nu = 0;
  for (int i = 0; i < n; ++i) {
    if (i == 0 || keys[order[i]] != keys[order[i - 1]]) {
      uniq[nu] = keys[order[i]];
      offsets[nu] = i;
      ++nu;
    }
  }
  offsets[nu] = n;
  return nu;
}

void or_stage2(int64_t npix, const float* l, const float* m, const float* n, int nbl, int nseg, const int* seg_t0,
               const int* seg_tlen, const float* u, const float* v, const float* w, const float* x1,
               const float* y1, const float* z1, const float* in1, const float* x2, const float* y2,
               const float* z2, const float* in2, const float* cp1, const float* cp2, float cosphi,
               const float* V_half, int mirror, int blockage, int occ_mode, float bl_max, float lambda,
               int grid_res, int precision, int mask_variant, int key_variant, const float* fa_in,
               const float* fb_in, double* Cout, uint32_t* Wout, float* sp_fa, float* sp_fb, int* sp_RES,
               float* sp_du, int* sp_nuniq) {
  std::vector<double> Cacc(npix, 0.0);
  std::vector<uint32_t> Wacc(npix, 0);
  long long wscalar = 0;
  const int n_half_total = [&] { int s = 0; for (int k = 0; k < nseg; ++k) s += seg_tlen[k]; return s * nbl; }();
  // signed V (conjugate completion) for the full grid
  std::vector<float> Vfull;
  if (!mirror) {
    Vfull.assign((size_t)4 * n_half_total, 0.f);
    for (int ih = 0; ih < n_half_total; ++ih) {
      const int ip = half_to_full(ih, nbl);
      Vfull[2 * ip] = V_half[2 * ih]; Vfull[2 * ip + 1] = V_half[2 * ih + 1];
      Vfull[2 * (ip + nbl)] = V_half[2 * ih]; Vfull[2 * (ip + nbl) + 1] = -V_half[2 * ih + 1];
    }
  }
  for (int s = 0; s < nseg; ++s) {
    const int i0 = 2 * nbl * seg_t0[s];
    const int segN = 2 * nbl * seg_tlen[s];
    const int segNh = nbl * seg_tlen[s];
    float fa, fb;
    double denom;
    or_fa_fb(u + i0, v + i0, w + i0, segN, &fa, &fb, &denom);
    if (fa_in) { fa = fa_in[s]; fb = fb_in[s]; }
    int RES, half;
    float du;
    or_grid_params(fa, fb, bl_max, lambda, grid_res, &RES, &half, &du);
    const float inv_du = 1.0f / du;
    const int nk = mirror ? segNh : segN;
    std::vector<int> keys(nk), order(nk), uniq(nk), offs(nk + 1);
    // keyed arrays relative to the segment
    or_keys(u + i0, v + i0, nk, nbl, mirror, inv_du, RES, half, key_variant, keys.data());
    const int nu = or_groups(keys.data(), nk, order.data(), uniq.data(), offs.data());
    if (sp_fa) sp_fa[s] = fa;
    if (sp_fb) sp_fb[s] = fb;
    if (sp_RES) sp_RES[s] = RES;
    if (sp_du) sp_du[s] = du;
    if (sp_nuniq) sp_nuniq[s] = nu;
    if (nu <= 0) continue;
    if (!blockage) wscalar += nu;
    // global index of keyed element j (mirror: half index; full: signed index)
    auto gidx = [&](int j) { return mirror ? nbl * seg_t0[s] + j : i0 + j; };
    auto fullidx = [&](int j) { return mirror ? half_to_full(nbl * seg_t0[s] + j, nbl) : i0 + j; };
    const float* Vk = mirror ? V_half : Vfull.data();
    std::vector<float> ugu(nu), vgu(nu);
    for (int q = 0; q < nu; ++q) {
      int key = uniq[q];
      if (key == 0) { ugu[q] = vgu[q] = 0.f; continue; }
      int tmp = key - 1, U = tmp / RES, Vc = tmp - U * RES;
      ugu[q] = (float)(U - half) * du;
      vgu[q] = (float)(Vc - half) * du;
    }
    std::vector<float> avx(nu, 0.f), avy(nu, 0.f);
    if (!blockage) {
      for (int q = 0; q < nu; ++q) {
        double sx = 0, sy = 0;
        for (int k = offs[q]; k < offs[q + 1]; ++k) { sx += Vk[2 * gidx(order[k])]; sy += Vk[2 * gidx(order[k]) + 1]; }
        const int L = offs[q + 1] - offs[q];
        avx[q] = (float)(sx / L);
        avy[q] = (float)(sy / L);
      }
    }
#pragma omp parallel for schedule(static)
    for (int64_t p = 0; p < npix; ++p) {
      const float lp0 = l[p], mp0 = m[p], np0 = n[p];
      double acc = 0.0;
      float accf = 0.f;
      uint32_t wacc = 0;
      for (int q = 0; q < nu; ++q) {
        if (uniq[q] == 0) continue;
        const int s0 = offs[q], s1 = offs[q + 1], L = s1 - s0;
        float vx, vy;
        if (!blockage) {
          vx = avx[q]; vy = avy[q];
        } else {
          float sx = 0.f, sy = 0.f;
          int cnt = 0;
          bool rep_path = (occ_mode == 2);
          auto handle = [&](int pos) {
            const int j = order[pos];
            const int f = fullidx(j);
            const float o1 = occ_dot(lp0, mp0, np0, x1[f], y1[f], z1[f], in1[f], mask_variant);
            const float o2 = occ_dot(lp0, mp0, np0, x2[f], y2[f], z2[f], in2[f], mask_variant);
            const float c1 = cp1 ? cp1[f] : cosphi, c2 = cp2 ? cp2[f] : cosphi;
            if (o1 >= c1 && o2 >= c2) {
              const float ax = Vk[2 * gidx(j)], ay = Vk[2 * gidx(j) + 1];
              // the mirror representative kernel adds V unchecked
              // (..._vissfast.cuh:1103-1108); the member paths skip non-finite V
              if ((rep_path && mirror) || (std::isfinite(ax) && std::isfinite(ay))) { sx += ax; sy += ay; ++cnt; }
            }
          };
          if (occ_mode == 0) for (int pos = s0; pos < s1; ++pos) handle(pos);
          else if (occ_mode == 1) handle(s0);
          else if (occ_mode == 2) handle(s0 + (L >> 1));
          else { handle(s0); handle(s0 + L / 3); handle(s0 + 2 * L / 3); handle(s1 - 1); }
          if (cnt == 0) continue;
          const float invc = 1.0f / (float)cnt;
          vx = sx * invc; vy = sy * invc;
          ++wacc;
        }
        if (precision == 1) {
          const double lp = (double)lp0 + (double)fa * np0, mp = (double)mp0 + (double)fb * np0;
          const double t = (double)ugu[q] * lp + (double)vgu[q] * mp;
          double c, sn;
          cis_turns(t, 1.0, &c, &sn);
          acc += (double)vx * c - (double)vy * sn;
        } else {
          const float lp = lp0 + fa * np0, mp = mp0 + fb * np0;
          const float ph = 6.2831853071795864769f * (ugu[q] * lp + vgu[q] * mp);
          accf += vx * std::cos(ph) - vy * std::sin(ph);
        }
      }
      Cacc[p] += precision == 1 ? acc : (double)accf;
      Wacc[p] += wacc;
    }
  }
  for (int64_t p = 0; p < npix; ++p) {
    if (blockage) Cout[p] = Wacc[p] > 0 ? Cacc[p] / Wacc[p] : 0.0;
    else Cout[p] = wscalar > 0 ? Cacc[p] / (double)wscalar : 0.0;
    if (Wout) Wout[p] = Wacc[p];
  }
}

void or_stage2_subset(int64_t npix, const float* l, const float* m, const float* n, int nbl, int nseg,
                      const int* seg_t0, const int* seg_tlen, const float* u, const float* v, const float* w,
                      const float* x1, const float* y1, const float* z1, const float* in1, const float* x2,
                      const float* y2, const float* z2, const float* in2, float cosphi, const float* V_half,
                      float bl_max, float lambda, int grid_res, int precision, int npx, const int64_t* pix,
                      double* Cout) {
  (void)npix;
  std::vector<double> Cacc(npx, 0.0);
  std::vector<uint32_t> Wacc(npx, 0);
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
    struct Rep { float ugu, vgu, vx, vy, px, py, pz, pi, qx, qy, qz, qi; int key; };
    std::vector<Rep> reps(nu);
    for (int q = 0; q < nu; ++q) {
      Rep r{};
      r.key = uniq[q];
      const int L = offs[q + 1] - offs[q];
      const int j = order[offs[q] + (L >> 1)];
      const int gh = nbl * seg_t0[s] + j;
      const int f = half_to_full(gh, nbl);
      if (r.key) {
        int tmp = r.key - 1, U = tmp / RES, Vc = tmp - U * RES;
        r.ugu = (float)(U - half) * du;
        r.vgu = (float)(Vc - half) * du;
      }
      r.vx = V_half[2 * gh]; r.vy = V_half[2 * gh + 1];
      r.px = x1[f]; r.py = y1[f]; r.pz = z1[f]; r.pi = in1[f];
      r.qx = x2[f]; r.qy = y2[f]; r.qz = z2[f]; r.qi = in2[f];
      reps[q] = r;
    }
#pragma omp parallel for schedule(dynamic, 16)
    for (int k = 0; k < npx; ++k) {
      const int64_t p = pix[k];
      const float lp0 = l[p], mp0 = m[p], np0 = n[p];
      double acc = 0;
      float accf = 0;
      uint32_t wc = 0;
      for (int q = 0; q < nu; ++q) {
        const Rep& r = reps[q];
        if (!r.key) continue;
        const float o1 = occ_dot(lp0, mp0, np0, r.px, r.py, r.pz, r.pi, 0);
        const float o2 = occ_dot(lp0, mp0, np0, r.qx, r.qy, r.qz, r.qi, 0);
        if (!(o1 >= cosphi && o2 >= cosphi)) continue;
        if (precision == 1) {
          const double lp = (double)lp0 + (double)fa * np0, mp = (double)mp0 + (double)fb * np0;
          double c, sn;
          cis_turns((double)r.ugu * lp + (double)r.vgu * mp, 1.0, &c, &sn);
          acc += (double)r.vx * c - (double)r.vy * sn;
        } else {
          const float lp = lp0 + fa * np0, mp = mp0 + fb * np0;
          const float ph = 6.2831853071795864769f * (r.ugu * lp + r.vgu * mp);
          accf += r.vx * std::cos(ph) - r.vy * std::sin(ph);
        }
        ++wc;
      }
      Cacc[k] += precision == 1 ? acc : (double)accf;
      Wacc[k] += wc;
    }
  }
  for (int k = 0; k < npx; ++k) Cout[k] = Wacc[k] ? Cacc[k] / Wacc[k] : 0.0;
}

void or_reference_plan(float lambda_m, int* orbit_res, int* nrev, int* seg_len) {
  *orbit_res = (int)std::ceil((double)(2.0 * kPi) * (double)(100e3 / (double)lambda_m));
  float x = 24.0f / 2.3f;
  *nrev = (x >= 0.0f) ? (int)std::floor(x + 0.5f) : (int)std::ceil(x - 0.5f);
  *seg_len = *orbit_res / 3;
}

void or_window_starts(float lambda_m, int day, uint64_t seed, int* t1s) {
  int OR, PC, SL;
  or_reference_plan(lambda_m, &OR, &PC, &SL);
  std::mt19937_64 rng(seed ^ (uint64_t)day * 0x9E3779B97F4A7C15ULL);
  for (int g = 0; g < PC; ++g) {
    const int start = g * OR, end = (g + 1) * OR - 1;
    double u01 = (double)(rng() >> 11) * (1.0 / 9007199254740992.0);
    float x = (float)(u01 * (double)OR * (2.0 / 3.0));
    int t1 = start + ((x >= 0.0f) ? (int)std::floor(x + 0.5f) : (int)std::ceil(x - 0.5f));
    int t2 = t1 + SL - 1;
    if (t2 > end) { t2 = end; t1 = t2 - SL + 1; }
    if (t1 < start) t1 = start;
    if (t1 + SL - 1 > end) t1 = end - SL + 1;
    t1s[g] = t1;
  }
}

void or_make_sky(int nside, uint64_t seed, int n_points, float amp, float* B) {
  const int64_t npix = 12LL * nside * nside;
  std::mt19937_64 rng(seed);
  for (int64_t i = 0; i < npix; ++i) B[i] = (float)(rng() >> 40) * (1.0f / 16777216.0f);
  for (int k = 0; k < n_points; ++k) B[(int64_t)(rng() % (uint64_t)npix)] += amp;
}

void or_syn_baselines(int nsat, int T, double dt_s, double alt_min, double alt_max, double spread_km,
                      double R_km, uint64_t seed, int day, float lambda_m, float* u, float* v, float* w, float* x1,
                      float* y1, float* z1, float* x2, float* y2, float* z2, float* in1, float* in2) {
  std::mt19937_64 rng(seed ^ (uint64_t)day * 0x9E3779B97F4A7C15ULL);
  auto U01 = [&]() { return (double)(rng() >> 11) * (1.0 / 9007199254740992.0); };
  const double mu = 398600.4418;
  const double incl0 = (20.0 + 60.0 * U01()) * kPi / 180.0, raan0 = 2 * kPi * U01(), u00 = 2 * kPi * U01();
  struct S { double r, nm, inc, raan, u0; };
  std::vector<S> sats(nsat);
  for (int k = 0; k < nsat; ++k) {
    double h = alt_min + (alt_max - alt_min) * U01();
    double r = R_km + h, ang = spread_km / r;
    S q{r, std::sqrt(mu / (r * r * r)), 0, 0, 0};
    q.inc = incl0 + ang * (2 * U01() - 1) * 0.5;
    q.raan = raan0 + ang * (2 * U01() - 1) * 0.5;
    q.u0 = u00 + ang * (2 * U01() - 1);
    sats[k] = q;
  }
  const int nbl = nsat * (nsat - 1) / 2;
  std::vector<int> pa, pb;
  for (int a = 0; a < nsat - 1; ++a)
    for (int b = a + 1; b < nsat; ++b) { pa.push_back(a); pb.push_back(b); }
  std::vector<float> X(nsat), Y(nsat), Z(nsat);
  for (int t = 0; t < T; ++t) {
    for (int k = 0; k < nsat; ++k) {
      const S& q = sats[k];
      double th = q.u0 + q.nm * t * dt_s;
      X[k] = (float)(q.r * (std::cos(th) * std::cos(q.raan) - std::sin(th) * std::cos(q.inc) * std::sin(q.raan)));
      Y[k] = (float)(q.r * (std::cos(th) * std::sin(q.raan) + std::sin(th) * std::cos(q.inc) * std::cos(q.raan)));
      Z[k] = (float)(q.r * (std::sin(th) * std::sin(q.inc)));
    }
    for (int bi = 0; bi < 2 * nbl; ++bi) {
      const int o = t * 2 * nbl + bi, k = bi % nbl, ma = pa[k], nb = pb[k];
      const float sg = bi < nbl ? -1.0f : 1.0f;
      u[o] = sg * (X[nb] - X[ma]) * 1e3f / lambda_m;
      v[o] = sg * (Y[nb] - Y[ma]) * 1e3f / lambda_m;
      w[o] = sg * (Z[nb] - Z[ma]) * 1e3f / lambda_m;
      const int e1 = bi < nbl ? nb : ma, e2 = bi < nbl ? ma : nb;
      x1[o] = X[e1]; y1[o] = Y[e1]; z1[o] = Z[e1];
      x2[o] = X[e2]; y2[o] = Y[e2]; z2[o] = Z[e2];
      in1[o] = 1.0f / std::sqrt(X[e1] * X[e1] + Y[e1] * Y[e1] + Z[e1] * Z[e1]);
      in2[o] = 1.0f / std::sqrt(X[e2] * X[e2] + Y[e2] * Y[e2] + Z[e2] * Z[e2]);
    }
  }
}

}  // extern "C"
