// Geometry of the run: HEALPix NESTED direction cosines, tile cones,
// occlusion masks, endpoint norms, and the online orbit / baseline generator.
//
// Parity rule: every float expression that feeds a discrete decision or a
// defined input (l, m, n, uvw, endpoint positions, invn, tile cones) is
// written as the same expression as upstream and compiled with the upstream
// flags, so the values are bit-identical; integer steps (bit de-interleave,
// index maps) are free to differ and do.
#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include "vb_common.cuh"
#include "vb_geom.cuh"
#include "vb_internal.h"

namespace vb {

constexpr float kPiF = (float)3.14159265358979323846;

// HEALPix base-face tables (row index in units of nside, column offset),
// the standard constants of the NESTED scheme (Gorski et al. 2005).
__constant__ int c_face_row[12] = {2, 2, 2, 2, 3, 3, 3, 3, 4, 4, 4, 4};
__constant__ int c_face_col[12] = {1, 3, 5, 7, 0, 2, 4, 6, 1, 3, 5, 7};

// Morton decode: even bits of v packed into the low half.
__device__ __forceinline__ unsigned compact_even_bits(unsigned v) {
  v &= 0x55555555u;
  v = (v | (v >> 1)) & 0x33333333u;
  v = (v | (v >> 2)) & 0x0F0F0F0Fu;
  v = (v | (v >> 4)) & 0x00FF00FFu;
  v = (v | (v >> 8)) & 0x0000FFFFu;
  return v;
}

// NEST -> (l, m, n); float steps follow viss_recon_kernel.cuh:67-111.
__global__ void k_pix2lmn(int nside, unsigned base, int64_t count, float* __restrict__ l,
                          float* __restrict__ m, float* __restrict__ n) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += stride) {
    unsigned ipix = base + (unsigned)i;
    unsigned npface = (unsigned)nside * (unsigned)nside;
    unsigned face = ipix / npface;
    unsigned ipf = ipix - face * npface;
    int ix = (int)compact_even_bits(ipf);
    int iy = (int)compact_even_bits(ipf >> 1);

    int jrt = ix + iy;
    int jpt = ix - iy;
    int nl4 = 4 * nside;
    int jr = c_face_row[face] * nside - jrt - 1;

    float fact1 = 1.0f / (3.0f * (float)nside * (float)nside);
    float fact2 = 2.0f / (3.0f * (float)nside);

    int nr, kshift;
    float z;
    if (jr < nside) {
      nr = jr;
      z = 1.0f - (float)(nr * nr) * fact1;
      kshift = 0;
    } else if (jr <= 3 * nside) {
      nr = nside;
      z = (float)(2 * nside - jr) * fact2;
      kshift = (jr - nside) & 1;
    } else {
      nr = nl4 - jr;
      z = -1.0f + (float)(nr * nr) * fact1;
      kshift = 0;
    }
    z = fminf(1.0f, fmaxf(-1.0f, z));
    float theta = acosf(z);

    int jp = ((c_face_col[face] * nr) + jpt + 1 + kshift) >> 1;
    if (jp > nl4) jp -= nl4;
    if (jp < 1) jp += nl4;

    float phi = (0.5f * kPiF) * (((float)jp) - 0.5f * (float)(kshift + 1)) / (float)nr;
    if (phi < 0.0f) phi += 2.0f * kPiF;

    float th = kPiF * 0.5f - theta;
    if (phi > kPiF) phi -= 2.0f * kPiF;
    phi = -phi;

    float st, ct, sp, cp;
    __sincosf(th, &st, &ct);
    __sincosf(phi, &sp, &cp);
    l[i] = ct * cp;
    m[i] = ct * sp;
    n[i] = st;
  }
}

__global__ void k_nm1(const float* __restrict__ n, float* __restrict__ nm1, int64_t count) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += stride)
    nm1[i] = n[i] - 1.0f;
}

// Tile cone meta with the upstream reduction order (256 threads: strided
// per-thread sums, then a pairwise tree), ..._vissfast.cuh:33-80.
constexpr int kMetaThreads = 256;
__global__ void __launch_bounds__(kMetaThreads)
k_tile_cone_meta(int tile_pix, const float* __restrict__ l, const float* __restrict__ m,
                 const float* __restrict__ n, int64_t npix, float* __restrict__ cx,
                 float* __restrict__ cy, float* __restrict__ cz, float* __restrict__ cosA,
                 float* __restrict__ sinA, int ntile) {
  __shared__ float rx[kMetaThreads], ry[kMetaThreads], rz[kMetaThreads];
  __shared__ float s_c[3];
  const int t = threadIdx.x;
  for (int tile = blockIdx.x; tile < ntile; tile += gridDim.x) {
    int64_t p0 = (int64_t)tile * tile_pix;
    int64_t rem = npix - p0;
    int tileN = (int)(rem < tile_pix ? rem : tile_pix);
    float sx = 0.0f, sy = 0.0f, sz = 0.0f;
    for (int k = t; k < tileN; k += kMetaThreads) {
      sx += l[p0 + k];
      sy += m[p0 + k];
      sz += n[p0 + k];
    }
    rx[t] = sx; ry[t] = sy; rz[t] = sz;
    __syncthreads();
    for (int off = kMetaThreads >> 1; off > 0; off >>= 1) {
      if (t < off) {
        rx[t] += rx[t + off];
        ry[t] += ry[t + off];
        rz[t] += rz[t + off];
      }
      __syncthreads();
    }
    if (t == 0) {
      float inv = rsqrtf(rx[0] * rx[0] + ry[0] * ry[0] + rz[0] * rz[0]);
      s_c[0] = rx[0] * inv;
      s_c[1] = ry[0] * inv;
      s_c[2] = rz[0] * inv;
    }
    __syncthreads();
    const float ccx = s_c[0], ccy = s_c[1], ccz = s_c[2];
    float mind = 1.0f;
    for (int k = t; k < tileN; k += kMetaThreads) {
      float d = ccx * l[p0 + k] + ccy * m[p0 + k] + ccz * n[p0 + k];
      mind = fminf(mind, d);
    }
    rx[t] = mind;
    __syncthreads();
    for (int off = kMetaThreads >> 1; off > 0; off >>= 1) {
      if (t < off) rx[t] = fminf(rx[t], rx[t + off]);
      __syncthreads();
    }
    if (t == 0) {
      float cA = fminf(1.0f, fmaxf(-1.0f, rx[0]));
      cx[tile] = ccx;
      cy[tile] = ccy;
      cz[tile] = ccz;
      cosA[tile] = cA;
      sinA[tile] = sqrtf(fmaxf(0.0f, 1.0f - cA * cA));
    }
    __syncthreads();
  }
}

// Conservative cones for VB_CULL_EXACT (this library's own; FP64): centre
// = normalised sum of unit pixel vectors, cos/sin of the largest angle.
__global__ void __launch_bounds__(kMetaThreads)
k_exact_cone_meta(int tile_pix, const float* __restrict__ l, const float* __restrict__ m,
                  const float* __restrict__ n, int64_t npix, ExactCone* __restrict__ out,
                  int ntile) {
  __shared__ double rx[kMetaThreads], ry[kMetaThreads], rz[kMetaThreads];
  const int t = threadIdx.x;
  for (int tile = blockIdx.x; tile < ntile; tile += gridDim.x) {
    int64_t p0 = (int64_t)tile * tile_pix;
    int64_t rem = npix - p0;
    int tileN = (int)(rem < tile_pix ? rem : tile_pix);
    double sx = 0, sy = 0, sz = 0;
    for (int k = t; k < tileN; k += kMetaThreads) {
      double a = l[p0 + k], b = m[p0 + k], c = n[p0 + k];
      double inv = 1.0 / sqrt(a * a + b * b + c * c);
      sx += a * inv; sy += b * inv; sz += c * inv;
    }
    rx[t] = sx; ry[t] = sy; rz[t] = sz;
    __syncthreads();
    for (int off = kMetaThreads >> 1; off > 0; off >>= 1) {
      if (t < off) { rx[t] += rx[t + off]; ry[t] += ry[t + off]; rz[t] += rz[t + off]; }
      __syncthreads();
    }
    double nrm = sqrt(rx[0] * rx[0] + ry[0] * ry[0] + rz[0] * rz[0]);
    double ccx = rx[0] / nrm, ccy = ry[0] / nrm, ccz = rz[0] / nrm;
    __syncthreads();
    double mind = 1.0;
    for (int k = t; k < tileN; k += kMetaThreads) {
      double a = l[p0 + k], b = m[p0 + k], c = n[p0 + k];
      double inv = 1.0 / sqrt(a * a + b * b + c * c);
      mind = fmin(mind, (ccx * a + ccy * b + ccz * c) * inv);
    }
    rx[t] = mind;
    __syncthreads();
    for (int off = kMetaThreads >> 1; off > 0; off >>= 1) {
      if (t < off) rx[t] = fmin(rx[t], rx[t + off]);
      __syncthreads();
    }
    if (t == 0) {
      const double alpha = acos(fmax(-1.0, fmin(1.0, rx[0]))) + 1e-9;
      ExactCone e;
      e.cx = ccx; e.cy = ccy; e.cz = ccz;
      e.cos_a = cos(alpha);
      e.sin_a = sin(alpha);
      e.pad = 0.0;
      out[tile] = e;
    }
    __syncthreads();
  }
}

__global__ void k_classify(const float* __restrict__ dotc, const float* __restrict__ cosA,
                           const float* __restrict__ sinA, float cosphi, int count,
                           uint8_t* __restrict__ vis, uint8_t* __restrict__ hid) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    bool v, h;
    cone_classify(dotc[i], cosA[i], sinA[i], cosphi, v, h);
    vis[i] = v ? 1 : 0;
    hid[i] = h ? 1 : 0;
  }
}

__global__ void k_invnorm3(const float* __restrict__ x, const float* __restrict__ y,
                           const float* __restrict__ z, float* __restrict__ invn, int count) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    float a = x[i], b = y[i], c = z[i];
    invn[i] = rsqrtf(a * a + b * b + c * c);
  }
}

__global__ void k_mask(const float* __restrict__ l, const float* __restrict__ m,
                       const float* __restrict__ n, int64_t npix, const float* __restrict__ x,
                       const float* __restrict__ y, const float* __restrict__ z,
                       const float* __restrict__ invn, const float* __restrict__ cpe,
                       float cosphi, int nend, uint8_t* __restrict__ mask) {
  const int64_t total = npix * (int64_t)nend;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
    int e = (int)(i / npix);
    int64_t p = i - (int64_t)e * npix;
    float c = occ_dot(l[p], m[p], n[p], x[e], y[e], z[e], invn[e]);
    float cp = cpe ? cpe[e] : cosphi;
    mask[i] = (c >= cp) ? 1 : 0;
  }
}

// Stage-1 pixel records: (l, m) as FP64, (n as FP64 bits, B, nm1), (l, m, n, B).
__global__ void k_pack_pixels(const float* __restrict__ B, const float* __restrict__ l,
                              const float* __restrict__ m, const float* __restrict__ n,
                              int64_t npix, PixRec* __restrict__ px) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < npix; i += stride) {
    float lf = l[i], mf = m[i], nf = n[i], bf = B[i];
    PixRec r;
    r.lm = make_double2((double)lf, (double)mf);
    double nd = (double)nf;
    r.nb = make_float4(__int_as_float(__double2loint(nd)), __int_as_float(__double2hiint(nd)),
                       bf, nf - 1.0f);
    r.f4 = make_float4(lf, mf, nf, bf);
    px[i] = r;
  }
}

// ---------------------------------------------------------------------------
// online orbit generator
// ---------------------------------------------------------------------------
// Upstream formation constants (orbit_online.cuh:4-13, 250-251): satellite 1 on
// a circular lunar orbit, trailing satellites offset along -velocity by a
// distance that ramps between r2 and r1 (metres) over a 14-day triangle.
constexpr int kRefSat = 8;
constexpr float kAKm = 2038.14f;
constexpr float kIncl = 30.0f * (float)(3.14159265358979323846 / 180.0);
constexpr float kArgp = 0.0f;
constexpr float kOrbitHours = 2.3f;
constexpr float kRaanPerRev = 0.08f;
constexpr float kRaanPerK = 0.08f;
constexpr float kRaanDay = 0.8f;

__device__ __forceinline__ float mean_anomaly_k(int k0, int orbit_res) {
  const float start = 1.0f / (float)orbit_res;
  const float end = (float)(2.0 * 3.14159265358979323846 + 3.14159265358979323846 / 200.0);
  if (orbit_res <= 1) return start;
  const float t = (float)k0 / (float)(orbit_res - 1);
  return start + (end - start) * t;
}

// Satellite 1 position per (revolution g, step k); orbit_online.cuh:48-83.
__global__ void k_ref_sat1(float* x, float* y, float* z, int orbit_res, int nrev, int dayid) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= orbit_res * nrev) return;
  const int g = idx / orbit_res;
  const int k = idx - g * orbit_res;
  const float d2r = (float)(3.14159265358979323846 / 180.0);
  const float raan = (float)g * d2r * kRaanPerRev +
                     ((float)(k + 1) / (float)orbit_res) * d2r * kRaanPerK +
                     (float)(dayid - 1) * d2r * kRaanDay;
  const float M = mean_anomaly_k(k, orbit_res);
  const float theta = M;
  const float r = kAKm;
  const float ww = theta + kArgp;
  float sw, cw, sr, cr, si, ci;
  sincosf(ww, &sw, &cw);
  sincosf(raan, &sr, &cr);
  sincosf(kIncl, &si, &ci);
  const float X = r * (cw * cr - sw * ci * sr);
  const float Y = r * (cw * sr + sw * ci * cr);
  const float Z = r * (sw * si);
  x[idx * kRefSat] = X;
  y[idx * kRefSat] = Y;
  z[idx * kRefSat] = Z;
}

__device__ __forceinline__ float ramp_triangle(float r2, float r1, int p, int T) {
  if (T <= 1) return r2;
  if (p < T) {
    float t = (float)p / (float)(T - 1);
    return r2 + (r1 - r2) * t;
  }
  int q = p - T;
  float t = (float)q / (float)(T - 1);
  return r1 + (r2 - r1) * t;
}

// Trailing satellites from satellite 1's step vector; orbit_online.cuh:85-161.
__global__ void k_ref_others(float* x, float* y, float* z, const float* __restrict__ r1,
                             const float* __restrict__ r2, int nrows, int T, int day_offset) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nrows - 1) return;
  const int a0 = i * kRefSat, a1 = (i + 1) * kRefSat;
  const float vx = x[a1] - x[a0];
  const float vy = y[a1] - y[a0];
  const float vz = z[a1] - z[a0];
  const float nv = sqrtf(vx * vx + vy * vy + vz * vz);
  const int period = 2 * T;
  const int p = (period > 0) ? ((day_offset + i) % period) : 0;
  const float mv = nv + 1e-20f;
  const float xr = x[a1], yr = y[a1], zr = z[a1];
#pragma unroll
  for (int sat = 1; sat < kRefSat; ++sat) {
    const float rt = ramp_triangle(r2[sat], r1[sat], p, T);
    const float ddx = rt * vx / mv / 1000.0f;
    const float ddy = rt * vy / mv / 1000.0f;
    const float ddz = rt * vz / mv / 1000.0f;
    x[a1 + sat] = xr - ddx;
    y[a1 + sat] = yr - ddy;
    z[a1 + sat] = zr - ddz;
  }
}

// Synthetic model: nsat circular Keplerian orbits, positions in FP64, stored
// as float32 km.  Row t = time step t.
__global__ void k_syn_positions(const SynSat* __restrict__ sats, int nsat, int T, double dt_s,
                                float* x, float* y, float* z) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= nsat * T) return;
  const int t = idx / nsat, s = idx - t * nsat;
  const SynSat q = sats[s];
  const double th = q.u0 + q.nmot * (double)t * dt_s;
  double sth, cth, sO, cO, si, ci;
  sincos(th, &sth, &cth);
  sincos(q.raan, &sO, &cO);
  sincos(q.incl, &si, &ci);
  x[idx] = (float)(q.r * (cth * cO - sth * ci * sO));
  y[idx] = (float)(q.r * (cth * sO + sth * ci * cO));
  z[idx] = (float)(q.r * (sth * si));
}

// Signed baselines of steps [t0, t0+tlen): gathers each step's row of
// satellite positions and forms uvw and endpoints; orbit_online.cuh:163-231.
__global__ void k_make_baselines(const float* __restrict__ X, const float* __restrict__ Y,
                                 const float* __restrict__ Z, int nsat,
                                 const int* __restrict__ row_start, int seg_len, int t0,
                                 int tlen, const int2* __restrict__ pairs, int nbl,
                                 float lambda_m, float* __restrict__ u, float* __restrict__ v,
                                 float* __restrict__ w, float* __restrict__ x1,
                                 float* __restrict__ y1, float* __restrict__ z1,
                                 float* __restrict__ x2, float* __restrict__ y2,
                                 float* __restrict__ z2, float* __restrict__ cp1,
                                 float* __restrict__ cp2, double occ_R_km) {
  const int per_t = 2 * nbl;
  const int total = per_t * tlen;
  for (int o = blockIdx.x * blockDim.x + threadIdx.x; o < total; o += gridDim.x * blockDim.x) {
    const int tl = o / per_t;
    const int bi = o - tl * per_t;
    const int tg = t0 + tl;
    int row;
    if (row_start) {
      const int orb = tg / seg_len;
      const int loc = tg - orb * seg_len;
      row = row_start[orb] + loc;
    } else {
      row = tg;
    }
    const int k = bi % nbl;
    const int2 pr = pairs[k];
    const float sgn = (bi < nbl) ? -1.0f : +1.0f;
    const int base = row * nsat;
    const float xm = X[base + pr.x], ym = Y[base + pr.x], zm = Z[base + pr.x];
    const float xn = X[base + pr.y], yn = Y[base + pr.y], zn = Z[base + pr.y];
    u[o] = sgn * (xn - xm) * 1e3f / lambda_m;
    v[o] = sgn * (yn - ym) * 1e3f / lambda_m;
    w[o] = sgn * (zn - zm) * 1e3f / lambda_m;
    float ax, ay, az, bx, by, bz;
    if (bi < nbl) { ax = xn; ay = yn; az = zn; bx = xm; by = ym; bz = zm; }
    else          { ax = xm; ay = ym; az = zm; bx = xn; by = yn; bz = zn; }
    x1[o] = ax; y1[o] = ay; z1[o] = az;
    x2[o] = bx; y2[o] = by; z2[o] = bz;
    if (cp1) {
      double ra = sqrt((double)ax * ax + (double)ay * ay + (double)az * az);
      double rb = sqrt((double)bx * bx + (double)by * by + (double)bz * bz);
      double qa = occ_R_km / ra, qb = occ_R_km / rb;
      cp1[o] = (float)(-sqrt(fmax(0.0, 1.0 - qa * qa)));
      cp2[o] = (float)(-sqrt(fmax(0.0, 1.0 - qb * qb)));
    }
  }
}

// +/- layout check (common.hpp:228-232 arithmetic: atol + rtol*max(|a|,|b|)).
__device__ __forceinline__ bool neg_pair_ok(float a, float b) {
  float ref = fmaxf(fabsf(a), fabsf(b));
  float tol = __fadd_rn(1e-5f, __fmul_rn(1e-5f, ref));
  return fabsf(__fadd_rn(a, b)) <= tol;
}

__global__ void k_validate_halfsym(const float* __restrict__ u, const float* __restrict__ v,
                                   const float* __restrict__ w, int n_full, int nbl,
                                   int* __restrict__ bad) {
  const int n_half = n_full / 2;
  for (int ih = blockIdx.x * blockDim.x + threadIdx.x; ih < n_half;
       ih += gridDim.x * blockDim.x) {
    int i0 = half_to_full_pos(ih, nbl);
    int i1 = i0 + nbl;
    if (!neg_pair_ok(u[i0], u[i1]) || !neg_pair_ok(v[i0], v[i1]) || !neg_pair_ok(w[i0], w[i1]))
      atomicMin(bad, i0);
  }
}

static int launch_grid(int64_t n, int threads) {
  int64_t g = ceil_div(n, threads);
  int cap = sm_count() * 32;
  if (g > cap) g = cap;
  return g < 1 ? 1 : (int)g;
}

// --- internal entry points used by the pipeline -----------------------------
int geom_pack_pixels(const float* B, const float* l, const float* m, const float* n,
                     int64_t npix, PixRec* px, cudaStream_t s) {
  if (npix <= 0) return VB_OK;
  k_pack_pixels<<<launch_grid(npix, 256), 256, 0, s>>>(B, l, m, n, npix, px);
  VB_LAUNCH_CHECK();
  return VB_OK;
}

int geom_exact_cones(int tile_pix, const float* l, const float* m, const float* n, int64_t npix,
                     ExactCone* out, cudaStream_t s) {
  if (npix <= 0) return VB_OK;
  int ntile = (int)ceil_div(npix, tile_pix);
  int grid = ntile < 65535 * 4 ? ntile : 65535 * 4;
  k_exact_cone_meta<<<grid, kMetaThreads, 0, s>>>(tile_pix, l, m, n, npix, out, ntile);
  VB_LAUNCH_CHECK();
  return VB_OK;
}

}  // namespace vb

using namespace vb;

// ---------------------------------------------------------------------------
// C ABI: geometry
// ---------------------------------------------------------------------------
extern "C" int vb_pix2lmn_nest(int nside, uint32_t base_ipix, int64_t count, float* l, float* m,
                               float* n, void* stream) {
  if (nside <= 0 || (nside & (nside - 1)) != 0 || nside > 16384)
    return fail(VB_ERR_INVALID, "vb_pix2lmn_nest: nside=%d must be a power of two <= 16384", nside);
  const int64_t npix = 12LL * nside * nside;
  if (count < 0 || (int64_t)base_ipix + count > npix)
    return fail(VB_ERR_INVALID, "vb_pix2lmn_nest: range [%u, +%lld) outside npix=%lld", base_ipix,
                (long long)count, (long long)npix);
  if (count == 0) return VB_OK;
  if (!l || !m || !n) return fail(VB_ERR_INVALID, "vb_pix2lmn_nest: null output");
  k_pix2lmn<<<launch_grid(count, 256), 256, 0, as_stream(stream)>>>(nside, base_ipix, count, l, m, n);
  VB_LAUNCH_CHECK();
  return VB_OK;
}

extern "C" int vb_build_nm1(const float* n, float* nm1, int64_t count, void* stream) {
  if (count < 0 || (count > 0 && (!n || !nm1))) return fail(VB_ERR_INVALID, "vb_build_nm1: bad args");
  if (count == 0) return VB_OK;
  k_nm1<<<launch_grid(count, 256), 256, 0, as_stream(stream)>>>(n, nm1, count);
  VB_LAUNCH_CHECK();
  return VB_OK;
}

extern "C" int vb_tile_cone_meta(int tile_pix, const float* l, const float* m, const float* n,
                                 int64_t npix, float* cx, float* cy, float* cz, float* cosA,
                                 float* sinA, void* stream) {
  if (tile_pix <= 0 || npix < 0) return fail(VB_ERR_INVALID, "vb_tile_cone_meta: tile_pix=%d npix=%lld", tile_pix, (long long)npix);
  if (npix == 0) return VB_OK;
  if (!l || !m || !n || !cx || !cy || !cz || !cosA || !sinA)
    return fail(VB_ERR_INVALID, "vb_tile_cone_meta: null pointer");
  int64_t ntile = ceil_div(npix, tile_pix);
  if (ntile > INT32_MAX) return fail(VB_ERR_INVALID, "vb_tile_cone_meta: too many tiles");
  int grid = ntile < 65535 * 4 ? (int)ntile : 65535 * 4;
  k_tile_cone_meta<<<grid, kMetaThreads, 0, as_stream(stream)>>>(tile_pix, l, m, n, npix, cx, cy, cz,
                                                                 cosA, sinA, (int)ntile);
  VB_LAUNCH_CHECK();
  return VB_OK;
}

extern "C" int vb_classify_tile_cone(const float* dotc, const float* cosA, const float* sinA,
                                     float cosphi, int count, uint8_t* all_vis, uint8_t* all_hid,
                                     void* stream) {
  if (count < 0) return fail(VB_ERR_INVALID, "vb_classify_tile_cone: count < 0");
  if (count == 0) return VB_OK;
  k_classify<<<launch_grid(count, 256), 256, 0, as_stream(stream)>>>(dotc, cosA, sinA, cosphi, count,
                                                                     all_vis, all_hid);
  VB_LAUNCH_CHECK();
  return VB_OK;
}

extern "C" int vb_invnorm3(const float* x, const float* y, const float* z, float* invn, int count,
                           void* stream) {
  if (count < 0) return fail(VB_ERR_INVALID, "vb_invnorm3: count < 0");
  if (count == 0) return VB_OK;
  k_invnorm3<<<launch_grid(count, 256), 256, 0, as_stream(stream)>>>(x, y, z, invn, count);
  VB_LAUNCH_CHECK();
  return VB_OK;
}

extern "C" int vb_occlusion_mask(const float* l, const float* m, const float* n, int64_t npix,
                                 const float* x, const float* y, const float* z, const float* invn,
                                 const float* cosphi_per_end, float cosphi, int nend, uint8_t* mask,
                                 void* stream) {
  if (npix < 0 || nend < 0) return fail(VB_ERR_INVALID, "vb_occlusion_mask: negative size");
  if (npix == 0 || nend == 0) return VB_OK;
  k_mask<<<launch_grid(npix * nend, 256), 256, 0, as_stream(stream)>>>(l, m, n, npix, x, y, z, invn,
                                                                       cosphi_per_end, cosphi, nend, mask);
  VB_LAUNCH_CHECK();
  return VB_OK;
}

// ---------------------------------------------------------------------------
// C ABI: orbit generator
// ---------------------------------------------------------------------------
struct vb_orbit {
  vb_orbit_params p{};
  int nsat = 0, nbl = 0, T = 0;
  int orbit_res = 0, nrev = 0, seg_len = 0;
  int nrows = 0;
  float *X = nullptr, *Y = nullptr, *Z = nullptr;   // [nrows][nsat]
  int* row_start = nullptr;                          // reference: window start per revolution
  int2* pairs = nullptr;
  float *r1 = nullptr, *r2 = nullptr;
  SynSat* sats = nullptr;
};

namespace vb {
// Host float helpers with the upstream host arithmetic (orbit_online.cuh:18-24).
int round_half_away_host(float x) { return (x >= 0.0f) ? (int)floorf(x + 0.5f) : (int)ceilf(x - 0.5f); }
static int mod_pos(int a, int m) { int r = a % m; return r < 0 ? r + m : r; }

void reference_plan(float lambda_m, int* orbit_res, int* nrev, int* seg_len) {
  *orbit_res = (int)std::ceil((double)(2.0 * 3.14159265358979323846) * (double)(100e3 / (double)lambda_m));
  *nrev = round_half_away_host(24.0f / kOrbitHours);
  *seg_len = *orbit_res / 3;
}
}  // namespace vb

static void orbit_free(vb_orbit* o) {
  cudaFree(o->X); cudaFree(o->Y); cudaFree(o->Z);
  cudaFree(o->row_start); cudaFree(o->pairs);
  cudaFree(o->r1); cudaFree(o->r2); cudaFree(o->sats);
  delete o;
}

extern "C" int vb_orbit_create(const vb_orbit_params* p, vb_orbit** out) {
  if (!p || !out) return fail(VB_ERR_INVALID, "vb_orbit_create: null argument");
  *out = nullptr;
  if (!(p->lambda_m > 0.0f)) return fail(VB_ERR_INVALID, "vb_orbit_create: lambda_m must be > 0");
  vb_orbit* o = new vb_orbit();
  o->p = *p;
  int rc = VB_OK;
  std::vector<int2> pairs;
  auto bail = [&](int code) { orbit_free(o); return code; };

  if (p->model == VB_ORBIT_REFERENCE) {
    if (p->nsat != 0 && p->nsat != kRefSat) {
      rc = fail(VB_ERR_UNSUPPORTED, "reference orbit model has 8 satellites (nsat=%d)", p->nsat);
      return bail(rc);
    }
    o->nsat = kRefSat;
    reference_plan(p->lambda_m, &o->orbit_res, &o->nrev, &o->seg_len);
    o->T = o->nrev * o->seg_len;
    o->nrows = o->orbit_res * o->nrev;
    if (o->seg_len <= 0 || o->nrows < 2) return bail(fail(VB_ERR_INVALID, "reference orbit plan is empty"));
  } else if (p->model == VB_ORBIT_SYNTHETIC) {
    if (p->nsat < 2 || p->nsat > 64) return bail(fail(VB_ERR_INVALID, "synthetic orbit: nsat=%d not in [2,64]", p->nsat));
    if (p->tsteps <= 0) return bail(fail(VB_ERR_INVALID, "synthetic orbit: tsteps must be > 0"));
    o->nsat = p->nsat;
    o->T = p->tsteps;
    o->nrows = p->tsteps;
  } else {
    return bail(fail(VB_ERR_INVALID, "unknown orbit model %d", p->model));
  }
  o->nbl = o->nsat * (o->nsat - 1) / 2;
  for (int a = 0; a < o->nsat - 1; ++a)
    for (int b = a + 1; b < o->nsat; ++b) pairs.push_back(make_int2(a, b));

  size_t tab = (size_t)o->nrows * o->nsat * sizeof(float);
  auto chk = [&](cudaError_t e, const char* what) {
    if (e != cudaSuccess && rc == VB_OK) rc = cuda_fail(e, what, __FILE__, __LINE__);
    if (e != cudaSuccess) cudaGetLastError();   // reported once, here
  };
  chk(cudaMalloc(&o->X, tab), "cudaMalloc X");
  chk(cudaMalloc(&o->Y, tab), "cudaMalloc Y");
  chk(cudaMalloc(&o->Z, tab), "cudaMalloc Z");
  chk(cudaMalloc(&o->pairs, pairs.size() * sizeof(int2)), "cudaMalloc pairs");
  if (rc != VB_OK) return bail(rc);
  chk(cudaMemcpy(o->pairs, pairs.data(), pairs.size() * sizeof(int2), cudaMemcpyHostToDevice), "pairs H2D");
  chk(cudaMemset(o->X, 0, tab), "memset X");
  chk(cudaMemset(o->Y, 0, tab), "memset Y");
  chk(cudaMemset(o->Z, 0, tab), "memset Z");
  if (rc != VB_OK) return bail(rc);

  if (p->model == VB_ORBIT_REFERENCE) {
    // trailing distances (m), orbit_online.cuh:250-251
    const float s = 100e3f / 23.0f;
    float h_r1[kRefSat] = {0, s, 4 * s, 10 * s, 16 * s, 18 * s, 21 * s, 23 * s};
    float h_r2[kRefSat] = {0, 0.1e3f, 0.4f * s, 1 * s, 1.6f * s, 1.8f * s, 2.1f * s, 2.3f * s};
    chk(cudaMalloc(&o->r1, sizeof(h_r1)), "cudaMalloc r1");
    chk(cudaMalloc(&o->r2, sizeof(h_r2)), "cudaMalloc r2");
    chk(cudaMalloc(&o->row_start, o->nrev * sizeof(int)), "cudaMalloc row_start");
    if (rc != VB_OK) return bail(rc);
    chk(cudaMemcpy(o->r1, h_r1, sizeof(h_r1), cudaMemcpyHostToDevice), "r1 H2D");
    chk(cudaMemcpy(o->r2, h_r2, sizeof(h_r2), cudaMemcpyHostToDevice), "r2 H2D");

    const int day = p->day;
    k_ref_sat1<<<(int)ceil_div(o->nrows, 256), 256>>>(o->X, o->Y, o->Z, o->orbit_res, o->nrev, day);
    const int T2 = round_half_away_host((float)o->orbit_res * 7.0f * 24.0f / kOrbitHours);
    const int mod14 = mod_pos(day - 1, 14);
    const int day_offset = round_half_away_host((float)mod14 * (float)o->orbit_res * 24.0f / kOrbitHours);
    k_ref_others<<<(int)ceil_div(o->nrows - 1, 256), 256>>>(o->X, o->Y, o->Z, o->r1, o->r2, o->nrows, T2,
                                                             day_offset);
    chk(cudaGetLastError(), "orbit kernels");

    // observation window per revolution, orbit_online.cuh:317-333
    uint64_t day_seed = p->seed ^ (uint64_t)day * 0x9E3779B97F4A7C15ULL;
    std::mt19937_64 rng(day_seed);
    std::vector<int> t1s(o->nrev);
    for (int g = 0; g < o->nrev; ++g) {
      const int orbit_start = g * o->orbit_res;
      const int orbit_end = (g + 1) * o->orbit_res - 1;
      double u01 = (double)(rng() >> 11) * (1.0 / 9007199254740992.0);
      int t1 = orbit_start + round_half_away_host((float)(u01 * (double)o->orbit_res * (2.0 / 3.0)));
      int t2 = t1 + o->seg_len - 1;
      if (t2 > orbit_end) { t2 = orbit_end; t1 = t2 - o->seg_len + 1; }
      if (t1 < orbit_start) t1 = orbit_start;
      if (t1 + o->seg_len - 1 > orbit_end) t1 = orbit_end - o->seg_len + 1;
      t1s[g] = t1;
    }
    chk(cudaMemcpy(o->row_start, t1s.data(), o->nrev * sizeof(int), cudaMemcpyHostToDevice), "t1s H2D");
  } else {
    // Synthetic formation: shared plane (seeded inclination / RAAN), each
    // satellite with its own altitude ~U[alt_min, alt_max] and small
    // along/cross-track offsets scaled by spread_km.
    std::mt19937_64 rng(p->seed ^ (uint64_t)p->day * 0x9E3779B97F4A7C15ULL);
    auto U01 = [&]() { return (double)(rng() >> 11) * (1.0 / 9007199254740992.0); };
    const double R = (p->occ_R_m > 0 ? p->occ_R_m : 6371e3) / 1000.0;
    const double mu = 398600.4418;   // km^3/s^2
    const double pi = 3.14159265358979323846;
    const double incl0 = (20.0 + 60.0 * U01()) * pi / 180.0;
    const double raan0 = 2.0 * pi * U01();
    const double u00 = 2.0 * pi * U01();
    std::vector<SynSat> sats(o->nsat);
    for (int k = 0; k < o->nsat; ++k) {
      double h = p->alt_min_km + (p->alt_max_km - p->alt_min_km) * U01();
      double r = R + h;
      double ang = p->spread_km / r;
      SynSat q;
      q.r = r;
      q.nmot = std::sqrt(mu / (r * r * r));
      q.incl = incl0 + ang * (2.0 * U01() - 1.0) * 0.5;
      q.raan = raan0 + ang * (2.0 * U01() - 1.0) * 0.5;
      q.u0 = u00 + ang * (2.0 * U01() - 1.0);
      sats[k] = q;
    }
    chk(cudaMalloc(&o->sats, sats.size() * sizeof(SynSat)), "cudaMalloc sats");
    if (rc != VB_OK) return bail(rc);
    chk(cudaMemcpy(o->sats, sats.data(), sats.size() * sizeof(SynSat), cudaMemcpyHostToDevice), "sats H2D");
    k_syn_positions<<<(int)ceil_div((int64_t)o->nsat * o->T, 256), 256>>>(o->sats, o->nsat, o->T, p->dt_s,
                                                                           o->X, o->Y, o->Z);
    chk(cudaGetLastError(), "synthetic orbit kernel");
  }
  chk(cudaDeviceSynchronize(), "orbit set-up");
  if (rc != VB_OK) return bail(rc);
  *out = o;
  return VB_OK;
}

extern "C" int vb_orbit_info(const vb_orbit* o, int* T, int* nbl, int* orbit_res, int* procession_count,
                             int* seg_len) {
  if (!o) return fail(VB_ERR_INVALID, "vb_orbit_info: null orbit");
  if (T) *T = o->T;
  if (nbl) *nbl = o->nbl;
  if (orbit_res) *orbit_res = o->orbit_res;
  if (procession_count) *procession_count = o->nrev;
  if (seg_len) *seg_len = o->seg_len;
  return VB_OK;
}

extern "C" int vb_orbit_make_segment(vb_orbit* o, int t0, int tlen, float* u, float* v, float* w,
                                     float* x1, float* y1, float* z1, float* x2, float* y2, float* z2,
                                     float* cosphi1, float* cosphi2, void* stream) {
  if (!o) return fail(VB_ERR_INVALID, "vb_orbit_make_segment: null orbit");
  if (t0 < 0 || tlen < 0 || t0 + tlen > o->T)
    return fail(VB_ERR_INVALID, "vb_orbit_make_segment: steps [%d,%d) outside [0,%d)", t0, t0 + tlen, o->T);
  if (tlen == 0) return VB_OK;
  if ((cosphi1 == nullptr) != (cosphi2 == nullptr))
    return fail(VB_ERR_INVALID, "vb_orbit_make_segment: cosphi1/cosphi2 must both be set or both NULL");
  if (cosphi1 && !(o->p.occ_R_m > 0))
    return fail(VB_ERR_INVALID, "vb_orbit_make_segment: per-endpoint cosphi needs occ_R_m > 0");
  int64_t total = (int64_t)2 * o->nbl * tlen;
  if (total > INT32_MAX) return fail(VB_ERR_UNSUPPORTED, "segment too large");
  k_make_baselines<<<launch_grid(total, 256), 256, 0, as_stream(stream)>>>(
      o->X, o->Y, o->Z, o->nsat, o->row_start, o->seg_len, t0, tlen, o->pairs, o->nbl, o->p.lambda_m,
      u, v, w, x1, y1, z1, x2, y2, z2, cosphi1, cosphi2, o->p.occ_R_m / 1000.0);
  VB_LAUNCH_CHECK();
  return VB_OK;
}

extern "C" int vb_orbit_destroy(vb_orbit* o) {
  if (o) orbit_free(o);
  return VB_OK;
}

extern "C" int vb_validate_uvw_halfsym(const float* u, const float* v, const float* w, int n_full, int nbl,
                                       int* bad_index, void* stream) {
  if (n_full < 0 || nbl <= 0 || n_full % (2 * nbl) != 0)
    return fail(VB_ERR_INVALID, "vb_validate_uvw_halfsym: n_full=%d not a multiple of 2*nbl=%d", n_full, 2 * nbl);
  if (bad_index) *bad_index = -1;
  if (n_full == 0) return VB_OK;
  cudaStream_t s = as_stream(stream);
  int* d_bad = nullptr;
  VB_CUDA(cudaMallocAsync(&d_bad, sizeof(int), s));
  const int big = INT32_MAX;
  VB_CUDA(cudaMemcpyAsync(d_bad, &big, sizeof(int), cudaMemcpyHostToDevice, s));
  k_validate_halfsym<<<launch_grid(n_full / 2, 256), 256, 0, s>>>(u, v, w, n_full, nbl, d_bad);
  int h = big;
  cudaError_t e = cudaMemcpyAsync(&h, d_bad, sizeof(int), cudaMemcpyDeviceToHost, s);
  cudaError_t e2 = cudaStreamSynchronize(s);
  cudaFreeAsync(d_bad, s);
  if (e != cudaSuccess) return cuda_fail(e, "validate D2H", __FILE__, __LINE__);
  if (e2 != cudaSuccess) return cuda_fail(e2, "validate sync", __FILE__, __LINE__);
  if (h != big) {
    if (bad_index) *bad_index = h;
    return fail(VB_ERR_HALFSYM, "uvw half-symmetry check failed at signed index %d (step %d, pair %d)", h,
                h / (2 * nbl), h % (2 * nbl));
  }
  return VB_OK;
}

// Launch helpers used by the pipeline's validation inside graphs.
namespace vb {
int geom_validate_async(const float* u, const float* v, const float* w, int n_full, int nbl, int* d_bad,
                        cudaStream_t s) {
  if (n_full <= 0) return VB_OK;
  k_validate_halfsym<<<launch_grid(n_full / 2, 256), 256, 0, s>>>(u, v, w, n_full, nbl, d_bad);
  VB_LAUNCH_CHECK();
  return VB_OK;
}
int geom_invnorm(const float* x, const float* y, const float* z, float* invn, int count, cudaStream_t s) {
  if (count <= 0) return VB_OK;
  k_invnorm3<<<launch_grid(count, 256), 256, 0, s>>>(x, y, z, invn, count);
  VB_LAUNCH_CHECK();
  return VB_OK;
}
}  // namespace vb
