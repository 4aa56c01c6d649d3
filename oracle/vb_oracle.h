/*
 * vb_oracle.h -- CPU restatement of the upstream two-stage direct-sum path
 * (viss_optimize_ws), used ONLY as test infrastructure: the checker of the
 * CUDA library in tests/, the smoke check, and the timed CPU baseline of
 * bench.py.  Nothing in the product links or calls it.
 *
 * Two arithmetic flavours of the direct sums:
 *   FP64  : phase with exact (n-1), sin/cos and sums in double -- the oracle
 *           against which every precision mode of the library is measured;
 *   REF32 : the upstream float arithmetic (FP32 phase, sincosf, FP32
 *           accumulators) -- the CPU stand-in for the upstream kernels.
 * Discrete steps (occlusion masks, plane fit, keys, groups, representatives)
 * are exact restatements and must agree bit for bit with the device.
 * All arrays are host memory.  Each function names the upstream file:line it
 * follows.
 */
#ifndef VB_ORACLE_H
#define VB_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

int or_num_threads(void);
void or_set_threads(int n);

/* HEALPix NEST pixel -> (face, ix, iy) by bit de-interleave and the ring
 * numbers (jr, nr, kshift, jp) of viss_recon_kernel.cuh:40-96 (exact ints). */
void or_nest_ints(int nside, int64_t first, int64_t count, int* face, int* ix, int* iy, int* jr, int* nr,
                  int* kshift, int* jp);
/* Same pixels in FP64: z = cos(theta) and phi, then (l, m, n) of the upstream
 * latitude / negated-longitude convention (viss_recon_kernel.cuh:98-111). */
void or_nest_lmn_f64(int nside, int64_t first, int64_t count, double* l, double* m, double* n);

/* Upstream per-pixel test (l x + m y + n z) * invn >= cosphi in FP32 with the
 * device's FMA contraction; variant 0: fma(n,z, fma(l,x, m*y)),
 * variant 1: fma(n,z, fma(m,y, l*x)).  mask[e*npix + p]. */
void or_occlusion_mask(int64_t npix, const float* l, const float* m, const float* n, int nend, const float* x,
                       const float* y, const float* z, const float* invn, const float* cpe, float cosphi,
                       int variant, uint8_t* mask);

/* Stage 1 (viss_recon_kernel.cuh:200-287; tile-cone semantics
 * viss_recon_kernel_mirror_tile_vissfast.cuh:506-558).  V[2*ih + {0,1}].
 * tile_cls (nullable): n_half x ntile classes (0 hidden, 1 visible = no
 * mask, 2 mixed = mask) with tiles of tile_pix pixels; NULL = mask every
 * pixel.  precision: 1 FP64, 0 REF32.  phase_corrected: 1 uses w*n (the
 * upstream V after phase correction), 0 uses w*(n-1). */
void or_stage1(int64_t npix, const float* B, const float* l, const float* m, const float* n, int n_full, int nbl,
               const float* u, const float* v, const float* w, const float* x1, const float* y1, const float* z1,
               const float* in1, const float* x2, const float* y2, const float* z2, const float* in2,
               const float* cp1, const float* cp2, float cosphi, int blockage, int phase_corrected, int tile_pix,
               const uint8_t* tile_cls, int precision, int mask_variant, double* V);

/* Same, for a subset of half-baselines (timing samples): ih_list[k]. */
void or_stage1_subset(int64_t npix, const float* B, const float* l, const float* m, const float* n, int nbl,
                      const float* u, const float* v, const float* w, const float* x1, const float* y1,
                      const float* z1, const float* in1, const float* x2, const float* y2, const float* z2,
                      const float* in2, float cosphi, int precision, int nsub, const int* ih_list, double* V);

/* V *= exp(-2 pi i w) (skipped if already) and conjugate completion, FP64
 * (common.hpp:255-277). Vh: 2*n_half, Vf: 4*n_half (nullable). */
void or_phase_correct_expand(const double* V, const float* w_full, int n_half, int nbl, int already, double* Vh,
                             double* Vf);

/* Plane fit in long double, viss_recon_kernel.cuh:673-701. */
void or_fa_fb(const float* u, const float* v, const float* w, int n, float* fa, float* fb, double* denom);
/* RES/half/du, main_recon_online.cu:377-383 (grid_res > 0 forces RES). */
void or_grid_params(float fa, float fb, float bl_max, float lambda, int grid_res, int* RES, int* half, float* du);
/* uv-cell keys: mirror=0 full signed set, round half away (viss_recon_kernel.cuh:295-312);
 * mirror=1 positive half set, floor(x+0.5) (..._vissfast.cuh:730-749).
 * variant: 0 fused multiply-add form fma(u, inv_du, 0.5), 1 separate rounding. */
void or_keys(const float* u, const float* v, int n, int nbl, int mirror, float inv_du, int RES, int half,
             int variant, int* keys);
/* Stable grouping of keys (sort by key, index ascending within a key):
 * order[n], nuniq, uniq[nuniq], offsets[nuniq+1] (viss_recon_kernel.cuh:375-456). */
int or_groups(const int* keys, int n, int* order, int* uniq, int* offsets);

/* Stage 2 of one day, every segment (viss_recon_kernel.cuh:470-659,
 * ..._vissfast.cuh:1039-1286, main_recon_online.cu:370-512).
 * seg_t0/seg_tlen in steps; V_half float (phase corrected, 2 per half
 * baseline); sp_* (nullable outputs, nseg each) receive fa, fb, RES, du, nuniq.
 * Outputs C[npix] (double, normalised) and W[npix]. precision 1 FP64 / 0 REF32. */
void or_stage2(int64_t npix, const float* l, const float* m, const float* n, int nbl, int nseg, const int* seg_t0,
               const int* seg_tlen, const float* u, const float* v, const float* w, const float* x1,
               const float* y1, const float* z1, const float* in1, const float* x2, const float* y2,
               const float* z2, const float* in2, const float* cp1, const float* cp2, float cosphi,
               const float* V_half, int mirror, int blockage, int occ_mode, float bl_max, float lambda,
               int grid_res, int precision, int mask_variant, int key_variant, const float* fa_in,
               const float* fb_in, double* C, uint32_t* W, float* sp_fa, float* sp_fb, int* sp_RES, float* sp_du,
               int* sp_nuniq);

/* Stage 2 for a subset of pixels (timing samples): pixel indices pix[k]. */
void or_stage2_subset(int64_t npix, const float* l, const float* m, const float* n, int nbl, int nseg,
                      const int* seg_t0, const int* seg_tlen, const float* u, const float* v, const float* w,
                      const float* x1, const float* y1, const float* z1, const float* in1, const float* x2,
                      const float* y2, const float* z2, const float* in2, float cosphi, const float* V_half,
                      float bl_max, float lambda, int grid_res, int precision, int npx, const int64_t* pix,
                      double* Cout);

/* Upstream orbit plan (main_recon_online.cu:116-121) and observation window
 * starts (orbit_online.cuh:317-333). */
void or_reference_plan(float lambda_m, int* orbit_res, int* nrev, int* seg_len);
void or_window_starts(float lambda_m, int day, uint64_t seed, int* t1s);

/* Seeded synthetic sky (mt19937_64: 24-bit uniforms, then point-source
 * indices) and synthetic formation positions, for CPU-only inputs. */
void or_make_sky(int nside, uint64_t seed, int n_points, float amp, float* B);
void or_syn_baselines(int nsat, int T, double dt_s, double alt_min, double alt_max, double spread_km,
                      double R_km, uint64_t seed, int day, float lambda_m, float* u, float* v, float* w, float* x1,
                      float* y1, float* z1, float* x2, float* y2, float* z2, float* in1, float* in2);

/* Vectorised CPU baseline of the upstream FP32 arithmetic (vb_oracle_simd.cpp):
 * the timed CPU leg of bench.py only, not a checker.  Stage 1 over the listed
 * half-baselines (V: 2 doubles each); stage 2 (mirror, occ_mode 2) over the
 * listed pixels, returning the number of gridded groups (t_group_s: the
 * grouping's time). */
void or_stage1_subset_simd(int64_t npix, const float* B, const float* l, const float* m, const float* n, int nbl,
                           const float* u, const float* v, const float* w, const float* x1, const float* y1,
                           const float* z1, const float* in1, const float* x2, const float* y2, const float* z2,
                           const float* in2, const float* cp1, const float* cp2, float cosphi, int nsub,
                           const int* ih_list, double* V);
int or_stage2_subset_simd(int64_t npix, const float* l, const float* m, const float* n, int nbl, int nseg,
                          const int* seg_t0, const int* seg_tlen, const float* u, const float* v, const float* w,
                          const float* x1, const float* y1, const float* z1, const float* in1, const float* x2,
                          const float* y2, const float* z2, const float* in2, const float* cp1, const float* cp2,
                          float cosphi, const float* V_half, float bl_max, float lambda, int grid_res, int npx,
                          const int64_t* pix, double* Cout, uint32_t* Wout, double* t_group_s);

#ifdef __cplusplus
}
#endif
#endif
