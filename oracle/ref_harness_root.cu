// Test-only harness around the upstream root variant (viss_optimize_ws:
// common.hpp, orbit_online.cuh, viss_recon_kernel.cuh).  The upstream headers
// are compiled from the upstream tree where they lie (-I <upstream root>,
// nothing copied) with the upstream flags (-O3 --use_fast_math), and their
// kernels and host functions are exposed through extern "C" wrappers so the
// parity tests can run the upstream code itself on the same inputs.
// Built by `make -C oracle ref` into oracle/_ref/libref_root.so.
#include "common.hpp"
#include "orbit_online.cuh"
#include "viss_recon_kernel.cuh"

#define REF_API extern "C" __attribute__((visibility("default")))

static int sync_rc() {
  cudaError_t e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaGetLastError();
  return (int)e;
}

REF_API int ref_pix2lmn(int nside, unsigned base, int n, float* l, float* m, float* nn) {
  if (n <= 0) return 0;
  pix2lmn_nest_kernel<<<(n + 255) / 256, 256>>>(nside, base, n, l, m, nn);
  return sync_rc();
}

REF_API int ref_invnorm3(const float* x, const float* y, const float* z, float* invn, int n) {
  if (n <= 0) return 0;
  invnorm3_kernel<<<(n + 255) / 256, 256>>>(x, y, z, invn, n);
  return sync_rc();
}

// Online orbit: steps [t0, t0+tlen) of day `day`, host outputs (segN = 56*tlen each).
REF_API int ref_orbit(float lambda_m, int day, unsigned long long seed, int t0, int tlen, float* u, float* v,
                      float* w, float* x1, float* y1, float* z1, float* x2, float* y2, float* z2, int* plan3) {
  OrbitGenCtx gen;
  orbit_gen_init(gen, 0, lambda_m, day, tlen, (uint64_t)seed);
  if (plan3) { plan3[0] = gen.OrbitRes; plan3[1] = gen.ProcessionCount; plan3[2] = gen.segLen; }
  orbit_gen_make_segment(gen, t0, tlen, true);
  const size_t b = (size_t)tlen * SIGNED_BASELINES_PER_T * sizeof(float);
  memcpy(u, gen.h_u, b); memcpy(v, gen.h_v, b); memcpy(w, gen.h_w, b);
  memcpy(x1, gen.h_x1, b); memcpy(y1, gen.h_y1, b); memcpy(z1, gen.h_z1, b);
  memcpy(x2, gen.h_x2, b); memcpy(y2, gen.h_y2, b); memcpy(z2, gen.h_z2, b);
  orbit_gen_destroy(gen);
  return sync_rc();
}

REF_API int ref_validate_halfsym(const float* u, const float* v, const float* w, int N) {
  return validate_uvw_halfsym_layout_ptr(u, v, w, N) ? 1 : 0;
}

REF_API int ref_viss_halfsym(const float* B, const float* l, const float* m, const float* n, long long npix,
                             const float* u, const float* v, const float* w, const float* x1, const float* y1,
                             const float* z1, const float* in1, const float* x2, const float* y2, const float* z2,
                             const float* in2, int N_half, float cosphi, float* Vpart) {
  if (N_half <= 0) return 0;
  const int TILE = 256;
  viss_partial_all_halfsym<TILE, true><<<(N_half + 255) / 256, 256, TILE * 4 * sizeof(float)>>>(
      B, l, m, n, npix, u, v, w, x1, y1, z1, in1, x2, y2, z2, in2, N_half, cosphi, (float2*)Vpart);
  return sync_rc();
}

REF_API void ref_fa_fb(const float* u, const float* v, const float* w, int n, float* fa, float* fb, double* denom) {
  compute_fa_fb_host_matlab_no_intercept(u, v, w, n, *fa, *fb, *denom);
}

REF_API void ref_phase_correct_expand(const float* Vhalf_in, const float* w_full, int N_half, float* Vhalf_out,
                                      float* Vfull_out) {
  std::vector<float2> h(N_half);
  for (int i = 0; i < N_half; ++i) h[i] = make_float2(Vhalf_in[2 * i], Vhalf_in[2 * i + 1]);
  phase_correct_viss_halfsym_host(h.data(), w_full, N_half);
  std::vector<float2> f(2 * (size_t)N_half);
  expand_viss_halfsym_to_full(h, f);
  for (int i = 0; i < N_half; ++i) { Vhalf_out[2 * i] = h[i].x; Vhalf_out[2 * i + 1] = h[i].y; }
  for (int i = 0; i < 2 * N_half; ++i) { Vfull_out[2 * i] = f[i].x; Vfull_out[2 * i + 1] = f[i].y; }
}

REF_API int ref_locg_full(const float* u, const float* v, int* locg, int n, float inv_du, int RES, int half) {
  if (n <= 0) return 0;
  build_locg_kernel<<<(n + 255) / 256, 256>>>(u, v, locg, n, inv_du, RES, half);
  return sync_rc();
}

// Groups of a full signed segment (device u, v, V).  Host outputs sized n
// (keys_unique, offsets n+1, idx_sorted, viss_avg 2n floats).
REF_API int ref_groups_full(const float* d_u, const float* d_v, const float* d_viss, int n, float du, int RES,
                            int half, int blockage, int* nuniq, int* keys_unique, int* offsets, int* idx_sorted,
                            float* viss_avg) {
  GroupArtifactsHost g;
  build_groups_device0(0, 0, d_u, d_v, (const float2*)d_viss, n, du, RES, half, blockage, g);
  *nuniq = g.nuniq;
  for (int i = 0; i < g.nuniq; ++i) keys_unique[i] = g.keys_unique[i];
  if (blockage) {
    for (int i = 0; i <= g.nuniq; ++i) offsets[i] = g.offsets[i];
    for (int i = 0; i < n; ++i) idx_sorted[i] = g.idx_sorted[i];
  } else {
    for (int i = 0; i < g.nuniq; ++i) { viss_avg[2 * i] = g.viss_avg[i].x; viss_avg[2 * i + 1] = g.viss_avg[i].y; }
  }
  return sync_rc();
}

REF_API int ref_recon_blockage(long long npix, const float* l, const float* m, const float* n, const int* keys,
                               const int* offsets, const int* idx, const float* Viss, const float* x1,
                               const float* y1, const float* z1, const float* in1, const float* x2, const float* y2,
                               const float* z2, const float* in2, int nuniq, int RES, int half, float du, float fa,
                               float fb, float cosphi, int occ_mode, float* Cseg, unsigned* Wseg) {
  int grid = (int)((npix + 255) / 256);
  recon_seg_blockage<64><<<grid, 256>>>(npix, l, m, n, keys, offsets, idx, (const float2*)Viss, x1, y1, z1, in1,
                                        x2, y2, z2, in2, nuniq, RES, half, du, fa, fb, cosphi, occ_mode, Cseg, Wseg);
  return sync_rc();
}

REF_API int ref_recon_keys_avg(long long npix, const float* l, const float* m, const float* n, const int* keys,
                               const float* vavg, int nuniq, int RES, int half, float du, float fa, float fb,
                               float* Cseg) {
  int grid = (int)((npix + 255) / 256);
  recon_seg_keys_avg<256><<<grid, 256>>>(npix, l, m, n, keys, (const float2*)vavg, nuniq, RES, half, du, fa, fb,
                                         Cseg);
  return sync_rc();
}

REF_API int ref_add_normalize(float* C, const unsigned* W, long long n) {
  normalize_by_weight<<<(int)((n + 255) / 256), 256>>>(C, W, n);
  return sync_rc();
}

// Device memory helpers so harness users need no other CUDA binding.
REF_API void* ref_malloc(size_t bytes) {
  void* p = nullptr;
  if (cudaMalloc(&p, bytes ? bytes : 1) != cudaSuccess) return nullptr;
  cudaMemset(p, 0, bytes ? bytes : 1);
  return p;
}
REF_API int ref_free(void* p) { return (int)cudaFree(p); }
REF_API int ref_h2d(void* dst, const void* src, size_t bytes) {
  return (int)cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice);
}
REF_API int ref_d2h(void* dst, const void* src, size_t bytes) {
  return (int)cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost);
}
