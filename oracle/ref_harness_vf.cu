// Test-only harness around the upstream superset variant
// (viss_optimize_ws/mirror_tile_vissfast: tile-cone culling, nm1 fast path,
// mirrored half grid, occ_mode=2 representative groups).  Compiled from the
// upstream tree where it lies with the upstream flags; see
// ref_harness_root.cu.  Built into oracle/_ref/libref_vf.so.
#include "common_mirror_tile_vissfast.hpp"
#include "orbit_online_mirror_tile_vissfast.cuh"
#include "viss_recon_kernel_mirror_tile_vissfast.cuh"

#define REF_API extern "C" __attribute__((visibility("default")))

static int sync_rc() {
  cudaError_t e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaGetLastError();
  return (int)e;
}

REF_API int ref_vf_pix2lmn(int nside, unsigned base, int n, float* l, float* m, float* nn) {
  if (n <= 0) return 0;
  pix2lmn_nest_kernel<<<(n + 255) / 256, 256>>>(nside, base, n, l, m, nn);
  return sync_rc();
}

REF_API int ref_vf_nm1(const float* n, float* nm1, long long count) {
  build_nm1_kernel<<<(int)((count + 255) / 256), 256>>>(n, nm1, count);
  return sync_rc();
}

// Tile cone meta for TILE_PIX in {256, 512, 1024, 4096, 16384}.
REF_API int ref_vf_tile_meta(int tile_pix, const float* l, const float* m, const float* n, long long npix,
                             float* cx, float* cy, float* cz, float* cosA, float* sinA) {
  int ntile = (int)((npix + tile_pix - 1) / tile_pix);
  switch (tile_pix) {
    case 256: build_tile_cone_meta_kernel<256><<<ntile, 256>>>(l, m, n, npix, cx, cy, cz, cosA, sinA, ntile); break;
    case 512: build_tile_cone_meta_kernel<512><<<ntile, 256>>>(l, m, n, npix, cx, cy, cz, cosA, sinA, ntile); break;
    case 1024: build_tile_cone_meta_kernel<1024><<<ntile, 256>>>(l, m, n, npix, cx, cy, cz, cosA, sinA, ntile); break;
    case 4096: build_tile_cone_meta_kernel<4096><<<ntile, 256>>>(l, m, n, npix, cx, cy, cz, cosA, sinA, ntile); break;
    case 16384: build_tile_cone_meta_kernel<16384><<<ntile, 256>>>(l, m, n, npix, cx, cy, cz, cosA, sinA, ntile); break;
    default: return -1;
  }
  return sync_rc();
}

__global__ void k_ref_classify(const float* dotc, const float* cosA, const float* sinA, float cosphi, int count,
                               unsigned char* vis, unsigned char* hid) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  bool v = false, h = false;
  classify_tile_cone(dotc[i], cosA[i], sinA[i], cosphi, v, h);
  vis[i] = v ? 1 : 0;
  hid[i] = h ? 1 : 0;
}

REF_API int ref_vf_classify(const float* dotc, const float* cosA, const float* sinA, float cosphi, int count,
                            unsigned char* vis, unsigned char* hid) {
  if (count <= 0) return 0;
  k_ref_classify<<<(count + 255) / 256, 256>>>(dotc, cosA, sinA, cosphi, count, vis, hid);
  return sync_rc();
}

// Tile-cone stage 1 (TILE in {256, 512, 1024}).
REF_API int ref_vf_viss_tilecone(int tile_pix, const float* B, const float* l, const float* m, const float* n,
                                 const float* nm1, long long npix, const float* cx, const float* cy,
                                 const float* cz, const float* cosA, const float* sinA, int ntile, const float* u,
                                 const float* v, const float* w, const float* x1, const float* y1, const float* z1,
                                 const float* in1, const float* x2, const float* y2, const float* z2,
                                 const float* in2, int N_half, float cosphi, float* Vpart) {
  if (N_half <= 0) return 0;
  int grid = (N_half + 255) / 256;
  size_t shm = (size_t)tile_pix * 5 * sizeof(float);
#define LAUNCH(T)                                                                                              \
  viss_partial_all_halfsym_tilecone<T, true><<<grid, 256, shm>>>(B, l, m, n, nm1, npix, cx, cy, cz, cosA, sinA, \
                                                                  ntile, u, v, w, x1, y1, z1, in1, x2, y2, z2,  \
                                                                  in2, N_half, cosphi, (float2*)Vpart)
  switch (tile_pix) {
    case 256: LAUNCH(256); break;
    case 512: LAUNCH(512); break;
    case 1024: LAUNCH(1024); break;
    default: return -1;
  }
#undef LAUNCH
  return sync_rc();
}

REF_API int ref_vf_orbit(float lambda_m, int day, unsigned long long seed, int t0, int tlen, float* u, float* v,
                         float* w, float* x1, float* y1, float* z1, float* x2, float* y2, float* z2) {
  OrbitGenCtx gen;
  orbit_gen_init(gen, 0, lambda_m, day, tlen, (uint64_t)seed);
  orbit_gen_make_segment_async(gen, 0, t0, tlen, true);
  orbit_gen_wait_slot(gen, 0);
  OrbitSegSlot& s = gen.slots[0];
  const size_t b = (size_t)tlen * SIGNED_BASELINES_PER_T * sizeof(float);
  memcpy(u, s.h_u, b); memcpy(v, s.h_v, b); memcpy(w, s.h_w, b);
  memcpy(x1, s.h_x1, b); memcpy(y1, s.h_y1, b); memcpy(z1, s.h_z1, b);
  memcpy(x2, s.h_x2, b); memcpy(y2, s.h_y2, b); memcpy(z2, s.h_z2, b);
  orbit_gen_destroy(gen);
  return sync_rc();
}

REF_API int ref_vf_locg_half(const float* u, const float* v, int* locg, int n_half, float inv_du, int RES,
                             int half) {
  if (n_half <= 0) return 0;
  build_locg_half_kernel<<<(n_half + 255) / 256, 256>>>(u, v, locg, n_half, inv_du, RES, half);
  return sync_rc();
}

// Half-grid groups (device u, v full layout; V half). Host outputs sized n_half.
REF_API int ref_vf_groups_half(const float* d_u, const float* d_v, const float* d_vhalf, int n_half, float du,
                               int RES, int half, int blockage, int occ_mode, int* nuniq, int* keys_unique,
                               int* counts, int* offsets, int* idx_sorted, int* rep_half_idx, float* viss_avg) {
  GroupArtifactsHost g;
  build_groups_device0_half(0, 0, d_u, d_v, (const float2*)d_vhalf, n_half, du, RES, half, blockage, occ_mode, g);
  *nuniq = g.nuniq;
  for (int i = 0; i < g.nuniq; ++i) { keys_unique[i] = g.keys_unique[i]; counts[i] = g.counts[i]; }
  if (blockage == 0) {
    for (int i = 0; i < g.nuniq; ++i) { viss_avg[2 * i] = g.viss_avg[i].x; viss_avg[2 * i + 1] = g.viss_avg[i].y; }
  } else if (occ_mode == 2) {
    for (int i = 0; i < g.nuniq; ++i) rep_half_idx[i] = g.rep_half_idx[i];
  } else {
    for (int i = 0; i <= g.nuniq; ++i) offsets[i] = g.offsets[i];
    for (int i = 0; i < n_half; ++i) idx_sorted[i] = g.idx_sorted[i];
  }
  return sync_rc();
}

// occ_mode=2 representative recon of one segment: gathers the dense inputs
// with the upstream kernel, then runs recon_seg_blockage_half_rep<64>.
REF_API int ref_vf_recon_rep(long long npix, const float* l, const float* m, const float* n, const int* keys,
                             const float* ugu, const float* vgu, const int* rep_half_idx, int nuniq,
                             const float* Vhalf, const float* x1, const float* y1, const float* z1, const float* in1,
                             const float* x2, const float* y2, const float* z2, const float* in2, float fa, float fb,
                             float cosphi, float* Cseg, unsigned* Wseg) {
  float2* repV = nullptr;
  float4 *p1 = nullptr, *p2 = nullptr;
  cudaMalloc(&repV, (size_t)(nuniq > 0 ? nuniq : 1) * sizeof(float2));
  cudaMalloc(&p1, (size_t)(nuniq > 0 ? nuniq : 1) * sizeof(float4));
  cudaMalloc(&p2, (size_t)(nuniq > 0 ? nuniq : 1) * sizeof(float4));
  if (nuniq > 0)
    gather_rep_half_inputs<<<(nuniq + 255) / 256, 256>>>(rep_half_idx, nuniq, (const float2*)Vhalf, x1, y1, z1, in1,
                                                         x2, y2, z2, in2, repV, p1, p2);
  int grid = (int)((npix + 255) / 256);
  recon_seg_blockage_half_rep<64><<<grid, 256>>>(npix, l, m, n, keys, ugu, vgu, repV, p1, p2, nuniq, fa, fb, cosphi,
                                                 Cseg, Wseg);
  int rc = sync_rc();
  cudaFree(repV);
  cudaFree(p1);
  cudaFree(p2);
  return rc;
}

REF_API int ref_vf_recon_half(long long npix, const float* l, const float* m, const float* n, const int* keys,
                              const int* offsets, const int* idx, const float* Vhalf, const float* x1,
                              const float* y1, const float* z1, const float* in1, const float* x2, const float* y2,
                              const float* z2, const float* in2, int nuniq, int RES, int half, float du, float fa,
                              float fb, float cosphi, int occ_mode, float* Cseg, unsigned* Wseg) {
  int grid = (int)((npix + 255) / 256);
  recon_seg_blockage_half<64><<<grid, 256>>>(npix, l, m, n, keys, offsets, idx, (const float2*)Vhalf, x1, y1, z1,
                                             in1, x2, y2, z2, in2, nuniq, RES, half, du, fa, fb, cosphi, occ_mode,
                                             Cseg, Wseg);
  return sync_rc();
}

REF_API int ref_vf_recon_keys_avg_half(long long npix, const float* l, const float* m, const float* n,
                                       const int* keys, const float* vavg, int nuniq, int RES, int half, float du,
                                       float fa, float fb, float* Cseg) {
  int grid = (int)((npix + 255) / 256);
  recon_seg_keys_avg_half<256><<<grid, 256>>>(npix, l, m, n, keys, (const float2*)vavg, nuniq, RES, half, du, fa,
                                              fb, Cseg);
  return sync_rc();
}
