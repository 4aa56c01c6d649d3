// Declarations shared between the translation units of libvissb200.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

#include "vissb200.h"

namespace vb {

// Conservative pixel-tile cone (FP64): unit centre and the largest angle
// between the centre and any pixel of the tile.
struct ExactCone {          // unit axis and cos / sin of the half-angle
  double cx, cy, cz, cos_a, sin_a, pad;
};

// One satellite of the synthetic formation (circular orbit).
struct SynSat {
  double r;      // km
  double nmot;   // rad/s
  double incl;   // rad
  double raan;   // rad
  double u0;     // argument of latitude at t=0 (rad)
};

// Phase reduction parameters of the FP64-phase kernels: t + magic puts the
// turn fraction of t in the low word of the double with frac_bits bits.
struct PhaseMagic {
  double magic;      // 1.5 * 2^e
  double bias;       // half an output LSB (2^-24 turns)
  int shift;         // (52 - e) - 23: low-word shift of the top 23 fraction bits
};
PhaseMagic phase_magic_for(double max_abs_turns, bool* ok);

int round_half_away_host(float x);
void reference_plan(float lambda_m, int* orbit_res, int* nrev, int* seg_len);

// One stage-1 pixel record: FP64 (l, m), (n as two FP64 words, B, n - 1),
// FP32 (l, m, n, B); 48 bytes, one record per pixel, so that a stage of
// consecutive pixels is one contiguous range in global and in shared memory.
struct __align__(16) PixRec {
  double2 lm;
  float4 nb;
  float4 f4;
};
int geom_pack_pixels(const float* B, const float* l, const float* m, const float* n, int64_t npix,
                     PixRec* px, cudaStream_t s);
int geom_exact_cones(int tile_pix, const float* l, const float* m, const float* n, int64_t npix,
                     ExactCone* out, cudaStream_t s);
int geom_validate_async(const float* u, const float* v, const float* w, int n_full, int nbl, int* d_bad,
                        cudaStream_t s);
int geom_invnorm(const float* x, const float* y, const float* z, float* invn, int count, cudaStream_t s);

// ----- stage 1 ---------------------------------------------------------------
struct Stage1Plan {
  int precision, cull, phase_corrected, blockage;
  int bpt, minb, stage_pix, chunk_pix, cull_tile, refine_pix;
  int mask_visible;   // tile-cone: tiles proven visible still take the per-pixel test
  int64_t npix;
  int n_half, nbl;
  int nchunk, n_btile, n_items, grid;
  int ntile_cull;
  double max_turns;
};

struct Stage1Buffers {       // slices of a workspace
  PixRec* px = nullptr;      // [npix] stage-1 pixel records
  ExactCone* cones = nullptr;
  ExactCone* subcones = nullptr;   // tile-cone refinement sub-tiles
  double2* partial = nullptr;
  int* queue = nullptr;
  unsigned* err = nullptr;
};

int stage1_plan(const vb_sky* sky, const vb_baselines* bl, const vb_stage1_opts* o, Stage1Plan* p);
size_t stage1_carve(const Stage1Plan& p, void* ws, size_t cap, Stage1Buffers* b, bool pack_pixels);
// pixels_ready: lm/nb/f4 (and cones for VB_CULL_EXACT) already hold this sky.
// accumulate: V_half += this sky's sum (slabs of one sky) instead of V_half =.
int stage1_run(const vb_sky* sky, const vb_baselines* bl, const Stage1Plan& p, const Stage1Buffers& b,
               bool pixels_ready, double* V_half, unsigned long long* counters, cudaStream_t s,
               cudaEvent_t kbeg = nullptr, cudaEvent_t kend = nullptr, bool accumulate = false);
int stage1_prepare_pixels(const vb_sky* sky, const Stage1Plan& p, const Stage1Buffers& b, cudaStream_t s);
int phase_correct_expand_async(const double* Vraw, const float* w_full, int n_half, int nbl,
                               int already_corrected, float* Vh, float* Vf, cudaStream_t s);

// ----- stage 2 ---------------------------------------------------------------
struct Stage2Plan {
  int mirror, blockage, occ_mode, precision, cull, grid_res, ppt;
  float bl_max, lambda;
  int n_half_total, n_keyed_total, nseg;
  int64_t npix;
  int block_pix;        // pixels per CTA
  int nblocks;          // pixel blocks
  int nchunk_target;    // group chunks per pixel block (upper bound; sizes the partials)
  size_t cub_sort_bytes, cub_scan_bytes;
};
struct Stage2Pixels {       // per-pixel state the caller already prepared
  bool cones_ready = false;  // block cones already computed in this workspace
};
int stage2_plan(int n_half_total, int nseg, int64_t npix, const vb_stage2_opts* o, Stage2Plan* p);
// Exact cones of the stage-2 pixel blocks into the workspace (VB_CULL_EXACT);
// stage2_run then skips them when Stage2Pixels::cones_ready is set.
int stage2_prepare_cones(const vb_sky* sky, const Stage2Plan& p, void* ws, size_t cap, cudaStream_t st);
size_t stage2_workspace(const Stage2Plan& p, void* ws, size_t cap, void** slices);
// stage2_run in two parts: stage2_group (per-segment fit, keys, sort, group
// starts; reads only the baselines) and stage2_finish (group records, the
// reconstruction, finalisation).  The caller orders finish after group.
struct Stage2Groups {
  int sorted_keys_alt = 0;   // the sorted keys / indices sit in the second buffer of their pair
  int sorted_vals_alt = 0;
};
int stage2_group(const vb_baselines* bl, int nseg, const int* seg_t0, const int* seg_tlen, const Stage2Plan& p,
                 void* ws, size_t cap, cudaStream_t s, Stage2Groups* out);
int stage2_finish(const vb_sky* sky, const vb_baselines* bl, const float* V_half, int nseg, const Stage2Plan& p,
                  void* ws, size_t cap, const Stage2Groups& gr, float* C, uint32_t* W, vb_seg_params* seg_params,
                  unsigned long long* counters, double* w_scalar_total, cudaStream_t s, const Stage2Pixels* pre,
                  cudaEvent_t kbeg = nullptr, cudaEvent_t kend = nullptr);
int stage2_run(const vb_sky* sky, const vb_baselines* bl, const float* V_half, int nseg, const int* seg_t0,
               const int* seg_tlen, const Stage2Plan& p, void* ws, size_t cap, float* C, uint32_t* W,
               vb_seg_params* seg_params, unsigned long long* counters, double* w_scalar_total,
               cudaStream_t s, const Stage2Pixels* pre, cudaEvent_t kbeg = nullptr,
               cudaEvent_t kend = nullptr);

}  // namespace vb
