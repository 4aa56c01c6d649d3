/*
 * vissb200.h -- C ABI of the B200 two-stage direct-sum pipeline
 * (stage 1: half-conjugate visibility sum over HEALPix NESTED pixels;
 *  stage 2: segmented short-time 2-D reconstruction).
 *
 * The upstream project (viss_optimize_ws) has no plugin or FFI layer: its
 * boundary is the main_recon_online executable (CLI, parameter script, output
 * files) plus header-only CUDA kernels with raw-pointer signatures that main()
 * calls directly.  Every entry point below replaces one of those internal
 * interfaces; the comment above each one names the upstream file:line.
 *
 * Conventions
 *  - Plain C types only.  Device buffers are raw device pointers; `stream` is a
 *    cudaStream_t passed as void* (NULL = legacy default stream).
 *  - The caller owns every buffer.  Kernel-level entry points never allocate;
 *    the ones that need scratch take a caller-provided workspace whose size a
 *    matching *_workspace_bytes() query returns, at a 256-byte aligned address
 *    (as cudaMalloc returns; VB_ERR_INVALID otherwise).  Only the pipeline and orbit
 *    objects (created once) allocate device memory, in their create calls.
 *  - Every call returns VB_OK (0) or a VB_ERR_* code and never exits the
 *    process; vb_last_error() gives a human-readable reason (thread-local).
 *  - All device work is enqueued on `stream`; kernel-level calls do not
 *    synchronise the host unless their comment says so.
 */
#ifndef VISSB200_H
#define VISSB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------ */
/* errors and library info                                                   */
/* ------------------------------------------------------------------------ */
#define VB_OK               0
#define VB_ERR_INVALID      1   /* bad argument / size / flag */
#define VB_ERR_CUDA         2   /* CUDA runtime error */
#define VB_ERR_TIMEOUT      3   /* a bounded device-side wait gave up */
#define VB_ERR_NOMEM        4   /* workspace too small or allocation failed */
#define VB_ERR_UNSUPPORTED  5   /* feature / size outside the supported range */
#define VB_ERR_HALFSYM      6   /* generated uvw violate the +/- pair layout */
#define VB_ERR_IO           7   /* file could not be read or written */

/* Bits of the device-side error word that the stage kernels set (atomicOr)
 * while they run.  A flag does not stop the kernels: flagged terms are still
 * summed (the access behind VB_DEVERR_BAD_INDEX excepted, which is skipped), so
 * a non-zero word means the outputs of that call are not to be trusted.  The
 * host reads the word after the stream has finished. */
#define VB_DEVERR_WAIT_TIMEOUT  1u  /* a bounded device-side wait gave up (stage 1: the bulk copy of
                                       a stage of pixel records into shared memory did not land) */
#define VB_DEVERR_BAD_INDEX     2u  /* an index check failed and the access was skipped */
#define VB_DEVERR_HALFSYM       4u  /* the +/- pair layout of the baselines is violated */
#define VB_DEVERR_PHASE_RANGE   8u  /* fp32_fp64phase: |u|+|v|+|w| of a term reached 2^28 turns, where
                                       the exact range reduction no longer holds (stage 1: checked as
                                       |u|, |v|, |w| >= 2^26 per baseline; stage 2: per group) */

/* The device error word of the last vb_viss_halfsym / vb_stage1 /
 * vb_recon_batched / vb_stage2 call that used this workspace (the word sits at
 * its start).  Copies it on `stream` and synchronises that stream. */
int vb_workspace_error_flags(const void* workspace, unsigned* flags, void* stream);

/* Numeric precision of the direct sums (stage 1 and stage 2). */
#define VB_PREC_REF32        0  /* FP32 phase, FP32 sincos, FP32 sums (upstream arithmetic) */
#define VB_PREC_FP64         1  /* plain FP64 direct sum: FP64 phase, FP64 sincos, FP64 sums */
#define VB_PREC_FP32_FP64PH  2  /* phase formed and range-reduced in FP64; FP32 sincos; FP32 tile sums + FP64 totals */
#define VB_PREC_FP32_DSPH    3  /* phase as an exact double-single FP32 product; FP32 sincos; Kahan sums */

/* Stage-1 culling semantics. */
#define VB_CULL_NONE         0  /* per-pixel occlusion mask on every term (upstream plain kernel) */
#define VB_CULL_TILECONE     1  /* upstream tile-cone semantics: hidden tiles skipped, all-visible tiles summed
                                   WITHOUT the per-pixel mask, mixed tiles masked per pixel */
#define VB_CULL_EXACT        2  /* same terms as VB_CULL_NONE; tiles proven all-visible / all-hidden with a
                                   margin skip the per-pixel test (an optimisation, bit-identical masks) */

int         vb_version(void);
const char* vb_error_string(int code);
const char* vb_last_error(void);
/* SM count and compute capability of the current device. */
int         vb_device_info(int* sm_count, int* cc_major, int* cc_minor);

/* ------------------------------------------------------------------------ */
/* geometry: HEALPix pixels, tile cones, endpoint norms                      */
/* ------------------------------------------------------------------------ */

/* NEST pixel index -> direction cosines (l, m, n), float32, bit-identical to
 * upstream.  Replaces pix2lmn_nest_kernel, viss_recon_kernel.cuh:29-112
 * (launched at main_recon_online.cu:182-185). */
int vb_pix2lmn_nest(int nside, uint32_t base_ipix, int64_t count,
                    float* l, float* m, float* n, void* stream);

/* nm1 = n - 1 rounded to float32 (the upstream fast-path input).
 * Replaces build_nm1_kernel, mirror_tile_vissfast/viss_recon_kernel_mirror_tile_vissfast.cuh:83-89. */
int vb_build_nm1(const float* n, float* nm1, int64_t count, void* stream);

/* Per tile of `tile_pix` consecutive NEST pixels: cone centre (cx,cy,cz),
 * cosA = min dot(centre, pixel), sinA.  Bit-identical to upstream for any
 * tile_pix (upstream supports 256/512).  Output arrays hold ceil(npix/tile_pix).
 * Replaces build_tile_cone_meta_kernel, viss_recon_kernel_mirror_tile_vissfast.cuh:21-81. */
int vb_tile_cone_meta(int tile_pix, const float* l, const float* m, const float* n,
                      int64_t npix, float* cx, float* cy, float* cz,
                      float* cosA, float* sinA, void* stream);

/* Three-way tile classification of `count` (dot, cosA, sinA) triples against
 * cosphi; writes 0/1 bytes.  Replaces the device function classify_tile_cone,
 * viss_recon_kernel_mirror_tile_vissfast.cuh:91-98 (exported for parity tests). */
int vb_classify_tile_cone(const float* dotc, const float* cosA, const float* sinA,
                          float cosphi, int count, uint8_t* all_vis,
                          uint8_t* all_hid, void* stream);

/* invn = rsqrtf(x^2+y^2+z^2) per endpoint, bit-identical to upstream.
 * Replaces invnorm3_kernel, orbit_online.cuh:443-449. */
int vb_invnorm3(const float* x, const float* y, const float* z, float* invn,
                int count, void* stream);

/* Occlusion mask of `npix` pixels against `nend` endpoints as one byte per
 * (endpoint, pixel), row-major [nend][npix]: 1 when
 * (l*x + m*y + n*z)*invn >= cosphi_e (the upstream per-pixel test,
 * viss_recon_kernel.cuh:271-273).  cosphi_e = cosphi_per_end[e] if that
 * pointer is non-NULL, else `cosphi`.  Exported for parity tests. */
int vb_occlusion_mask(const float* l, const float* m, const float* n, int64_t npix,
                      const float* x, const float* y, const float* z,
                      const float* invn, const float* cosphi_per_end, float cosphi,
                      int nend, uint8_t* mask, void* stream);

/* ------------------------------------------------------------------------ */
/* online orbit and baseline (uvw) generation                                */
/* ------------------------------------------------------------------------ */
#define VB_ORBIT_REFERENCE  0  /* upstream formation: lunar orbit A=2038.14 km, i=30 deg, trailing satellites */
#define VB_ORBIT_SYNTHETIC  1  /* seeded circular Keplerian orbits (Earth), altitude U[alt_min, alt_max] */

typedef struct vb_orbit vb_orbit;

typedef struct {
  int      model;          /* VB_ORBIT_* */
  float    lambda_m;       /* wavelength (m) */
  int      day;            /* day id (>=1); drives RAAN drift and the window RNG */
  uint64_t seed;           /* upstream --orbit_seed */
  int      nsat;           /* satellites (reference model: must be 8) */
  int      tsteps;         /* synthetic: time steps; reference: 0 = derived plan */
  double   dt_s;           /* synthetic: seconds per step */
  double   alt_min_km, alt_max_km;   /* synthetic altitude range */
  double   spread_km;      /* synthetic: formation spread (along/cross track, radial 1/3) */
  double   occ_R_m;        /* occluder radius; <=0 selects the upstream global cosphi */
} vb_orbit_params;

/* Allocates the per-day satellite position tables and runs the generator
 * set-up kernels (synchronises).  Replaces orbit_gen_init, orbit_online.cuh:233-336. */
int vb_orbit_create(const vb_orbit_params* p, vb_orbit** out);

/* Plan numbers of the generator: total steps T, pairs per step, and the
 * upstream plan terms (OrbitRes, ProcessionCount, segLen; 0 for synthetic).
 * Upstream computes them in main_recon_online.cu:116-121. */
int vb_orbit_info(const vb_orbit* o, int* T, int* nbl, int* orbit_res,
                  int* procession_count, int* seg_len);

/* Baselines of steps [t0, t0+tlen): 2*nbl signed baselines per step in the
 * upstream layout ([nbl "-" pairs][nbl "+" pairs], orbit_online.cuh:186-231):
 * u,v,w in wavelengths and endpoint positions (km).  cosphi1/cosphi2
 * (nullable) receive the per-endpoint horizon cosine.  Device pointers,
 * each of length 2*nbl*tlen.  Replaces orbit_gen_make_segment, orbit_online.cuh:338-366. */
int vb_orbit_make_segment(vb_orbit* o, int t0, int tlen,
                          float* u, float* v, float* w,
                          float* x1, float* y1, float* z1,
                          float* x2, float* y2, float* z2,
                          float* cosphi1, float* cosphi2, void* stream);

int vb_orbit_destroy(vb_orbit* o);

/* The +/- pair check of generated uvw (atol = rtol = 1e-5) on device data;
 * synchronises; *bad_index = first failing signed index or -1.  Returns
 * VB_ERR_HALFSYM on failure.  Replaces validate_uvw_halfsym_layout_ptr,
 * orbit_online.cuh:403-418 (host, per segment). */
int vb_validate_uvw_halfsym(const float* u, const float* v, const float* w,
                            int n_full, int nbl, int* bad_index, void* stream);

/* ------------------------------------------------------------------------ */
/* stage 1: half-conjugate visibility sum                                     */
/* ------------------------------------------------------------------------ */
typedef struct {
  int64_t      npix;
  const float *B, *l, *m, *n;        /* B already scaled by 4*pi/npix */
  int          tile_pix;             /* tile of the tile-cone meta (VB_CULL_TILECONE) */
  const float *cx, *cy, *cz, *cosA, *sinA;   /* tile-cone meta (VB_CULL_TILECONE only) */
} vb_sky;

typedef struct {
  int          n_full;               /* signed baselines, = 2*nbl*steps */
  int          nbl;                  /* unique pairs per step (28 for 8 satellites) */
  const float *u, *v, *w;
  const float *x1, *y1, *z1, *invn1, *x2, *y2, *z2, *invn2;
  const float *cosphi1, *cosphi2;    /* nullable: per-endpoint horizon cosine */
  float        cosphi;               /* used when cosphi1/cosphi2 are NULL */
} vb_baselines;

typedef struct {
  int precision;        /* VB_PREC_* */
  int cull;             /* VB_CULL_* */
  int phase_corrected;  /* 1: sum exp(-2pi i(ul+vm+wn)) (= upstream V after phase_correct);
                           0: sum exp(-2pi i(ul+vm+w(n-1))) as the upstream kernel */
  int blockage;         /* 1: apply occlusion (upstream DO_BLOCKAGE=true) */
  int bpt;              /* baselines per thread: 1, 2 or 4 (0 = auto) */
  int stage_pix;        /* pixels staged in shared memory per step (0 = auto) */
  int chunk_pix;        /* pixels per work item (0 = auto) */
  int exact_tile_pix;   /* tile of the VB_CULL_EXACT cones (0 = auto) */
  int ctas_per_sm;      /* resident CTAs per SM the kernel is built for: 2, or 3 with bpt <= 2 (0 = 2) */
  int items_per_cta;    /* work-queue items per resident CTA when chunk_pix = 0 (0 = auto) */
  int refine_pix;       /* tile-cone culling: inside mixed tiles, exact sub-tiles of this many
                           pixels skip or drop the per-pixel test where they can (0 = 256 on
                           cull tiles of 4096 pixels or more, else 128; < 0 = off); results are
                           identical either way */
  int mask_visible_tiles; /* tile-cone culling: 0 = tiles the cone test proves visible skip the
                           per-pixel test (upstream's all-visible nm1 fast path,
                           ..._vissfast.cuh:530-539); 1 = they take it like mixed tiles, so
                           only tiles proven hidden are culled */
} vb_stage1_opts;

size_t vb_stage1_workspace_bytes(const vb_sky* sky, const vb_baselines* bl,
                                 const vb_stage1_opts* o);

/* V_half[2*ih+{0,1}] = (re, im) for half-baseline ih, ih in [0, n_full/2),
 * with upstream index map ih -> (ih/nbl)*2*nbl + ih%nbl
 * (common.hpp:213-220).  term_counters (nullable, device, 4 x uint64) are
 * incremented by the terms evaluated as [visible-fast, masked, hidden-skipped, total].
 * Replaces viss_partial_all_halfsym<256,true> (viss_recon_kernel.cuh:200-287)
 * and viss_partial_all_halfsym_tilecone<TILE,true>
 * (viss_recon_kernel_mirror_tile_vissfast.cuh:437-561). */
int vb_viss_halfsym(const vb_sky* sky, const vb_baselines* bl,
                    const vb_stage1_opts* o, void* workspace, size_t ws_bytes,
                    double* V_half, unsigned long long* term_counters, void* stream);

/* Largest scratch of vb_viss_halfsym_noalloc, in bytes (64 MiB). */
#define VB_VISS_NOALLOC_MAX_BYTES (64u << 20)

/* vb_viss_halfsym for callers that cannot allocate device memory: hosts whose
 * device memory belongs to another allocator with a fixed budget, and
 * real-time loops that cannot afford the latency and implicit device
 * synchronisation of cudaMalloc / cudaFree.
 * The caller passes only inputs and outputs.  No counterpart in the upstream
 * project (upstream allocates everything in main()).
 * Scratch is one file-scope device array of VB_VISS_NOALLOC_MAX_BYTES that
 * every GPU which loads the library holds until the process exits.  Under
 * CUDA's default lazy module loading the array is reserved at the first call
 * on each device, and that call can fail with out-of-memory: hosts with their
 * own allocator should make the first call before that allocator takes its
 * budget (or run with CUDA_MODULE_LOADING=EAGER), and before any stream
 * capture.  Every call looks up the array's address in the current context.
 * A sky / baseline set that needs more scratch (about npix * 48 bytes +
 * partial sums, e.g. nside >= 512) returns VB_ERR_UNSUPPORTED.  With
 * o->chunk_pix = 0 the pixel chunks may be widened until the partial sums fit;
 * a chunk_pix the caller sets is kept, and a plan that does not fit with it
 * returns VB_ERR_UNSUPPORTED.  All calls share the one array and it keeps the
 * last call's contents: calls that overlap on the GPU (other streams or
 * threads) race.  error_flags (nullable, device, one uint32) receives this
 * call's VB_DEVERR_* bits on `stream`.  No cudaMalloc, cudaFree or allocating
 * library routine is called. */
int vb_viss_halfsym_noalloc(const vb_sky* sky, const vb_baselines* bl,
                            const vb_stage1_opts* o, double* V_half,
                            unsigned long long* term_counters,
                            unsigned* error_flags, void* stream);

/* Phase correction V *= exp(-2 pi i w) (skipped when already_corrected) in
 * FP64, then float32 outputs: V_half_out (2*n_half floats) and, if non-NULL,
 * the conjugate-completed signed layout V_full_out (4*n_half floats).
 * Replaces phase_correct_viss_halfsym_host and expand_viss_halfsym_to_full,
 * common.hpp:255-277. */
int vb_phase_correct_expand(const double* V_half_raw, const float* w_full,
                            int n_half, int nbl, int already_corrected,
                            float* V_half_out, float* V_full_out, void* stream);

/* ------------------------------------------------------------------------ */
/* stage 2: plane fit, uv grouping, reconstruction                           */
/* ------------------------------------------------------------------------ */

/* No-intercept least squares w ~ fa*u + fb*v in long double (host arrays).
 * Replaces compute_fa_fb_host_matlab_no_intercept, viss_recon_kernel.cuh:673-701. */
int vb_fa_fb_host(const float* u, const float* v, const float* w, int n,
                  float* fa, float* fb, double* denom);

/* RES (odd), half=(RES-1)/2, du from fa, fb, bl_max, lambda; grid_res > 0
 * forces RES = grid_res (+1 when even).  Replaces main_recon_online.cu:377-383. */
int vb_grid_params(float fa, float fb, float bl_max, float lambda, int grid_res,
                   int* RES, int* half, float* du);

/* uv-cell keys: key = U*RES + V + 1, 0 when off-grid.
 * mirror=0: full signed set, round half away from zero (viss_recon_kernel.cuh:295-312);
 * mirror=1: positive half set via the half->full map, floor(x+0.5)
 * (viss_recon_kernel_mirror_tile_vissfast.cuh:730-749).  n = number of keys written. */
int vb_build_keys(const float* u_full, const float* v_full, int n, int nbl,
                  int mirror, float inv_du, int RES, int half, int* keys, void* stream);

typedef struct {
  int mirror;           /* 1: mirrored half grid (positive half-baselines only) */
  int blockage;         /* 1: occlusion-aware groups; 0: group averages */
  int occ_mode;         /* 0 all members, 1 first, 2 median representative, else 4 samples */
  int precision;        /* VB_PREC_* */
  int cull;             /* 0: per-pixel masks; 2: proven all-visible/hidden pixel blocks skip the test */
  int grid_res;         /* > 0 forces RES */
  float bl_max;         /* metres */
  float lambda;         /* metres */
  int ppt;              /* pixels per thread of the occ_mode=2 / blockage=0 path: 1, 2 or 4
                           (0 = 4 for VB_PREC_FP32_FP64PH, 2 otherwise) */
  int items_per_cta;    /* work-queue items (pixel block x group chunk) per resident CTA (0 = auto) */
} vb_stage2_opts;

typedef struct {       /* per-segment plane-fit and grid numbers, device or host copy */
  float fa, fb, du, inv_du;
  int   RES, half, nuniq, group_start;
  double denom;
  int   n_keyed;        /* baselines grouped (segN or segN_half) */
  int   pad;
} vb_seg_params;

/* Workspace for vb_recon_batched with at most n_half_total half-baselines,
 * nseg segments and npix pixels. */
size_t vb_stage2_workspace_bytes(int n_half_total, int nseg, int64_t npix,
                                 const vb_stage2_opts* o);

/* All segments of a day in one batch, device-only (no host syncs, graph
 * capturable): per-segment fa/fb (double-double on device), RES/du, keys,
 * stable (key, index) sort, run-length groups, representatives
 * (idx_sorted[s0 + (L>>1)]), then one reconstruction launch over
 * (pixel block x group chunk) and the normalisation C = sum C / sum W.
 * seg_t0/seg_tlen: device int arrays (steps, relative to the baselines given);
 * V_half: phase-corrected float2 of every half-baseline (from
 * vb_phase_correct_expand).  Outputs C (npix float), W (npix uint32,
 * nullable), seg_params (device, nseg entries, nullable) and
 * term_counters (nullable, 4 x uint64 as in stage 1).
 * Replaces the per-segment loop main_recon_online.cu:370-512 /
 * main_recon_online_mirror_tile_vissfast.cu:427-604 with build_groups_device0
 * (viss_recon_kernel.cuh:349-467), build_groups_device0_half
 * (..._mirror_tile_vissfast.cuh:751-890), recon_seg_keys_avg / recon_seg_blockage
 * (viss_recon_kernel.cuh:470-639), recon_seg_blockage_half_rep /
 * recon_seg_keys_avg_half / recon_seg_blockage_half (..._vissfast.cuh:1039-1286)
 * and add_inplace / normalize_by_weight / scale_inplace (viss_recon_kernel.cuh:641-659). */
int vb_recon_batched(const vb_sky* sky, const vb_baselines* bl, const float* V_half,
                     int nseg, const int* seg_t0, const int* seg_tlen,
                     const vb_stage2_opts* o, void* workspace, size_t ws_bytes,
                     float* C, uint32_t* W, vb_seg_params* seg_params,
                     unsigned long long* term_counters, void* stream);

/* Short names for the two stage kernels: vb_stage1 is vb_viss_halfsym without
 * the term counters, vb_stage2 is vb_recon_batched without seg_params and the
 * term counters.  Same upstream kernels replaced as those two entries. */
int vb_stage1(const vb_sky* sky, const vb_baselines* bl, const vb_stage1_opts* o,
              void* workspace, size_t ws_bytes, double* V_half, void* stream);
int vb_stage2(const vb_sky* sky, const vb_baselines* bl, const float* V_half,
              int nseg, const int* seg_t0, const int* seg_tlen, const vb_stage2_opts* o,
              void* workspace, size_t ws_bytes, float* C, uint32_t* W, void* stream);

/* ------------------------------------------------------------------------ */
/* whole pipeline (the main_recon_online run)                                */
/* ------------------------------------------------------------------------ */
typedef struct vb_pipeline vb_pipeline;


typedef struct {
  /* upstream flags (main_recon_online.cu:6-27, ..._mirror_tile_vissfast.cu:7-31) */
  int      nside;          /* power of two <= 16384 (3.2e9 pixels: beyond one device, use slab_pix) */
  int      day;
  int      segs;
  int      blockage;
  int      occ_mode;
  uint64_t orbit_seed;
  float    lambda_m;       /* from --btag: 1M -> 300, 10M -> 30, 30M -> 10 */
  int      viss_tile_pix;  /* tile of the tile-cone culling */
  /* additive flags */
  int      mirror;         /* 1: mirrored half-grid recon */
  int      cull;           /* VB_CULL_* for stage 1 */
  int      precision;      /* VB_PREC_* */
  int      orbit_model;    /* VB_ORBIT_* */
  int      nsat;
  int      tsteps;         /* synthetic model: total steps */
  double   dt_s;
  double   alt_min_km, alt_max_km, spread_km;
  double   occ_R_m;        /* <= 0: upstream global cosphi from R=1737.1 km, h=300 km */
  float    bl_max_m;       /* upstream 100e3; <= 0: the uv grid covers the day's largest |u|, |v| */
  int      grid_res;       /* > 0 forces RES */
  int      seg_plan;       /* 0: even split (upstream); 1: seeded uneven counts */
  int      seg_min_half, seg_max_half;  /* seg_plan=1: half-baseline count range per segment */
  uint64_t seg_seed;
  int      stage2_cull;    /* 2: exact pixel-block culling in stage 2, 0: off */
  int      stage2_ppt;     /* stage-2 pixels per thread (vb_stage2_opts.ppt; 0 = auto) */
  int      stage2_items_per_cta;  /* vb_stage2_opts.items_per_cta */
  int      stage1_bpt;            /* vb_stage1_opts.bpt */
  int      stage1_stage_pix;      /* vb_stage1_opts.stage_pix */
  int      stage1_ctas_per_sm;    /* vb_stage1_opts.ctas_per_sm */
  int      stage1_items_per_cta;  /* vb_stage1_opts.items_per_cta */
  int      stage1_refine_pix;     /* vb_stage1_opts.refine_pix */
  int64_t  slab_pix;       /* > 0 and < npix: stream the sky through the device in slabs of this
                              many pixels (a multiple of 1024 and of viss_tile_pix); run with
                              vb_pipeline_run_host.  0: the whole sky is resident */
  int      use_graph;      /* 1: capture stages in one CUDA graph */
  int      device;         /* CUDA device ordinal */
  int      nm1_fast;       /* 1 (default): upstream all-visible fast path; 0: visible tiles take the
                              per-pixel test (vb_stage1_opts.mask_visible_tiles = 1) */
} vb_run_config;

typedef struct {
  int      npix_hi;        /* npix >> 31 */
  int      npix_lo;        /* npix & 0x7fffffff */
  int      nseg;
  int      n_half_total;
  long long stage1_terms;  /* nominal: sum_seg npix * N_half */
  long long stage2_terms;  /* nominal: sum_seg npix * nuniq */
  long long groups_total;
  double   t_stage1_ms;    /* CUDA-event time of the last run */
  double   t_stage2_ms;
  double   t_orbit_ms;
  unsigned long long s1_counters[4];
  unsigned long long s2_counters[4];
  double   w_scalar_total; /* blockage=0 normaliser (sum nuniq) */
  double   t_s1_kernel_ms; /* the stage-1 direct-sum kernel alone */
  double   t_s2_kernel_ms; /* the stage-2 reconstruction kernel alone */
  double   t_e2e_ms;       /* vb_pipeline_run_host: H2D, baselines, both stages, D2H */
  int      error_flags;    /* OR of the stage-1 and stage-2 device error words of the run
                              (VB_DEVERR_* bits, 0 = ok) */
  int      graph_kernels;  /* kernel nodes of the captured run graph (0 = eager) */
  double   bl_max_m;       /* bl_max the uv grids were built with (the automatic value when bl_max_m <= 0) */
} vb_report;

void vb_run_config_defaults(vb_run_config* c);

/* Allocates every device buffer for the run (no allocation afterwards),
 * generates the pixel geometry and tile meta.  Replaces the set-up block
 * main_recon_online.cu:150-218. */
int vb_pipeline_create(const vb_run_config* c, vb_pipeline** out);

/* Sky B (npix float32, NEST order, host memory) -> device; scale=1 applies
 * B *= 4*pi/npix in FP64 as main_recon_online.cu:106-112. */
int vb_pipeline_set_sky(vb_pipeline* p, const float* B_host, int scale);

/* Generates the day's baselines (all segments, resident) and validates the
 * +/- layout.  Replaces orbit_gen_init / orbit_gen_make_segment /
 * validate_uvw_halfsym_layout_ptr calls of main_recon_online.cu:260-287. */
int vb_pipeline_make_baselines(vb_pipeline* p);

/* Stage 1 + stage 2 for every segment (inputs resident on the device),
 * timed with CUDA events; synchronises.  Replaces the loop
 * main_recon_online.cu:274-512. */
int vb_pipeline_run(vb_pipeline* p, vb_report* r);

/* End to end from host memory: B_host -> device, baselines, both stages,
 * C_host (npix floats) and, if non-NULL, V_half_host (2*n_half floats) back. */
int vb_pipeline_run_host(vb_pipeline* p, const float* B_host, int scale,
                         float* C_host, float* V_half_host, vb_report* r);

/* One whole run in one call, as upstream main() does for one day
 * (main_recon_online.cu:5-586 without the file IO): builds a pipeline from c,
 * uploads B_host (npix floats, scaled by 4 pi / npix when scale is set),
 * generates the day's baselines, runs both stages, copies C (npix floats)
 * and, if V_half_host is non-NULL, the phase-corrected half-set V
 * (2 * n_half floats) back, and frees everything.  r (nullable) receives the
 * run's report.  npix_expected must equal 12 * nside^2 (a size check of the
 * caller's buffers). */
int vb_run(const vb_run_config* c, const float* B_host, int scale, int64_t npix_expected,
           float* C_host, float* V_half_host, vb_report* r);

/* Device pointers owned by the pipeline (valid until destroy), for tests and
 * writers.  name: "C","W","V_half","V_full","V_half_d","u","v","w","x1","y1","z1",
 * "x2","y2","z2","invn1","invn2","cosphi1","cosphi2","l","m","n","B","nm1",
 * "cx","cy","cz","cosA","sinA","seg_t0","seg_tlen","seg_params". */
int vb_pipeline_device_ptr(vb_pipeline* p, const char* name, void** ptr, int64_t* count);
int vb_pipeline_info(vb_pipeline* p, int64_t* npix, int* nseg, int* n_half_total,
                     int* nbl, int* ntile, float* cosphi);
int vb_pipeline_seg_plan(vb_pipeline* p, int* seg_t0, int* seg_tlen);   /* host arrays of nseg */
int vb_pipeline_seg_params(vb_pipeline* p, vb_seg_params* host_out);     /* host array of nseg; syncs */
int vb_pipeline_destroy(vb_pipeline* p);

/* Switches the pipeline to another day of the same run (new orbit window /
 * formation draw for that day, same buffers, plans and captured graph); the
 * next run generates the day's baselines.  Fails if the day's orbit has a
 * different step or pair count.  Replaces the per-day re-initialisation of
 * the upstream day loop (main_recon_online_mirror_tile_vissfast.cu:274-290). */
int vb_pipeline_set_day(vb_pipeline* p, int day);

/* acc[i] += C[i] in FP64 on the device (n values): the cross-day running sum
 * of daily images that the upstream post-processing keeps in a file
 * (combine.py:42-126, mirror_tile_vissfast/viss_monitor.py:92-139). */
int vb_accumulate(const float* C, int64_t n, double* acc, void* stream);

/* Autotuner (no upstream counterpart: upstream fixes 256-thread blocks and one
 * block per 256 baselines or pixels).  Times the stage-1 kernel over baselines
 * per thread x staged pixels x resident CTAs per SM x work-queue granularity,
 * then the stage-2 kernel over pixels per thread x granularity, on this
 * pipeline's own resident inputs (sky and baselines must be set), keeps the
 * fastest shape of each stage in the pipeline's config (the next run
 * re-captures its graph) and reports it.  reps: timed runs per candidate
 * (min taken; 0 = 2).  The pipeline's workspaces grow when a candidate needs
 * more; nothing else is allocated. */
typedef struct {
  int    stage1_bpt, stage1_stage_pix, stage1_ctas_per_sm, stage1_items_per_cta;
  int    stage2_ppt, stage2_items_per_cta;
  double stage1_ms, stage2_ms;                 /* best kernel times */
  double stage1_default_ms, stage2_default_ms; /* the untuned (auto) shapes */
  int    candidates;                           /* shapes timed */
} vb_tune_report;
int vb_pipeline_autotune(vb_pipeline* p, int reps, vb_tune_report* out);

/* sizeof() of a public struct by its type name ("vb_sky", "vb_baselines",
 * "vb_stage1_opts", "vb_stage2_opts", "vb_seg_params", "vb_orbit_params",
 * "vb_run_config", "vb_report", "vb_tune_report"); 0 for an unknown name.
 * Lets FFI bindings check their struct layouts. */
size_t vb_abi_sizeof(const char* type_name);

/* ------------------------------------------------------------------------ */
/* measurement helpers                                                        */
/* ------------------------------------------------------------------------ */
/* Throughput of the SFU sincos pipe and the FP32 / FP64 FMA pipes on this GPU
 * (results per second over the whole device), by a short dependent-chain-free
 * microbenchmark (~50 ms).  Used as the roofline denominator. */
int vb_measure_peaks(double* sfu_sincos_per_s, double* fp32_fma_per_s,
                     double* fp64_fma_per_s, double* sm_clock_mhz);

/* Writes `bytes` of zeros to a device buffer (L2 flush helper). */
int vb_flush_l2(void* buf, size_t bytes, void* stream);

/* ------------------------------------------------------------------------ */
/* host plumbing for callers without a CUDA binding (cgo / JNI / ctypes)     */
/* ------------------------------------------------------------------------ */
#define VB_H2D 0
#define VB_D2H 1
#define VB_D2D 2
int vb_set_device(int device);
int vb_host_alloc(void** ptr, size_t bytes);   /* page-locked host memory */
int vb_host_free(void* ptr);
int vb_malloc(void** ptr, size_t bytes);
int vb_free(void* ptr);
int vb_memcpy(void* dst, const void* src, size_t bytes, int kind);   /* synchronous */
int vb_memset(void* ptr, int value, size_t bytes);
int vb_synchronize(void);

/* Seeded synthetic sky in NEST order: B_p ~ U[0,1) (24-bit uniform) plus
 * `n_points` point sources of amplitude `amp` at seeded indices (added).
 * std::mt19937_64(seed).  Host memory, npix = 12*nside^2 floats. */
int vb_make_synthetic_sky(int nside, uint64_t seed, int n_points, float amp, float* B_host);

/* Stage-1 tile class of every (half-baseline, cull tile) pair as used by
 * vb_viss_halfsym for opts->cull: 0 hidden, 1 visible (no per-pixel mask),
 * 2 mixed (per-pixel mask).  cls (device memory; VB_ERR_INVALID otherwise) has
 * n_half * ntile bytes, row-major per half-baseline; *ntile_out = number of cull tiles.  Exported for parity
 * tests (the upstream decision is the inline block at
 * viss_recon_kernel_mirror_tile_vissfast.cuh:519-529). */
int vb_stage1_tile_classes(const vb_sky* sky, const vb_baselines* bl, const vb_stage1_opts* o,
                           void* workspace, size_t ws_bytes, uint8_t* cls, int* ntile_out,
                           void* stream);

#ifdef __cplusplus
}
#endif
#endif /* VISSB200_H */
