// Stage-1 visibility sum for callers that cannot allocate device memory.
//
// vb_viss_halfsym needs scratch (packed pixel records, per-chunk partial
// sums, a work counter) that its caller allocates.  Some callers cannot call
// cudaMalloc at all: plug-in hosts whose device memory is owned by another
// allocator with a fixed budget (a cudaMalloc behind its back can fail or
// break its accounting), and real-time loops that must not pay the latency
// and implicit device synchronisation of cudaMalloc / cudaFree.  This entry
// point takes only its inputs and outputs and keeps its scratch in one
// file-scope device array of fixed maximum size, which every GPU that loads
// the library holds until exit.  Under CUDA's lazy module loading (the
// default), the array is reserved when this file's module is first loaded on
// a device, i.e. at the first call on that device.
#include "vb_common.cuh"
#include "vb_internal.h"

namespace vb {
namespace {

// The scratch lives here.  In host code `g_viss_scratch` names a host-side
// stand-in, never the device memory: only the address returned by
// cudaGetSymbolAddress (taken with the device current) may be given to kernels.
static __device__ __align__(256) unsigned char g_viss_scratch[VB_VISS_NOALLOC_MAX_BYTES];

// Device address of the scratch in the current device's context.  Looked up on
// every call: the lookup is cheap once the module is loaded, and a cached
// address would dangle after the context is torn down and re-created
// (cudaDeviceReset), when the module can load at another address.  The first
// call on a device loads the module (and so reserves the array).
int scratch_address(void** out) {
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_viss_scratch);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_viss_scratch)", __FILE__, __LINE__);
  *out = p;
  return VB_OK;
}

}  // namespace
}  // namespace vb

using namespace vb;

extern "C" int vb_viss_halfsym_noalloc(const vb_sky* sky, const vb_baselines* bl, const vb_stage1_opts* o,
                                       double* V_half, unsigned long long* term_counters, unsigned* error_flags,
                                       void* stream) {
  Stage1Plan p;
  VB_TRY(stage1_plan(sky, bl, o, &p));
  cudaStream_t s = as_stream(stream);
  if (p.n_half == 0) {
    if (error_flags) VB_CUDA(cudaMemsetAsync(error_flags, 0, sizeof(unsigned), s));
    return VB_OK;
  }
  if (!V_half) return fail(VB_ERR_INVALID, "vb_viss_halfsym_noalloc: V_half is NULL");
  if (!sky->B || !sky->l || !sky->m || !sky->n) return fail(VB_ERR_INVALID, "vb_viss_halfsym_noalloc: sky arrays missing");
  if (!bl->u || !bl->v || !bl->w) return fail(VB_ERR_INVALID, "vb_viss_halfsym_noalloc: u/v/w missing");
  if (p.blockage && (!bl->x1 || !bl->y1 || !bl->z1 || !bl->invn1 || !bl->x2 || !bl->y2 || !bl->z2 || !bl->invn2))
    return fail(VB_ERR_INVALID, "vb_viss_halfsym_noalloc: endpoint arrays missing");
  size_t need = stage1_carve(p, nullptr, 0, nullptr, true);
  // Fit an automatic plan into the fixed scratch: fewer, larger pixel chunks
  // shrink the partial-sum buffer (results stay within FP32-sum rounding of
  // the default plan).  A chunk size the caller set is kept as given.
  while (o->chunk_pix <= 0 && need > (size_t)VB_VISS_NOALLOC_MAX_BYTES && p.nchunk > 1) {
    int64_t chunk = (int64_t)p.chunk_pix * 2;
    int64_t max_chunk = ceil_div(p.npix, p.cull_tile) * (int64_t)p.cull_tile;
    if (chunk > max_chunk) chunk = max_chunk;
    if (chunk > INT32_MAX) break;
    p.chunk_pix = (int)chunk;
    p.nchunk = (int)ceil_div(p.npix, p.chunk_pix);
    p.n_items = p.n_btile * p.nchunk;
    if (p.grid > p.n_items) p.grid = p.n_items;
    need = stage1_carve(p, nullptr, 0, nullptr, true);
  }
  if (need > (size_t)VB_VISS_NOALLOC_MAX_BYTES)
    return fail(VB_ERR_UNSUPPORTED,
                "vb_viss_halfsym_noalloc: this sky/baseline set%s needs %zu bytes of scratch, above the fixed "
                "maximum of %zu bytes (npix=%lld, n_half=%d); use vb_viss_halfsym with a caller workspace",
                o->chunk_pix > 0 ? " with the given chunk_pix" : "", need, (size_t)VB_VISS_NOALLOC_MAX_BYTES,
                (long long)p.npix, p.n_half);
  void* base = nullptr;
  VB_TRY(scratch_address(&base));
  Stage1Buffers b;
  stage1_carve(p, base, (size_t)VB_VISS_NOALLOC_MAX_BYTES, &b, true);
  // the array keeps the previous call's contents: clear what must start at zero
  VB_CUDA(cudaMemsetAsync(b.err, 0, sizeof(unsigned), s));
  VB_TRY(stage1_run(sky, bl, p, b, false, V_half, term_counters, s));
  if (error_flags) VB_CUDA(cudaMemcpyAsync(error_flags, b.err, sizeof(unsigned), cudaMemcpyDeviceToDevice, s));
  return VB_OK;
}
