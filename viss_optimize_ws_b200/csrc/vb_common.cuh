// Internal helpers shared by every translation unit of libvissb200.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <cstdarg>

#include "vissb200.h"

namespace vb {

// --- error reporting -------------------------------------------------------
// Sets the thread-local message returned by vb_last_error() and returns code.
int fail(int code, const char* fmt, ...);
int cuda_fail(cudaError_t e, const char* what, const char* file, int line);

#define VB_CUDA(call)                                                       \
  do {                                                                      \
    cudaError_t vb_e_ = (call);                                             \
    if (vb_e_ != cudaSuccess)                                               \
      return ::vb::cuda_fail(vb_e_, #call, __FILE__, __LINE__);             \
  } while (0)

#define VB_LAUNCH_CHECK() VB_CUDA(cudaGetLastError())

#define VB_TRY(expr)                                                        \
  do {                                                                      \
    int vb_rc_ = (expr);                                                    \
    if (vb_rc_ != VB_OK) return vb_rc_;                                     \
  } while (0)

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }
inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// Device-side error word bits (written with atomicOr, read by the host).
enum : unsigned {
  ERR_WAIT_TIMEOUT = 1u << 0,   // a bounded wait gave up
  ERR_BAD_INDEX    = 1u << 1,   // an index check failed and the access was skipped
  ERR_HALFSYM      = 1u << 2,   // +/- pair layout violated
  ERR_PHASE_RANGE  = 1u << 3,   // F32X phase outside its exact range (|u|+|v|+|w| >= 2^28 turns)
};

// Upstream half -> full signed index map (common.hpp:213-220 generalised to
// `nbl` pairs per step): step = ih / nbl, j = ih % nbl, full = step*2*nbl + j.
__host__ __device__ inline int half_to_full_pos(int ih, int nbl) {
  int step = ih / nbl;
  return step * 2 * nbl + (ih - step * nbl);
}

// Bump allocator over a caller-provided workspace (256-byte aligned slices).
struct Carve {
  char* base;
  size_t cap;
  size_t off = 0;
  bool ok = true;
  Carve(void* b, size_t c) : base(static_cast<char*>(b)), cap(c) {}
  template <class T>
  T* take(size_t count) {
    off = align_up(off, 256);
    size_t bytes = count * sizeof(T);
    if (base == nullptr) { off += bytes; return nullptr; }   // size query
    if (off + bytes > cap) { ok = false; off += bytes; return nullptr; }
    T* p = reinterpret_cast<T*>(base + off);
    off += bytes;
    return p;
  }
  size_t used() const { return align_up(off, 256); }
};

int sm_count();   // cached SM count of the current device

// Records an event so that it also records when the work is replayed from a
// CUDA graph: inside a stream capture it must be an external event node
// (a plain record there only orders streams).
inline cudaError_t record_event(cudaEvent_t e, cudaStream_t s) {
  cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
  cudaError_t r = cudaStreamIsCapturing(s, &st);
  if (r != cudaSuccess) return r;
  if (st == cudaStreamCaptureStatusActive) return cudaEventRecordWithFlags(e, s, cudaEventRecordExternal);
  return cudaEventRecord(e, s);
}

}  // namespace vb
