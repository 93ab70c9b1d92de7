// noalloc.cu -- an entry point that applies the assembled stiffness operator
// without allocating any device memory.
//
// Who needs it: callers that cannot call cudaMalloc during a run.  Examples
// are host frameworks that own every byte of device memory through their own
// pool (a solver embedded as a custom operator, a memory-capped service that
// reserves its budget up front) and code paths that must not touch the
// allocator at all while they run.  Such a caller hands in its own input and
// output buffers; the element-local residual that the deterministic assembly
// needs between the stiffness kernel and the node gather lives in the
// file-scope array below instead of a buffer this library allocates.
//
// Limits and sharing rules:
//  * the array holds kScratchBytes (32 MiB); a mesh whose element-local
//    residual E * P * c * sizeof(real) exceeds that is rejected with
//    SALVUS_E_INVALID and a message giving both sizes;
//  * every GPU that loads this library holds the array until the process
//    exits;
//  * all calls share the one array and it keeps the last call's contents.
//    Nothing in it has to start at zero: the stiffness kernel writes every
//    residual word before the gather reads it.  Calls that overlap on the GPU
//    (different streams, or different host threads on one device) race on
//    the array and must be serialised by the caller;
//  * the first call on a device looks up the array's device address with
//    cudaGetSymbolAddress while that device is current, and caches it.  Make
//    that first call before any stream capture.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "internal.h"

namespace salvus {
// Defined with the other launches in abi.cu: a = -K u for the caller's
// device buffers, element-local residual in `scratch`.
int apply_stiffness_into(const salvus_mesh *m, int precision, const void *u, void *a,
                         void *scratch, cudaStream_t st);
}  // namespace salvus

namespace {

constexpr size_t kScratchBytes = size_t(32) << 20;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_scratch_mutex;
void *g_scratch_ptr[kMaxDevices] = {nullptr};

// Device address of g_noalloc_scratch on the current device (looked up once
// per device; in host code the symbol itself is only a host-side stand-in).
int scratch_address(int device, void **out) {
  if (device < 0 || device >= kMaxDevices)
    return salvus::fail(SALVUS_E_INVALID, "device %d out of range", device);
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  if (!g_scratch_ptr[device]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return salvus::fail(SALVUS_E_CUDA, "cudaGetSymbolAddress(scratch) failed: %s",
                          cudaGetErrorString(e));
    g_scratch_ptr[device] = p;
  }
  *out = g_scratch_ptr[device];
  return SALVUS_OK;
}

}  // namespace

extern "C" int salvus_apply_stiffness_noalloc(const salvus_mesh *mesh, int32_t precision,
                                              const void *u, void *a, void *stream) {
  if (!mesh || !u || !a) return salvus::fail(SALVUS_E_INVALID, "null argument");
  if (mesh->host_only) return salvus::fail(SALVUS_E_STATE, "host-only mesh");
  if (precision != SALVUS_FP32 && precision != SALVUS_FP64)
    return salvus::fail(SALVUS_E_INVALID, "unknown precision %d", precision);
  const size_t rsize = precision == SALVUS_FP32 ? 4 : 8;
  const size_t need = (size_t)mesh->E * mesh->P * mesh->c * rsize;
  if (need > kScratchBytes)
    return salvus::fail(SALVUS_E_INVALID,
                        "mesh needs %zu bytes of element-local scratch; the allocation-free "
                        "entry point holds at most %zu bytes",
                        need, kScratchBytes);
  cudaError_t e = cudaSetDevice(mesh->device);
  if (e != cudaSuccess)
    return salvus::fail(SALVUS_E_CUDA, "cudaSetDevice failed: %s", cudaGetErrorString(e));
  void *scratch = nullptr;
  int rc = scratch_address(mesh->device, &scratch);
  if (rc) return rc;
  return salvus::apply_stiffness_into(mesh, precision, u, a, scratch, (cudaStream_t)stream);
}
