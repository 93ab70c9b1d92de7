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
//  * every GPU that loads this library holds the array (and the status word
//    beside it) until the process exits;
//  * all calls share the one array and it keeps the last call's contents.
//    Nothing in it has to start at zero: the stiffness kernel writes every
//    residual word before the gather reads it.  The status word does start at
//    zero: each call clears it on its stream before the launches.  Calls that
//    overlap on the GPU (different streams, or different host threads on one
//    device) race on the array and the status word and must be serialised by
//    the caller;
//  * the first call on a device looks up the device addresses of the array
//    and the status word with cudaGetSymbolAddress while that device is
//    current, and caches them.  Make that first call before any stream
//    capture;
//  * meshes whose stiffness kernel has bounded device waits (FP32 tensor-core
//    tetrahedra and triangles) report a wait that gave up through the status
//    word; for them the call reads the word back and synchronises the stream
//    before it returns, and returns SALVUS_E_TIMEOUT when a wait gave up.
//    Every other mesh returns as soon as the work is queued;
//  * the call makes the mesh's device current for its launches and restores
//    the caller's current device before it returns.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "internal.h"

namespace salvus {
// Defined with the other launches in abi.cu: a = -K u for the caller's
// device buffers, element-local residual in `scratch`, bounded-wait timeouts
// recorded in the device word `err`.
int apply_stiffness_into(const salvus_mesh *m, int precision, const void *u, void *a,
                         void *scratch, int *err, cudaStream_t st);
bool stiffness_reports_errors(const salvus_mesh *m, int precision);
}  // namespace salvus

namespace {

constexpr size_t kScratchBytes = size_t(32) << 20;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];
static __device__ __align__(256) int g_noalloc_status;

std::mutex g_scratch_mutex;
void *g_scratch_ptr[kMaxDevices] = {nullptr};
int *g_status_ptr[kMaxDevices] = {nullptr};

// Device addresses of g_noalloc_scratch and g_noalloc_status on the current
// device (looked up once per device; in host code the symbols themselves are
// only host-side stand-ins).
int scratch_address(int device, void **scratch, int **status) {
  if (device < 0 || device >= kMaxDevices)
    return salvus::fail(SALVUS_E_INVALID, "device %d out of range", device);
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  if (!g_scratch_ptr[device]) {
    void *p = nullptr, *q = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return salvus::fail(SALVUS_E_CUDA, "cudaGetSymbolAddress(scratch) failed: %s",
                          cudaGetErrorString(e));
    e = cudaGetSymbolAddress(&q, g_noalloc_status);
    if (e != cudaSuccess || !q)
      return salvus::fail(SALVUS_E_CUDA, "cudaGetSymbolAddress(status) failed: %s",
                          cudaGetErrorString(e));
    g_status_ptr[device] = static_cast<int *>(q);
    g_scratch_ptr[device] = p;
  }
  *scratch = g_scratch_ptr[device];
  *status = g_status_ptr[device];
  return SALVUS_OK;
}

// Makes `device` current and puts the caller's device back on scope exit.
struct DeviceGuard {
  int prev = -1;
  bool changed = false;
  int enter(int device) {
    cudaError_t e = cudaGetDevice(&prev);
    if (e != cudaSuccess)
      return salvus::fail(SALVUS_E_CUDA, "cudaGetDevice failed: %s", cudaGetErrorString(e));
    if (prev != device) {
      e = cudaSetDevice(device);
      if (e != cudaSuccess)
        return salvus::fail(SALVUS_E_CUDA, "cudaSetDevice failed: %s", cudaGetErrorString(e));
      changed = true;
    }
    return SALVUS_OK;
  }
  ~DeviceGuard() {
    if (changed) cudaSetDevice(prev);
  }
};

}  // namespace

extern "C" int salvus_apply_stiffness_noalloc(const salvus_mesh *mesh, int32_t precision,
                                              const void *u, void *a, void *stream) {
  if (!mesh || !u || !a) return salvus::fail(SALVUS_E_INVALID, "null argument");
  if (precision != SALVUS_FP32 && precision != SALVUS_FP64)
    return salvus::fail(SALVUS_E_INVALID, "unknown precision %d", precision);
  if (precision == SALVUS_FP64 && mesh->fp32_only)
    return salvus::fail(SALVUS_E_STATE,
                        "FP64 call on a mesh created with SALVUS_MESH_FP32_ONLY (no FP64 records)");
  if (mesh->physics == SALVUS_COUPLED2D)
    return salvus::fail(SALVUS_E_UNSUPPORTED,
                        "fluid-solid meshes: the coupling terms act on the velocity field, which "
                        "this entry point does not take");
  if (mesh->host_only) return salvus::fail(SALVUS_E_STATE, "host-only mesh");
  const size_t rsize = precision == SALVUS_FP32 ? 4 : 8;
  const size_t need = (size_t)mesh->E * mesh->P * mesh->c * rsize;
  if (need > kScratchBytes)
    return salvus::fail(SALVUS_E_INVALID,
                        "mesh needs %zu bytes of element-local scratch; the allocation-free "
                        "entry point holds at most %zu bytes",
                        need, kScratchBytes);
  DeviceGuard guard;
  int rc = guard.enter(mesh->device);
  if (rc) return rc;
  void *scratch = nullptr;
  int *status = nullptr;
  if ((rc = scratch_address(mesh->device, &scratch, &status))) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e = cudaMemsetAsync(status, 0, sizeof(int), st);
  if (e != cudaSuccess)
    return salvus::fail(SALVUS_E_CUDA, "clearing the status word failed: %s",
                        cudaGetErrorString(e));
  if ((rc = salvus::apply_stiffness_into(mesh, precision, u, a, scratch, status, st))) return rc;
  if (!salvus::stiffness_reports_errors(mesh, precision)) return SALVUS_OK;
  int h = 0;
  e = cudaMemcpyAsync(&h, status, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess)
    return salvus::fail(SALVUS_E_CUDA, "reading the status word failed: %s", cudaGetErrorString(e));
  if (h)
    return salvus::fail(SALVUS_E_TIMEOUT,
                        "a bounded device wait gave up (code %d); the output is invalid", h);
  return SALVUS_OK;
}
