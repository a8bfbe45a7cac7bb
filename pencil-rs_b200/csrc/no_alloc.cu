// Allocation-free execution of an existing plan.
//
// Some callers of this library cannot call cudaMalloc at the point where they
// execute a transform: code running inside a host callback or a real-time loop
// where an allocation could block on the device, frameworks whose device
// memory is owned by a pool that does not hand out raw scratch, and embedders
// with a fixed device-memory budget decided up front.  pb_execute needs a
// caller workspace (the intermediate pencil buffers and the C2R spectrum-check
// words); pb_execute_no_alloc runs the same passes with that workspace taken
// from one file-scope device array instead, so the call allocates nothing.
//
// The array has a fixed size, PB_NO_ALLOC_SCRATCH_BYTES, and every GPU that
// loads the library holds it until the process exits.  Plans whose workspace
// is larger are rejected with PB_ENO_ALLOC_LIMIT before any device work.
#include <cuda_runtime.h>

#include <mutex>

#include "pb_aux.hpp"
#include "pencil_b200.h"

namespace pb {

static __device__ __align__(256) unsigned char g_no_alloc_scratch[PB_NO_ALLOC_SCRATCH_BYTES];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_scratch_mutex;
void* g_scratch_ptr[kMaxDevices] = {};
}  // namespace

// Device address of the scratch array on the current device.  In host code the
// array's name is only a host-side stand-in, so the address is looked up once
// per device (with that device current) and cached.
static int no_alloc_scratch(void** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return PB_ECUDA;
  if (dev < 0 || dev >= kMaxDevices) return PB_EUNSUPPORTED;
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  if (g_scratch_ptr[dev] == nullptr) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_no_alloc_scratch) != cudaSuccess || p == nullptr) return PB_ECUDA;
    g_scratch_ptr[dev] = p;
  }
  *out = g_scratch_ptr[dev];
  return PB_OK;
}

}  // namespace pb

extern "C" int pb_execute_no_alloc(pb_plan* plan, int32_t op, const void* in, void* out, void* stream) {
  if (!plan) return PB_ENULL;
  const long long need = pb::plan_workspace_bytes(plan);
  if (need < 0) return PB_EINVALID_ARGUMENT;
  if ((unsigned long long)need > (unsigned long long)PB_NO_ALLOC_SCRATCH_BYTES) return PB_ENO_ALLOC_LIMIT;
  void* scratch = nullptr;
  const int rc = pb::no_alloc_scratch(&scratch);
  if (rc != PB_OK) return rc;
  return pb::execute_with_workspace(plan, op, in, out, scratch, stream, /*report_spectrum=*/1);
}
