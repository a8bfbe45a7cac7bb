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
unsigned long long g_scratch_ctx[kMaxDevices] = {};  // context the address was looked up in

using CtxGetCurrent = int (*)(void** ctx);
using CtxGetId = int (*)(void* ctx, unsigned long long* id);

// Unique id of the calling thread's current context (driver entry points
// cuCtxGetCurrent / cuCtxGetId, resolved through the runtime so the library
// does not link libcuda).  Returns false when no context is current yet.
bool current_context_id(unsigned long long* id) {
  static CtxGetCurrent get_current = nullptr;
  static CtxGetId get_id = nullptr;
  static bool resolved = false;
  if (!resolved) {
    void* f0 = nullptr;
    void* f1 = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f0, cudaEnableDefault, nullptr) == cudaSuccess &&
        cudaGetDriverEntryPoint("cuCtxGetId", &f1, cudaEnableDefault, nullptr) == cudaSuccess) {
      get_current = reinterpret_cast<CtxGetCurrent>(f0);
      get_id = reinterpret_cast<CtxGetId>(f1);
    }
    resolved = true;
  }
  if (!get_current || !get_id) return false;
  void* ctx = nullptr;
  if (get_current(&ctx) != 0 || ctx == nullptr) return false;
  return get_id(ctx, id) == 0;
}
}  // namespace

// Device address of the scratch array in the current device's context.  In
// host code the array's name is only a host-side stand-in, so the address is
// looked up with cudaGetSymbolAddress once per device (with that device
// current) and cached together with the id of the context it belongs to.  A
// new context on the same device (after cudaDeviceReset the runtime creates a
// fresh primary context and loads the module again, at another address) has
// another id, and the address is looked up again.
static int no_alloc_scratch(void** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return PB_ECUDA;
  if (dev < 0 || dev >= kMaxDevices) return PB_EUNSUPPORTED;
  std::lock_guard<std::mutex> lock(g_scratch_mutex);  // also guards the entry-point resolution
  unsigned long long ctx = 0;
  bool have_ctx = current_context_id(&ctx);
  if (g_scratch_ptr[dev] == nullptr || !have_ctx || g_scratch_ctx[dev] != ctx) {
    void* p = nullptr;
    // makes the device's primary context current when none is
    if (cudaGetSymbolAddress(&p, g_no_alloc_scratch) != cudaSuccess || p == nullptr) return PB_ECUDA;
    if (!have_ctx) have_ctx = current_context_id(&ctx);
    g_scratch_ptr[dev] = p;
    g_scratch_ctx[dev] = have_ctx ? ctx : 0;
    if (!have_ctx) {  // no context id to key on: look the address up on every call
      *out = p;
      g_scratch_ptr[dev] = nullptr;
      return PB_OK;
    }
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
