// cl_noalloc.cu -- the ensemble entry point that allocates nothing.
//
// Some callers cannot allocate GPU memory while they call in: a host that owns the whole device heap through its
// own pool (a Julia or Python runtime with its own caching allocator, where a foreign cudaMalloc would fragment or
// fail against it), a sandboxed plugin host that forbids allocation calls from plugins, or a latency-bound loop that
// cannot afford the synchronisation a cudaMalloc / cudaFree may cost. For them `cl_b200_ensemble_device_noalloc`
// runs the same ensemble kernels with the queue heads (the kernels' only scratch memory) in a fixed array that
// lives in this file: CL_NOALLOC_MAX_CLASSES heads of 8 bytes (512 bytes), resident on every GPU that loads the
// library until the process exits.
//
// In host code `g_queue_heads` names a host-side stand-in, not the device array, so a kernel is never handed the
// symbol itself: every call asks the runtime for the array's device address in the current context
// (cudaGetSymbolAddress, a lookup that allocates nothing and is allowed during stream capture) and passes it to the
// kernels, so a reset of the device or its primary context between calls leaves no stale address. Every call shares
// the array and clears the heads it uses (cudaMemsetAsync, on the caller's stream) before its launches; calls that
// overlap on the GPU race on it. A call whose classes are rejected enqueues nothing.
#include <cuda_runtime.h>

#include <string>

#include "../../include/chaoslab_b200.h"
#include "cl_ensemble.cuh"

namespace cl {

int capi_fail(int code, const std::string& msg);
int capi_map_cuda(cudaError_t e, const char* where);
int validate_classes(const cl_ensemble_class* cs, int nc);
int enqueue_classes_in_order(const cl_ensemble_class* cs, int nc, unsigned long long* heads, cudaStream_t st);

namespace {

static __device__ __align__(256) unsigned long long g_queue_heads[CL_NOALLOC_MAX_CLASSES];

// The device address of g_queue_heads in the current context, looked up on every call (a lookup, no allocation):
// a cached address would go stale when the context is reset and the module reloaded.
int heads_on_current_device(unsigned long long** out) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_queue_heads);
    if (e != cudaSuccess) return capi_map_cuda(e, "address of the fixed queue heads");
    *out = static_cast<unsigned long long*>(p);
    return 0;
}

}  // namespace
}  // namespace cl

using namespace cl;

extern "C" int cl_b200_ensemble_device_noalloc(const cl_ensemble_class* classes, int32_t n_classes, void* stream) {
    if (!classes || n_classes < 1) return capi_fail(CL_EINVAL, "no classes");
    if (n_classes > CL_NOALLOC_MAX_CLASSES)
        return capi_fail(CL_EINVAL, "at most " + std::to_string(CL_NOALLOC_MAX_CLASSES) +
                                        " classes per call without allocation (the fixed queue-head array)");
    // a rejected call enqueues nothing, not even the clearing of the shared heads
    int rc = validate_classes(classes, n_classes);
    if (rc) return rc;
    unsigned long long* heads = nullptr;
    rc = heads_on_current_device(&heads);
    if (rc) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const cudaError_t e = cudaMemsetAsync(heads, 0, sizeof(unsigned long long) * n_classes, st);
    if (e != cudaSuccess) return capi_map_cuda(e, "clear the queue heads");
    return enqueue_classes_in_order(classes, n_classes, heads, st);
}
