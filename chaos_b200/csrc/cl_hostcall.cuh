// cl_hostcall.cuh -- the host-buffer form of the recorder entry points: device copies of the caller's arrays on a
// private stream, the launch windows [run.n0, run.N) of run.steps steps each (the reference's step-chunked
// relaunch), the arrays marked for return copied back, the device time of the launches in the provenance, and every
// buffer given back to the library's pool on every path.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../../include/chaoslab_b200.h"

namespace cl {

int capi_map_cuda(cudaError_t e, const char* where);  // cl_capi.cu

// Device buffers of a host-buffer call, from the library's per-device stream-ordered pool (cl_capi.cu), which keeps
// the memory between calls; pool_free gives the buffer back in the order of `st`.
cudaError_t pool_alloc(void** p, size_t bytes, cudaStream_t st);
void pool_free(void* p, cudaStream_t st);

// Write one byte in every page of a caller's output array while the device computes: a fresh array's pages are
// mapped and zeroed by the operating system on first touch, and when that happens inside the copy back from the
// device it costs about as much as the copy itself (38 MB: 9.4 ms into fresh pages, 2.3 ms into touched ones); here
// it overlaps the kernels. The array's contents are overwritten by the copy that follows. Only pageable memory is
// touched: a copy from it to the device has read it before cudaMemcpyAsync returns, while a pinned (or managed)
// array is resident already and may still be in flight as an input.
inline void touch_pages(void* p, size_t bytes) {
    if (!p || !bytes) return;
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return;
    }
    if (at.type != cudaMemoryTypeUnregistered) return;
    volatile char* c = static_cast<volatile char*>(p);
    for (size_t o = 0; o < bytes; o += 4096) c[o] = 0;
    c[bytes - 1] = 0;
}

// One caller array: `host` may be NULL (then `dev` stays NULL and the device entry point skips it); `back` copies
// it to the host after the last window.
struct HostArray {
    void* host;
    size_t bytes;
    bool back;
    void* dev;
};

// `window(r, stream)` enqueues one launch window `r` (r.n0, r.steps set) on the device copies and returns 0 or the
// library's error code.
template <class Window>
int host_windows(const cl_run& run, std::vector<HostArray>& arrays, Window&& window, cl_prov* prov, const char* what) {
    cudaStream_t st = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int rc = 0;
    int64_t launches = 0;
    const int64_t L = run.steps > 0 ? run.steps : run.N - run.n0;
    cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    for (HostArray& a : arrays) {
        a.dev = nullptr;
        if (e == cudaSuccess && a.host) e = pool_alloc(&a.dev, std::max<size_t>(a.bytes, 1), st);
    }
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    if (e == cudaSuccess) {
        for (const HostArray& a : arrays)
            if (a.host && a.bytes) cudaMemcpyAsync(a.dev, a.host, a.bytes, cudaMemcpyHostToDevice, st);
        cudaEventRecord(e0, st);
        cl_run r = run;
        for (int64_t n0 = run.n0; n0 < run.N && rc == 0; n0 += L) {
            r.n0 = n0;
            r.steps = std::min<int64_t>(L, run.N - n0);
            rc = window(r, st);
            ++launches;
        }
        cudaEventRecord(e1, st);
        if (rc == 0) {
            for (const HostArray& a : arrays)
                if (a.host && a.back) touch_pages(a.host, a.bytes);
            for (const HostArray& a : arrays)
                if (a.host && a.back && a.bytes) cudaMemcpyAsync(a.host, a.dev, a.bytes, cudaMemcpyDeviceToHost, st);
        }
        e = cudaStreamSynchronize(st);
    }
    if (rc == 0 && e != cudaSuccess) rc = capi_map_cuda(e, what);
    if (rc == 0 && prov) {
        std::memset(prov, 0, sizeof *prov);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        prov->gpu_ms = ms;
        prov->launches = launches;
        prov->launch_steps = L;
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    for (HostArray& a : arrays)
        if (a.dev) pool_free(a.dev, st);
    if (st) cudaStreamDestroy(st);
    return rc;
}

}  // namespace cl
