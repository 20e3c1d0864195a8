// Rendering without any device allocation.
//
// lmgpu_render_device caches its wavefront workspace (path state, ray and
// shadow queues) in memory it allocates with cudaMalloc on first use. Some
// callers cannot allow that: a render callback of a host application whose
// memory manager forbids device allocations, or a process already at its
// memory budget. This entry point runs the same waves over a fixed workspace
// that lives in this file's static device array instead, so a call allocates
// nothing. Like lmgpu_render_device, it reads each bounce's queue sizes back
// to the host, so it synchronises its stream after every bounce.
#include <cuda_runtime.h>
#include <mutex>

#include "../../include/lmgpu.h"
#include "internal.h"

namespace lmgpu {
namespace {

// Size of the static workspace: every GPU that loads this module holds it
// until the process exits. 32 MiB gives waves of 155,343 paths.
constexpr size_t NOALLOC_WORKSPACE_BYTES = size_t(32) << 20;

__device__ __align__(256) unsigned char g_noalloc_workspace[NOALLOC_WORKSPACE_BYTES];

constexpr int MAX_DEVICES = 64;
std::mutex g_mu;
void* g_workspace_ptr[MAX_DEVICES] = {};          // device address of the array, per device
uint32_t g_host_counts[MAX_DEVICES][4] = {};       // queue-counter readback, per device

// Device address of the array on the current device. In host code the
// array's name is a host-side stand-in, not a device address, so it is
// looked up once per device with that device current.
int workspace_address(void** out)
{
    int dev = 0;
    LMGPU_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= MAX_DEVICES) return fail(LMGPU_ERR_UNSUPPORTED, "device index beyond the no-alloc table");
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_workspace_ptr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_workspace);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(no-alloc workspace)");
        g_workspace_ptr[dev] = p;
    }
    *out = g_workspace_ptr[dev];
    return LMGPU_OK;
}

}  // namespace
}  // namespace lmgpu

using namespace lmgpu;

extern "C" {

int lmgpu_render_device_noalloc(LmgpuScene* scene, const LmgpuRenderParams* params, void* film_device, void* stream)
{
    if (!scene || !params || !film_device) return fail(LMGPU_ERR_INVALID, "null argument");
    const int64_t max_paths = workspace_paths_for_bytes(NOALLOC_WORKSPACE_BYTES);
    if (params->wave_paths > max_paths)
        return fail(LMGPU_ERR_INVALID, "wave_paths exceeds the no-alloc workspace (at most " +
                                       std::to_string(max_paths) + " paths per wave)");
    void* ws = nullptr;
    int rc = workspace_address(&ws);
    if (rc != LMGPU_OK) return rc;
    int dev = 0;
    LMGPU_CUDA_TRY(cudaGetDevice(&dev));
    return render_device_preallocated(scene, *params, film_device, static_cast<cudaStream_t>(stream), ws,
                                      NOALLOC_WORKSPACE_BYTES, g_host_counts[dev]);
}

}  // extern "C"
