// Host-side internals shared by the CUDA translation units.
#pragma once
#include <cuda_runtime.h>
#include <atomic>
#include <string>
#include <vector>
#include "../../include/lmgpu.h"
#include "scene.cuh"

// Staging for the host-buffer entry points: SLOTS streams, each with a
// device chunk of AoS rays and SoA hits. With four slots the upload of chunk
// c + 2 does not queue behind the download of chunk c, so both copy
// directions stay busy at once.
struct HostPipeline {
    static constexpr int SLOTS = 4;
    bool ready = false;
    int64_t chunk = 0;
    cudaStream_t stream[SLOTS] = {};
    float* rays[SLOTS] = {};
    float* hits[SLOTS] = {};
    // Pinned staging for callers' pageable buffers (allocated on first use):
    // a chunk of rays and a chunk of hits per slot, and the event that marks
    // the slot's hits as copied back.
    float* stage_rays[SLOTS] = {};
    float* stage_hits[SLOTS] = {};
    cudaEvent_t done[SLOTS] = {};
};

struct LmgpuScene {
    lmgpu::DeviceScene dev{};         // the reference's tree (intersection entry points)
    lmgpu::DeviceScene rdev{};        // what renders traverse: `dev` with the render tree's accelerator
    LmgpuSceneInfo info{};
    std::vector<void*> allocations;   // device buffers owned by the scene
    int device = 0;
    int32_t* d_status = nullptr;      // device error word (0 = ok)
    // Ring of ray counters for the persistent traversal kernels: each launch
    // takes the next slot, so launches in flight on different streams do not
    // share a counter (WORK_SLOTS bounds the launches in flight per scene).
    static constexpr int WORK_SLOTS = 256;
    unsigned long long* d_work = nullptr;
    std::atomic<uint64_t> work_slot{0};
    HostPipeline pipe;
    // Host copies needed by host-side helpers (light selection tables etc.)
    std::vector<float> bounds_min, bounds_max;
};

namespace lmgpu {

void set_error(const std::string& msg);
int fail(int code, const std::string& msg);
int cuda_fail(cudaError_t e, const char* what);

// Device error word values (OR-ed together by kernels).
constexpr int32_t STATUS_STACK_OVERFLOW = 1;
constexpr int32_t STATUS_QUEUE_OVERFLOW = 2;
constexpr int32_t STATUS_TIMEOUT = 4;
constexpr int32_t STATUS_BOUNDS = 8;       // bounds-checked build: an index out of range

// The bounds-checked build (LMGPU_BOUNDS_CHECK=1, liblmgpu_check.so) takes
// the limits its checks compare with from these variables when they are
// set and lower than the real sizes (LMGPU_CHECK_NODE_LIMIT: tree nodes;
// LMGPU_CHECK_QUEUE_LIMIT: wavefront queue slots), so that a test can make
// a check fire while every access stays inside the buffers. Unset: no
// limit (INT64_MAX). The unchecked build never reads them.
int64_t check_limit_from_env(const char* name);

// Path-tracer waves over caller-owned workspace memory (pathtrace.cu).
int64_t workspace_paths_for_bytes(size_t bytes);
int render_device_preallocated(LmgpuScene* sc, const LmgpuRenderParams& p, void* film, cudaStream_t stream,
                               void* ws_mem, size_t ws_bytes, uint32_t* host_counts);

// Reads and clears the device status word; maps it to an LMGPU status.
int consume_status(LmgpuScene* s, cudaStream_t stream);
// The LMGPU status (and message) of a non-zero device status word.
int status_error(int32_t st);

// Sample indices of a render stay below 2^53 (stratified_raster's
// double-precision quotient); offset and count are non-negative.
inline bool sample_range_ok(int64_t offset, int64_t count)
{
    constexpr int64_t LIMIT = int64_t(1) << 53;
    return offset < LIMIT && count <= LIMIT - offset;
}

// The calling thread's current device must be the one the scene was created
// on: the scene's buffers live there, and kernels launched elsewhere would
// read another GPU's memory.
inline int check_scene_device(const LmgpuScene* s)
{
    int cur = 0;
    const cudaError_t e = cudaGetDevice(&cur);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    if (cur != s->device) return fail(LMGPU_ERR_INVALID, "scene used on another device than it was created on");
    return LMGPU_OK;
}

}  // namespace lmgpu

#define LMGPU_CUDA_TRY(expr)                                              \
    do {                                                                  \
        cudaError_t e_ = (expr);                                          \
        if (e_ != cudaSuccess) return lmgpu::cuda_fail(e_, #expr);        \
    } while (0)
