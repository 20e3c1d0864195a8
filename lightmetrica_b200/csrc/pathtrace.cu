// Full hit records (Scene::Intersect) and the wavefront path tracer.
#include <cuda_runtime.h>
#include <cstring>
#include <vector>

#include "../../include/lmgpu.h"
#include "internal.h"
#include "shading.cuh"
#include "trace.cuh"
#include "trace4.cuh"

namespace lmgpu {
namespace {

template <int LAYOUT, bool ANY_HIT, int STACK>
__device__ __forceinline__ bool trace_scene(const DeviceScene& s, TraversalRay& r, Hit& h, int2* stack)
{
    if (s.num_tris == 0) { h.tri = -1; return true; }   // empty scene: no node arrays exist
    if (LAYOUT == LMGPU_LAYOUT_BVH2)
        return trace_bvh2<ANY_HIT>(s.bvh2, s.tris, s.root_ref, s.root_box, r, h, stack, STACK, nullptr);
    if (LAYOUT == LMGPU_LAYOUT_BVH4)
        return trace_bvh4<ANY_HIT>(s.bvh4, s.tris, s.root_ref4, s.root_box, r, h, stack, STACK, nullptr);
    trace_naive<ANY_HIT>(s.tris_by_id, s.num_tris, r, h, nullptr);
    return true;
}

// Scene::Intersect (scene.cpp:67-72): triangles, then the environment's
// emitter shape on a miss. kind: 0 miss, 1 triangle, 2 environment.
template <int LAYOUT, int STACK>
__global__ void __launch_bounds__(128) k_intersect_full(const DeviceScene s, const float* __restrict__ rays, int64_t n,
                                                        int32_t* tri_id, float* t_out, float* geom, int32_t* kind,
                                                        int32_t* status)
{
    int2 stack[STACK];
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* q = rays + 8 * i;
    RayIn in;
    for (int c = 0; c < 3; c++) { in.o[c] = q[c]; in.d[c] = q[3 + c]; }
    in.tmin = q[6]; in.tmax = q[7];
    TraversalRay r;
    setup_ray(r, in);
    Hit h;
    if (!trace_scene<LAYOUT, false, STACK>(s, r, h, stack)) { atomicOr(status, STATUS_STACK_OVERFLOW); h.tri = -1; }
    Geom g;
    int k = 0;
    float t = 0.0f;
    const V3 o = v3(in.o[0], in.o[1], in.o[2]), d = v3(in.d[0], in.d[1], in.d[2]);
    if (h.tri >= 0) {
        k = 1; t = h.t;
        surface_from_hit(s, h.tri, h.u, h.v, o, d, t, g);
    } else if (s.has_env && env_sphere_intersect(s, o, d, in.tmin, in.tmax, t)) {
        k = 2;
        env_surface(s, o, d, t, g);
    }
    tri_id[i] = h.tri;
    t_out[i] = k ? t : 0.0f;
    kind[i] = k;
    float* G = geom + 17 * i;
    if (k) {
        const V3 vs[5] = { g.p, g.gn, g.sn, g.ss, g.st };
        for (int j = 0; j < 5; j++) { G[3 * j] = vs[j].x; G[3 * j + 1] = vs[j].y; G[3 * j + 2] = vs[j].z; }
        G[15] = g.u; G[16] = g.v;
    } else {
        for (int j = 0; j < 17; j++) G[j] = 0.0f;
    }
}

template <int STACK>
void launch_full(const LmgpuScene* sc, const float* rays, int64_t n, int32_t* id, float* t, float* g, int32_t* kind)
{
    const int threads = 128;
    const int64_t blocks = (n + threads - 1) / threads;
    const DeviceScene& s = sc->dev;
    switch (s.layout) {
    case LMGPU_LAYOUT_BVH2: k_intersect_full<LMGPU_LAYOUT_BVH2, STACK><<<blocks, threads>>>(s, rays, n, id, t, g, kind, sc->d_status); break;
    case LMGPU_LAYOUT_BVH4: k_intersect_full<LMGPU_LAYOUT_BVH4, STACK><<<blocks, threads>>>(s, rays, n, id, t, g, kind, sc->d_status); break;
    default: k_intersect_full<LMGPU_LAYOUT_NAIVE, 1><<<blocks, threads>>>(s, rays, n, id, t, g, kind, sc->d_status); break;
    }
}

}  // namespace
}  // namespace lmgpu

using namespace lmgpu;

extern "C" {

int lmgpu_intersect_full_host(LmgpuScene* scene, const float* rays_aos, int64_t n, int32_t* tri_id, float* t,
                              float* geom, int32_t* kind)
{
    if (!scene || n < 0 || (n > 0 && (!rays_aos || !tri_id || !t || !geom || !kind)))
        return fail(LMGPU_ERR_INVALID, "null argument or negative count");
    if (n == 0) return LMGPU_OK;
    const size_t N = static_cast<size_t>(n);
    char* buf = nullptr;
    const size_t bytes = N * (8 + 1 + 1 + 17 + 1) * sizeof(float);
    LMGPU_CUDA_TRY(cudaMalloc(&buf, bytes));
    float* dr = reinterpret_cast<float*>(buf);
    int32_t* did = reinterpret_cast<int32_t*>(dr + 8 * N);
    float* dt = dr + 9 * N;
    float* dg = dr + 10 * N;
    int32_t* dk = reinterpret_cast<int32_t*>(dr + 27 * N);
    int rc = LMGPU_OK;
    cudaError_t e = cudaMemcpy(dr, rays_aos, 8 * N * sizeof(float), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) rc = cuda_fail(e, "cudaMemcpy(rays)");
    if (rc == LMGPU_OK) {
        const int cap = scene->dev.stack_cap;
        if (cap <= 32) launch_full<32>(scene, dr, n, did, dt, dg, dk);
        else if (cap <= 64) launch_full<64>(scene, dr, n, did, dt, dg, dk);
        else if (cap <= 128) launch_full<128>(scene, dr, n, did, dt, dg, dk);
        else if (cap <= 256) launch_full<256>(scene, dr, n, did, dt, dg, dk);
        else rc = fail(LMGPU_ERR_UNSUPPORTED, "BVH deeper than the largest compiled traversal stack (256)");
        if (rc == LMGPU_OK && (e = cudaGetLastError()) != cudaSuccess) rc = cuda_fail(e, "k_intersect_full");
        if (rc == LMGPU_OK) rc = consume_status(scene, nullptr);
    }
    if (rc == LMGPU_OK) {
        if ((e = cudaMemcpy(tri_id, did, N * sizeof(int32_t), cudaMemcpyDeviceToHost)) != cudaSuccess ||
            (e = cudaMemcpy(t, dt, N * sizeof(float), cudaMemcpyDeviceToHost)) != cudaSuccess ||
            (e = cudaMemcpy(geom, dg, 17 * N * sizeof(float), cudaMemcpyDeviceToHost)) != cudaSuccess ||
            (e = cudaMemcpy(kind, dk, N * sizeof(int32_t), cudaMemcpyDeviceToHost)) != cudaSuccess)
            rc = cuda_fail(e, "cudaMemcpy(full hits)");
    }
    cudaFree(buf);
    return rc;
}

int lmgpu_render_device(LmgpuScene* scene, const LmgpuRenderParams* params, void* film_device, void* stream,
                        LmgpuRenderStats* stats)
{
    (void)scene; (void)params; (void)film_device; (void)stream; (void)stats;
    return fail(LMGPU_ERR_UNSUPPORTED, "render not built yet");
}

int lmgpu_render(LmgpuScene* scene, const LmgpuRenderParams* params, float* film_host, LmgpuRenderStats* stats)
{
    (void)scene; (void)params; (void)film_host; (void)stats;
    return fail(LMGPU_ERR_UNSUPPORTED, "render not built yet");
}

}  // extern "C"
