// Full hit records (Scene::Intersect) and the one-scene wavefront path
// tracer's driver (the kernels are in pt_kernels.cuh).
//
// Path state lives in HBM as structure-of-arrays (float4 records, 16-byte
// coalesced accesses); surviving paths and shadow rays are appended to
// compacted queues with one warp-aggregated atomic per warp (ballot/popc).
// The driver reads the queue counts back after each pass to size the next
// launch; the multi-scene batch (batch.cu) keeps them on the device instead.
#include <cuda_runtime.h>
#include <algorithm>
#include <cstring>
#include <memory>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "../../include/lmgpu.h"
#include "internal.h"
#include "pathtrace.cuh"
#include "pt_kernels.cuh"
#include "rng.cuh"
#include "shading.cuh"
#include "trace.cuh"
#include "trace4.cuh"
#include "trace_kernels.cuh"

namespace lmgpu {
namespace {

// ------------------------------------------------------ full hit record ----

template <int LAYOUT, bool ANY_HIT, int STACK>
__device__ __forceinline__ bool trace_scene(const DeviceScene& s, TraversalRay& r, Hit& h, int2* stack)
{
    if (s.num_tris == 0) { h.tri = -1; return true; }   // empty scene: no node arrays exist
    if (LAYOUT == LMGPU_LAYOUT_BVH2)
        return trace_bvh2<ANY_HIT>(s.bvh2, s.tris, s.root_ref, s.root_box, r, h, stack, s.stack_cap < STACK ? s.stack_cap : STACK, nullptr);
    if (LAYOUT == LMGPU_LAYOUT_BVH4)
        return trace_bvh4<ANY_HIT>(s.bvh4, s.tris, s.root_ref4, s.root_box, r, h, stack, s.stack_cap < STACK ? s.stack_cap : STACK, nullptr);
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

// ------------------------------------------------------------ driver ------

// Wave workspace (scratch), one per device, grown on demand.
// Default paths per wave (128M: 29 GB of path state; a render allocates
// for min(wave, its samples)). Each bounce launch ends with a
// latency-bound tail of the wave's longest rays, so fewer, larger waves
// keep the GPU busier: on the 1080p terrain (64 spp, one 128M-path wave),
// waves of 32M, 64M and 128M paths took 208.6, 196.8 and 189.5 ms a frame.
constexpr int64_t DEFAULT_WAVE_PATHS = int64_t(1) << 27;
constexpr int64_t MIN_DEFAULT_WAVE_PATHS = int64_t(1) << 20;

struct Workspace {
    int64_t capacity = 0;
    void* mem = nullptr;
    uint32_t* host_counts = nullptr;   // pinned
    PathState st{};
};

// Path state bytes per path (two queues of 64-byte ray records, hits,
// radiance, shadow rays, raster) and the fixed header of counters.
constexpr size_t WS_BYTES_PER_PATH = 16 * 13 + 8;
constexpr size_t WS_HEADER_BYTES = 256;

// Lays the path state of P paths out from `p` (WS_HEADER_BYTES +
// P * WS_BYTES_PER_PATH bytes, 256-byte aligned).
void carve_state(PathState& st, char* p, size_t P)
{
    auto take = [&](size_t b) { char* r = p; p += b; return r; };
    st.counters = reinterpret_cast<uint32_t*>(take(WS_HEADER_BYTES));
    for (int q = 0; q < 2; q++) {
        st.qo[q] = reinterpret_cast<float4*>(take(16 * P));
        st.qd[q] = reinterpret_cast<float4*>(take(16 * P));
        st.qt[q] = reinterpret_cast<float4*>(take(16 * P));
        st.qn[q] = reinterpret_cast<float4*>(take(16 * P));
    }
    st.hit = reinterpret_cast<float4*>(take(16 * P));
    st.L = reinterpret_cast<float4*>(take(16 * P));
    st.sh_o = reinterpret_cast<float4*>(take(16 * P));
    st.sh_d = reinterpret_cast<float4*>(take(16 * P));
    st.sh_c = reinterpret_cast<float4*>(take(16 * P));
    st.raster = reinterpret_cast<float2*>(take(8 * P));
    for (uint32_t& c : st.cap) c = (uint32_t)P;
}

int ensure_workspace(Workspace& ws, int64_t paths)
{
    if (!ws.host_counts) LMGPU_CUDA_TRY(cudaMallocHost(&ws.host_counts, 16));
    if (ws.capacity >= paths && ws.mem) return LMGPU_OK;
    if (ws.mem) { cudaFree(ws.mem); ws.mem = nullptr; ws.capacity = 0; }
    const size_t P = (size_t)paths;
    cudaError_t e = cudaMalloc(&ws.mem, WS_HEADER_BYTES + P * WS_BYTES_PER_PATH);
    if (e != cudaSuccess) return e == cudaErrorMemoryAllocation ? fail(LMGPU_ERR_OOM, "render workspace allocation failed")
                                                                 : cuda_fail(e, "cudaMalloc(workspace)");
    carve_state(ws.st, static_cast<char*>(ws.mem), P);
    ws.capacity = paths;
    return LMGPU_OK;
}

template <class F>
int shadow_pass(LmgpuScene* sc, const PathState& st, const OneScene<F>& ctx, int64_t max_rays, cudaStream_t stream)
{
    ShadowIO<OneScene<F>> io{ st.counters + 2, st.sh_o, st.sh_d, st.sh_c, st.L, ctx };
    return launch_trace<true, ShadowIO<OneScene<F>>>(sc, io, max_rays, stream, nullptr, true);
}

int read_counts(Workspace& ws, cudaStream_t stream)
{
    LMGPU_CUDA_TRY(cudaMemcpyAsync(ws.host_counts, ws.st.counters, 16, cudaMemcpyDeviceToHost, stream));
    LMGPU_CUDA_TRY(cudaStreamSynchronize(stream));
    return LMGPU_OK;
}

template <int TECH, class F>
int render_waves(LmgpuScene* sc, const LmgpuRenderParams& p, F* film, cudaStream_t stream, LmgpuRenderStats& stats,
                 Workspace& ws)
{
    const DeviceScene& s = sc->rdev;
    const int64_t pixels = (int64_t)s.cam.width * s.cam.height;
    int64_t P = p.wave_paths > 0 ? p.wave_paths : DEFAULT_WAVE_PATHS;
    P = std::min<int64_t>(P, p.num_samples);
    int rc = ensure_workspace(ws, P);
    // Without an explicit wave size, a device short of memory gets smaller waves.
    while (rc == LMGPU_ERR_OOM && p.wave_paths == 0 && P > MIN_DEFAULT_WAVE_PATHS) {
        P /= 2;
        rc = ensure_workspace(ws, P);
    }
    if (rc != LMGPU_OK) return rc;
    PathState st = ws.st;
    st.status = sc->d_status;
#if LMGPU_BOUNDS_CHECK
    const int64_t qlim = check_limit_from_env("LMGPU_CHECK_QUEUE_LIMIT");
    for (uint32_t& q : st.cap) q = (uint32_t)std::min<int64_t>(q, qlim);
#endif
    RenderConsts c;
    c.technique = TECH;
    c.rr_depth = p.rr_depth;
    c.max_pv = p.max_path_vertices;
    c.sampling = p.sampling;
    c.seed = p.seed;
    c.pixels = pixels;
    c.inv_pixels = 1.0 / double(pixels);
    const int shade_blocks = 148 * 8;
    for (int64_t base = 0; base < p.num_samples && rc == LMGPU_OK; base += P) {
        const int64_t cnt = std::min<int64_t>(P, p.num_samples - base);
        c.sample_base = p.sample_offset + base;
        const OneScene<F> ctx{ s, c, film };
        stats.waves++;
        stats.paths += cnt;
        if (c.max_pv != -1 && c.max_pv <= 1) continue;   // no path vertex beyond the camera
        LMGPU_CUDA_TRY(cudaMemsetAsync(st.counters, 0, 16, stream));
        k_pt_init<TECH, OneScene<F>><<<(unsigned)((cnt + 127) / 128), 128, 0, stream>>>(ctx, st, cnt, 0);
        LMGPU_CUDA_TRY(cudaGetLastError());
        if (TECH != LMGPU_RENDER_PT) {
            if ((rc = read_counts(ws, stream)) != LMGPU_OK) break;
            stats.shadow_rays += ws.host_counts[2];
            if (ws.host_counts[2]) rc = shadow_pass(sc, st, ctx, ws.host_counts[2], stream);
        }
        int qin = 0;
        for (int k = 1; rc == LMGPU_OK; k++) {
            if (c.max_pv != -1 && k >= c.max_pv) break;
            if ((rc = read_counts(ws, stream)) != LMGPU_OK) break;
            const uint32_t n = ws.host_counts[qin];
            if (n == 0) break;
            stats.rays_traced += n;
            stats.max_bounces_run = std::max(stats.max_bounces_run, k);
            PathRayIO<false> io{ st.counters + qin, st.qo[qin], st.qd[qin], st.hit, nullptr };
            rc = launch_trace<false, PathRayIO<false>>(sc, io, n, stream, nullptr, true);
            if (rc != LMGPU_OK) break;
            LMGPU_CUDA_TRY(cudaMemsetAsync(st.counters + (1 - qin), 0, 4, stream));
            LMGPU_CUDA_TRY(cudaMemsetAsync(st.counters + 2, 0, 4, stream));
            const unsigned blocks = (unsigned)std::min<int64_t>((n + 127) / 128, shade_blocks);
            k_pt_shade<TECH, OneScene<F>><<<blocks, 128, 0, stream>>>(ctx, st, k, qin, 1 - qin);
            LMGPU_CUDA_TRY(cudaGetLastError());
            if (TECH != LMGPU_RENDER_PT) {
                if ((rc = read_counts(ws, stream)) != LMGPU_OK) break;
                stats.shadow_rays += ws.host_counts[2];
                if (ws.host_counts[2]) rc = shadow_pass(sc, st, ctx, ws.host_counts[2], stream);
            }
            qin = 1 - qin;
        }
        if (rc == LMGPU_OK) {
            k_pt_splat<OneScene<F>><<<(unsigned)((cnt + 127) / 128), 128, 0, stream>>>(ctx, st, cnt);
            LMGPU_CUDA_TRY(cudaGetLastError());
        }
    }
    stats.rays_traced += stats.shadow_rays;
    return rc;
}

template <class F>
int render_dispatch(LmgpuScene* sc, const LmgpuRenderParams& p, F* film, cudaStream_t stream, LmgpuRenderStats& stats,
                    Workspace& ws)
{
    switch (p.technique) {
    case LMGPU_RENDER_PT: return render_waves<LMGPU_RENDER_PT, F>(sc, p, film, stream, stats, ws);
    case LMGPU_RENDER_PT_DIRECT: return render_waves<LMGPU_RENDER_PT_DIRECT, F>(sc, p, film, stream, stats, ws);
    case LMGPU_RENDER_PT_MIS: return render_waves<LMGPU_RENDER_PT_MIS, F>(sc, p, film, stream, stats, ws);
    default: return fail(LMGPU_ERR_INVALID, "unknown technique");
    }
}

int check_params(LmgpuScene* sc, const LmgpuRenderParams* p)
{
    if (!sc || !p) return fail(LMGPU_ERR_INVALID, "null argument");
    if (const int rc = check_scene_device(sc)) return rc;
    if (!sc->dev.cam.valid) return fail(LMGPU_ERR_INVALID, "scene has no camera");
    if (p->num_samples <= 0) return fail(LMGPU_ERR_INVALID, "num_samples must be positive");
    if (p->sample_offset < 0) return fail(LMGPU_ERR_INVALID, "negative sample offset");
    if (!sample_range_ok(p->sample_offset, p->num_samples)) return fail(LMGPU_ERR_INVALID, "sample indices reach 2^53");
    if (p->technique < LMGPU_RENDER_PT || p->technique > LMGPU_RENDER_PT_MIS) return fail(LMGPU_ERR_INVALID, "unknown technique");
    if (p->sampling != LMGPU_SAMPLING_STRATIFIED && p->sampling != LMGPU_SAMPLING_UNIFORM) return fail(LMGPU_ERR_INVALID, "unknown sampling");
    if (p->wave_paths < 0) return fail(LMGPU_ERR_INVALID, "negative wave size");
    return LMGPU_OK;
}

// One wave workspace per device, shared by every scene rendered there: a
// render holds its device's lock from its first launch until its device
// work has completed, so renders from several threads take turns. The
// workspace grows to the largest wave asked for and is kept until exit.
struct DeviceWorkspace {
    std::mutex mu;
    Workspace ws;
};

DeviceWorkspace& device_workspace(int device)
{
    static std::mutex map_mu;
    static std::unordered_map<int, std::unique_ptr<DeviceWorkspace>> all;
    std::lock_guard<std::mutex> lock(map_mu);
    auto& e = all[device];
    if (!e) e.reset(new DeviceWorkspace);
    return *e;
}

template <class F>
__global__ void k_rescale(const F* film, float* out, int64_t n, double scale)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = (float)((double)film[i] * scale);
}

// lmgpu_render's film buffers, one set per device, kept between calls: the
// device film, its rescaled float copy and a pinned host copy. The result
// reaches the caller's (pageable) buffer through the pinned copy and a host
// memcpy: a device-to-host copy straight into freshly allocated pageable
// memory (a new numpy array, say) took 0.7-1.1 s for a 25 MB film in the
// driver, against ~5 ms this way.
struct HostFilmBuffers {
    std::mutex mu;
    void* film = nullptr;
    size_t film_bytes = 0;
    float* out = nullptr;
    float* pinned = nullptr;
    size_t out_bytes = 0;
};

HostFilmBuffers& host_film_buffers(int device)
{
    static std::mutex map_mu;
    static std::unordered_map<int, std::unique_ptr<HostFilmBuffers>> all;
    std::lock_guard<std::mutex> lock(map_mu);
    auto& e = all[device];
    if (!e) e.reset(new HostFilmBuffers);
    return *e;
}

// Grows the buffers to hold `film_bytes` (device film) and `out_bytes`
// (float copies); called with hb.mu held.
int ensure_host_film(HostFilmBuffers& hb, size_t film_bytes, size_t out_bytes)
{
    if (hb.film_bytes < film_bytes) {
        cudaFree(hb.film);
        hb.film = nullptr;
        hb.film_bytes = 0;
        cudaError_t e = cudaMalloc(&hb.film, film_bytes);
        if (e != cudaSuccess) { hb.film = nullptr; return cuda_fail(e, "cudaMalloc(film)"); }
        hb.film_bytes = film_bytes;
    }
    if (hb.out_bytes < out_bytes) {
        cudaFree(hb.out);
        cudaFreeHost(hb.pinned);
        hb.out = nullptr;
        hb.pinned = nullptr;
        hb.out_bytes = 0;
        cudaError_t e = cudaMalloc(&hb.out, out_bytes);
        if (e == cudaSuccess) e = cudaMallocHost(&hb.pinned, out_bytes);
        if (e != cudaSuccess) {
            cudaFree(hb.out);
            hb.out = nullptr;
            hb.pinned = nullptr;
            return cuda_fail(e, "film buffers");
        }
        hb.out_bytes = out_bytes;
    }
    return LMGPU_OK;
}

// Points a Workspace at caller-owned memory (same layout as
// ensure_workspace, no allocation); host_counts is the caller's readback
// buffer for the queue counters.
void carve_workspace(Workspace& ws, void* mem, int64_t paths, uint32_t* host_counts)
{
    carve_state(ws.st, static_cast<char*>(mem), (size_t)paths);
    ws.mem = mem;
    ws.capacity = paths;
    ws.host_counts = host_counts;
}

}  // namespace

int64_t workspace_paths_for_bytes(size_t bytes)
{
    return bytes <= WS_HEADER_BYTES ? 0 : (int64_t)((bytes - WS_HEADER_BYTES) / WS_BYTES_PER_PATH);
}

// Renders like lmgpu_render_device over a caller-owned wave workspace of
// `ws_bytes` at `ws_mem` (device) and a host readback buffer of 4 counters:
// waves never exceed the workspace's capacity, and nothing is allocated.
int render_device_preallocated(LmgpuScene* sc, const LmgpuRenderParams& p, void* film, cudaStream_t stream,
                               void* ws_mem, size_t ws_bytes, uint32_t* host_counts)
{
    // The same checks as the allocating entry points, without creating the
    // scene's cached workspace.
    if (!sc) return fail(LMGPU_ERR_INVALID, "null scene");
    if (const int rc = check_scene_device(sc)) return rc;
    if (!film) return fail(LMGPU_ERR_INVALID, "null film");
    if (!sc->dev.cam.valid) return fail(LMGPU_ERR_INVALID, "scene has no camera");
    if (p.num_samples <= 0) return fail(LMGPU_ERR_INVALID, "num_samples must be positive");
    if (p.sample_offset < 0) return fail(LMGPU_ERR_INVALID, "negative sample offset");
    if (!sample_range_ok(p.sample_offset, p.num_samples)) return fail(LMGPU_ERR_INVALID, "sample indices reach 2^53");
    if (p.technique < LMGPU_RENDER_PT || p.technique > LMGPU_RENDER_PT_MIS) return fail(LMGPU_ERR_INVALID, "unknown technique");
    if (p.sampling != LMGPU_SAMPLING_STRATIFIED && p.sampling != LMGPU_SAMPLING_UNIFORM) return fail(LMGPU_ERR_INVALID, "unknown sampling");
    if (p.wave_paths < 0) return fail(LMGPU_ERR_INVALID, "negative wave size");
    int rc = LMGPU_OK;
    const int64_t cap = workspace_paths_for_bytes(ws_bytes);
    if (cap <= 0) return fail(LMGPU_ERR_INVALID, "workspace too small");
    LmgpuRenderParams q = p;
    q.wave_paths = (int32_t)std::min<int64_t>(p.wave_paths > 0 ? p.wave_paths : cap, cap);
    Workspace ws;
    carve_workspace(ws, ws_mem, cap, host_counts);
    LmgpuRenderStats stats;
    std::memset(&stats, 0, sizeof(stats));
    switch (q.technique) {
    case LMGPU_RENDER_PT:
        rc = q.film_fp64 ? render_waves<LMGPU_RENDER_PT, double>(sc, q, static_cast<double*>(film), stream, stats, ws)
                         : render_waves<LMGPU_RENDER_PT, float>(sc, q, static_cast<float*>(film), stream, stats, ws);
        break;
    case LMGPU_RENDER_PT_DIRECT:
        rc = q.film_fp64 ? render_waves<LMGPU_RENDER_PT_DIRECT, double>(sc, q, static_cast<double*>(film), stream, stats, ws)
                         : render_waves<LMGPU_RENDER_PT_DIRECT, float>(sc, q, static_cast<float*>(film), stream, stats, ws);
        break;
    default:
        rc = q.film_fp64 ? render_waves<LMGPU_RENDER_PT_MIS, double>(sc, q, static_cast<double*>(film), stream, stats, ws)
                         : render_waves<LMGPU_RENDER_PT_MIS, float>(sc, q, static_cast<float*>(film), stream, stats, ws);
        break;
    }
    if (rc == LMGPU_OK) rc = consume_status(sc, stream);
    return rc;
}


}  // namespace lmgpu

using namespace lmgpu;

extern "C" {

int lmgpu_intersect_full_host(LmgpuScene* scene, const float* rays_aos, int64_t n, int32_t* tri_id, float* t,
                              float* geom, int32_t* kind)
{
    if (!scene || n < 0 || (n > 0 && (!rays_aos || !tri_id || !t || !geom || !kind)))
        return fail(LMGPU_ERR_INVALID, "null argument or negative count");
    if (const int rc = check_scene_device(scene)) return rc;
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
    int rc = check_params(scene, params);
    if (rc != LMGPU_OK) return rc;
    if (!film_device) return fail(LMGPU_ERR_INVALID, "null film");
    LmgpuRenderStats st;
    std::memset(&st, 0, sizeof(st));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    DeviceWorkspace& dw = device_workspace(scene->device);
    std::lock_guard<std::mutex> lock(dw.mu);     // held until the render's device work is done
    cudaEvent_t e0, e1;
    LMGPU_CUDA_TRY(cudaEventCreate(&e0));
    LMGPU_CUDA_TRY(cudaEventCreate(&e1));
    LMGPU_CUDA_TRY(cudaEventRecord(e0, s));
    if (params->film_fp64) rc = render_dispatch(scene, *params, static_cast<double*>(film_device), s, st, dw.ws);
    else rc = render_dispatch(scene, *params, static_cast<float*>(film_device), s, st, dw.ws);
    if (rc == LMGPU_OK) {
        cudaError_t e = cudaEventRecord(e1, s);
        if (e == cudaSuccess) e = cudaEventSynchronize(e1);
        if (e != cudaSuccess) rc = cuda_fail(e, "render completion");
        float ms = 0.0f;
        if (rc == LMGPU_OK) cudaEventElapsedTime(&ms, e0, e1);
        st.device_ms = ms;
        if (rc == LMGPU_OK) rc = consume_status(scene, s);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (stats) *stats = st;
    return rc;
}

int lmgpu_render(LmgpuScene* scene, const LmgpuRenderParams* params, float* film_host, LmgpuRenderStats* stats)
{
    int rc = check_params(scene, params);
    if (rc != LMGPU_OK) return rc;
    if (!film_host) return fail(LMGPU_ERR_INVALID, "null film");
    const int64_t n = 3 * (int64_t)scene->dev.cam.width * scene->dev.cam.height;
    const size_t esize = params->film_fp64 ? sizeof(double) : sizeof(float);
    HostFilmBuffers& hb = host_film_buffers(scene->device);
    std::lock_guard<std::mutex> lock(hb.mu);
    if ((rc = ensure_host_film(hb, n * esize, n * sizeof(float))) != LMGPU_OK) return rc;
    LMGPU_CUDA_TRY(cudaMemsetAsync(hb.film, 0, n * esize, nullptr));
    if ((rc = lmgpu_render_device(scene, params, hb.film, nullptr, stats)) != LMGPU_OK) return rc;
    // Rescale(W * H / num_samples) (sched.mt.cpp:250-256, hdrfilm.cpp:334-341).
    const double scale = double(scene->dev.cam.width) * scene->dev.cam.height / double(params->num_samples);
    const unsigned blocks = (unsigned)((n + 255) / 256);
    if (params->film_fp64) k_rescale<double><<<blocks, 256>>>(static_cast<const double*>(hb.film), hb.out, n, scale);
    else k_rescale<float><<<blocks, 256>>>(static_cast<const float*>(hb.film), hb.out, n, scale);
    LMGPU_CUDA_TRY(cudaGetLastError());
    LMGPU_CUDA_TRY(cudaMemcpyAsync(hb.pinned, hb.out, n * sizeof(float), cudaMemcpyDeviceToHost, nullptr));
    LMGPU_CUDA_TRY(cudaStreamSynchronize(nullptr));
    std::memcpy(film_host, hb.pinned, n * sizeof(float));
    return LMGPU_OK;
}

int lmgpu_render_release(void)
{
    int dev = 0;
    LMGPU_CUDA_TRY(cudaGetDevice(&dev));
    // Every field is reset whatever its free returns, so no later render
    // reuses (or frees again) memory that this call handed back; the first
    // failure is reported once all of them are reset.
    cudaError_t first = cudaSuccess;
    const char* what = nullptr;
    auto note = [&](cudaError_t e, const char* w) {
        if (e != cudaSuccess && first == cudaSuccess) { first = e; what = w; }
    };
    {
        // Takes the lock a render holds until its device work is done.
        DeviceWorkspace& dw = device_workspace(dev);
        std::lock_guard<std::mutex> lock(dw.mu);
        if (dw.ws.mem) note(cudaFree(dw.ws.mem), "cudaFree(workspace)");
        dw.ws.mem = nullptr;
        dw.ws.capacity = 0;
    }
    HostFilmBuffers& hb = host_film_buffers(dev);
    std::lock_guard<std::mutex> lock(hb.mu);
    if (hb.film) note(cudaFree(hb.film), "cudaFree(film)");
    if (hb.out) note(cudaFree(hb.out), "cudaFree(rescaled film)");
    if (hb.pinned) note(cudaFreeHost(hb.pinned), "cudaFreeHost(film copy)");
    hb.film = nullptr;
    hb.out = nullptr;
    hb.pinned = nullptr;
    hb.film_bytes = hb.out_bytes = 0;
    if (first != cudaSuccess) return cuda_fail(first, what);
    return LMGPU_OK;
}

}  // extern "C"
