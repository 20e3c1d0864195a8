// Full hit records (Scene::Intersect) and the wavefront path tracer.
//
// Path tracing follows the reference renderers' per-sample loops
//   pt         pathtrace.cpp:165-266
//   pt.direct  pathtrace.direct.cpp:170-338
//   pt.mis     pathtrace.mis.cpp:167-369
// restructured into waves of paths that advance one bounce per kernel
// sequence: trace (closest hit) -> shade (emission, next-event estimation,
// Russian roulette, BSDF sampling) -> shadow (any hit) -> ... -> splat.
// Path state lives in HBM as structure-of-arrays (float4 records, 16-byte
// coalesced accesses); surviving paths and shadow rays are appended to
// compacted queues with one warp-aggregated atomic per warp (ballot/popc).
#include <cuda_runtime.h>
#include <algorithm>
#include <cstring>
#include <vector>

#include "../../include/lmgpu.h"
#include "internal.h"
#include "pathtrace.cuh"
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

// --------------------------------------------------------- path state ------

constexpr uint32_t PREV_DEGENERATED = 1u;   // previous vertex is the pinhole
constexpr uint32_t PREV_SPECULAR = 2u;      // last BSDF sample was specular

// Device pointers of one wave's path state (capacity paths).
struct PathState {
    float4* ray_o;     // o.xyz, minT
    float4* ray_d;     // d.xyz
    float4* hit;       // tri (int bits), t, u, v
    float4* thr;       // throughput
    float4* L;         // radiance to splat at the path's raster position
    float2* raster;
    float4* prev_p;    // previous vertex position, BSDF pdf (projected solid angle)
    float4* prev_n;    // previous vertex shading normal, flags (uint bits)
    int32_t* queue[2];
    float4* sh_o;      // shadow ray origin, maxT
    float4* sh_d;      // direction, target (int bits: path index, or ~pixel)
    float4* sh_c;      // contribution
    uint32_t* counters;   // [0], [1] ray queues; [2] shadow queue
};

struct RenderConsts {
    int32_t technique;
    int32_t rr_depth;
    int32_t max_pv;
    int32_t sampling;
    uint64_t seed;
    int64_t sample_base;   // sample index of the wave's path 0
    int64_t pixels;
};

// Warp-aggregated append: returns this lane's slot in the queue (the whole
// warp must reach the call).
__device__ __forceinline__ uint32_t queue_append(uint32_t* counter, bool want)
{
    const unsigned active = __activemask();
    const unsigned mask = __ballot_sync(active, want);
    if (!want) return 0xffffffffu;
    const unsigned lane = threadIdx.x & 31u;
    const int leader = __ffs(mask) - 1;
    uint32_t base = 0;
    if ((int)lane == leader) base = atomicAdd(counter, (uint32_t)__popc(mask));
    base = __shfl_sync(mask, base, leader);
    return base + __popc(mask & ((1u << lane) - 1u));
}

__device__ __forceinline__ V3 f3(float4 q) { return v3(q.x, q.y, q.z); }
__device__ __forceinline__ float4 f4(V3 v, float w) { return make_float4(v.x, v.y, v.z, w); }

template <class F>
__device__ __forceinline__ void film_add(F* film, int pixel, V3 c)
{
    if (pixel < 0 || (c.x == 0.0f && c.y == 0.0f && c.z == 0.0f)) return;
    atomicAdd(film + 3 * pixel, (F)c.x);
    atomicAdd(film + 3 * pixel + 1, (F)c.y);
    atomicAdd(film + 3 * pixel + 2, (F)c.z);
}

// RenderUtils::Visible (renderutils.cpp:58-70) as a queued shadow ray:
// minT = Eps, maxT = |target - p| (1 - Eps).
__device__ __forceinline__ void write_shadow(const PathState& st, uint32_t slot, V3 p, V3 target, V3 c, int32_t dest)
{
    const V3 d = target - p;
    const float len = sqrtf(length2(d));
    st.sh_o[slot] = f4(p, len * (1.0f - EPS_F));
    st.sh_d[slot] = f4(d / len, __int_as_float(dest));
    st.sh_c[slot] = f4(c, 0.0f);
}

// Camera vertex of pt.direct / pt.mis (numPathVertices == 1): a light sample
// seen through the pinhole, splatted at its own raster position
// (pathtrace.direct.cpp:206-250, pathtrace.mis.cpp:188-247).
template <int TECH>
__device__ __forceinline__ bool camera_nee(const DeviceScene& s, uint64_t key, V3& target, V3& c, int32_t& dest)
{
    LightPoint lp;
    if (!sample_light(s, rng_uniform(key, dim_vertex(1) + DIM_LIGHT), rng_uniform(key, dim_vertex(1) + DIM_LIGHT + 1), lp))
        return false;
    const V3 cp = load3(s.cam.position);
    const V3 ppL = normalize(lp.p - cp);
    float rx, ry, We;
    if (!camera_project(s.cam, cp, ppL, rx, ry, We) || We == 0.0f) return false;
    const float G = geometry_term(cp, v3(0, 0, 1), true, lp.p, lp.n, false);
    if (G == 0.0f) return false;
    const V3 Le = emitted(lp.Le, lp.n, -ppL);
    float w = 1.0f;
    if (TECH == LMGPU_RENDER_PT_MIS) {
        const float pdf_dl = lp.pdf_area / G;
        w = pdf_dl / (pdf_dl + We);   // the pinhole's pdf is its importance (proj. solid angle)
    }
    c = Le * (w * We * G / lp.pdf_area);
    target = lp.p;
    dest = ~film_pixel(s.cam, rx, ry);
    return !is_zero(c) && dest != ~(-1);
}

// Wave initialisation: raster sample and camera ray; for pt.direct / pt.mis
// the whole camera vertex (light sample, Russian roulette).
template <int TECH>
__global__ void __launch_bounds__(128) k_pt_init(const DeviceScene s, const RenderConsts rc, const PathState st,
                                                 int64_t count)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const uint64_t sample = (uint64_t)(rc.sample_base + i);
    const uint64_t key = sample_key(rc.seed, sample);
    const float u0 = rng_uniform(key, DIM_RASTER), u1 = rng_uniform(key, DIM_RASTER + 1);
    float rx, ry;
    if (rc.sampling == LMGPU_SAMPLING_STRATIFIED) {
        const int64_t pix = (int64_t)(sample % (uint64_t)rc.pixels);
        rx = (float(pix % s.cam.width) + u0) / float(s.cam.width);
        ry = (float(pix / s.cam.width) + u1) / float(s.cam.height);
    } else {
        rx = u0; ry = u1;
    }
    float pdf_cam;
    const V3 dir = camera_direction(s.cam, rx, ry, pdf_cam);
    const V3 cp = load3(s.cam.position);
    st.raster[i] = make_float2(rx, ry);
    st.L[i] = make_float4(0, 0, 0, 0);
    V3 thr = v3(1, 1, 1);
    bool alive = true;
    if (TECH != LMGPU_RENDER_PT) {
        V3 target, c;
        int32_t dest;
        const bool shadow = camera_nee<TECH>(s, key, target, c, dest);
        const uint32_t sslot = queue_append(&st.counters[2], shadow);
        if (shadow) write_shadow(st, sslot, cp, target, c, dest);
        if (rc.rr_depth != -1 && 1 >= rc.rr_depth) {
            const float p = fminf(0.5f, luminance(thr));
            if (rng_uniform(key, dim_vertex(1) + DIM_RR) > p) alive = false;
            else thr = thr / p;
        }
        st.prev_p[i] = f4(cp, pdf_cam);
        st.prev_n[i] = make_float4(0, 0, 1, __uint_as_float(PREV_DEGENERATED));
    }
    st.thr[i] = f4(thr, 0.0f);
    const uint32_t slot = queue_append(&st.counters[0], alive);
    if (alive) {
        st.ray_o[i] = f4(cp, TECH == LMGPU_RENDER_PT ? 0.0f : EPS_F);
        st.ray_d[i] = f4(dir, 0.0f);
        st.queue[0][slot] = (int32_t)i;
    }
}

// Closest-hit traversal of the queued rays (writes hit records).
struct PathRayIO {
    const int32_t* queue;
    const uint32_t* count_ptr;
    const float4* ray_o;
    const float4* ray_d;
    float4* hit;
    __device__ int64_t count() const { return (int64_t)*count_ptr; }
    __device__ RayIn load(int64_t j) const
    {
        const int32_t i = queue[j];
        const float4 o = ray_o[i], d = ray_d[i];
        RayIn r;
        r.o[0] = o.x; r.o[1] = o.y; r.o[2] = o.z;
        r.d[0] = d.x; r.d[1] = d.y; r.d[2] = d.z;
        r.tmin = o.w; r.tmax = FLT_MAX;
        return r;
    }
    __device__ void store(int64_t j, const Hit& h, const TraversalRay&) const
    {
        hit[queue[j]] = make_float4(__int_as_float(h.tri), h.t, h.u, h.v);
    }
};

// Shadow rays: visible iff neither a triangle nor the environment's emitter
// shape is hit within [Eps, maxT] (Scene::Intersect inside Visible); visible
// contributions go to the path's radiance or straight to the film.
template <class F>
struct ShadowIO {
    const uint32_t* count_ptr;
    const float4* sh_o;
    const float4* sh_d;
    const float4* sh_c;
    float4* L;
    F* film;
    DeviceScene s;
    __device__ int64_t count() const { return (int64_t)*count_ptr; }
    __device__ RayIn load(int64_t j) const
    {
        const float4 o = sh_o[j], d = sh_d[j];
        RayIn r;
        r.o[0] = o.x; r.o[1] = o.y; r.o[2] = o.z;
        r.d[0] = d.x; r.d[1] = d.y; r.d[2] = d.z;
        r.tmin = EPS_F; r.tmax = o.w;
        return r;
    }
    __device__ void store(int64_t j, const Hit& h, const TraversalRay& r) const
    {
        if (h.tri >= 0) return;
        const V3 o = v3(r.o[0], r.o[1], r.o[2]), d = v3(r.d[0], r.d[1], r.d[2]);
        float te;
        if (s.has_env && env_sphere_intersect(s, o, d, r.tmin, sh_o[j].w, te)) return;
        const V3 c = f3(sh_c[j]);
        const int32_t dest = __float_as_int(sh_d[j].w);
        if (dest >= 0) {
            const float4 l = L[dest];
            L[dest] = make_float4(l.x + c.x, l.y + c.y, l.z + c.z, 0.0f);
        } else {
            film_add(film, ~dest, c);
        }
    }
};

// Shading of the hits of iteration k: emission at the hit (vertex k + 1),
// then for pt.direct / pt.mis next-event estimation at it, Russian roulette
// and BSDF sampling; pt samples the BSDF first and applies Russian roulette
// with numPathVertices = k (pathtrace.cpp:223-260).
template <int TECH>
__global__ void __launch_bounds__(128) k_pt_shade(const DeviceScene s, const RenderConsts rc, const PathState st,
                                                  int k, int qin, int qout)
{
    const int64_t count = (int64_t)st.counters[qin];
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    // Whole warps iterate together so that the queue appends stay warp-wide.
    const int64_t rounds = (count + stride - 1) / stride;
    for (int64_t r = 0; r < rounds; r++) {
        const int64_t j = r * stride + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
        const bool valid = j < count;
        const int32_t i = valid ? st.queue[qin][j] : 0;
        bool alive = false, shadow = false;
        V3 thr = v3(0, 0, 0), L = v3(0, 0, 0);
        Geom g;
        BsdfSample bs;
        V3 sh_target = v3(0, 0, 0), sh_c = v3(0, 0, 0);
        if (valid) {
            const uint64_t key = sample_key(rc.seed, (uint64_t)(rc.sample_base + i));
            const float4 h4 = st.hit[i];
            const float4 o4 = st.ray_o[i], d4 = st.ray_d[i];
            const V3 ro = f3(o4), rd = f3(d4);
            const V3 wi = -rd;
            thr = f3(st.thr[i]);
            L = f3(st.L[i]);
            const int32_t tri = __float_as_int(h4.x);
            V3 Le = v3(0, 0, 0);
            float light_pdf_area = 0.0f;   // EvaluatePositionPDF of the light that was hit
            bool hit_surface = false, is_env = false;
            Material m;
            m.type = LMGPU_BSDF_BLACK;
            m.R = v3(0, 0, 0);
            if (tri < 0) {
                float t;
                if (s.has_env && env_sphere_intersect(s, ro, rd, o4.w, FLT_MAX, t)) {
                    env_surface(s, ro, rd, t, g);
                    Le = emitted(load3(s.env_Le), g.sn, wi);
                    light_pdf_area = s.env_inv_area;
                    is_env = true;
                }
            } else {
                surface_from_hit(s, tri, h4.z, h4.w, ro, rd, h4.y, g);
                const int prim = s.tri_prim[tri];
                const int li = s.prim_light[prim];
                if (li >= 0) {
                    const AreaLightGpu al = s.area_lights[li];
                    Le = emitted(load3(al.Le), g.sn, wi);
                    light_pdf_area = al.inv_area;
                }
                m = material_of(s, prim);
                hit_surface = true;
            }
            // ---- emission reached by BSDF sampling
            if (!is_zero(Le)) {
                if (TECH == LMGPU_RENDER_PT) {
                    L = L + thr * Le;
                } else {
                    const float4 pp = st.prev_p[i], pn = st.prev_n[i];
                    const uint32_t flags = __float_as_uint(pn.w);
                    if (flags & PREV_SPECULAR) {
                        L = L + thr * Le;
                    } else if (TECH == LMGPU_RENDER_PT_MIS) {
                        const float G = geometry_term(f3(pp), f3(pn), (flags & PREV_DEGENERATED) != 0, g.p, g.sn, false);
                        const float pdf_dl = G == 0.0f ? 0.0f : light_pdf_area / (float(s.num_lights) * G);
                        L = L + thr * Le * (pp.w / (pp.w + pdf_dl));
                    }
                }
            }
            (void)is_env;
            const int v = k + 1;   // numPathVertices once this hit is accepted
            alive = hit_surface;
            if (TECH != LMGPU_RENDER_PT && alive && rc.max_pv != -1 && v >= rc.max_pv) alive = false;
            if (alive && TECH != LMGPU_RENDER_PT && has_non_delta(m.type)) {
                // ---- next-event estimation at vertex v
                LightPoint lp;
                if (sample_light(s, rng_uniform(key, dim_vertex(v) + DIM_LIGHT), rng_uniform(key, dim_vertex(v) + DIM_LIGHT + 1), lp)) {
                    const V3 ppL = normalize(lp.p - g.p);
                    float pdf_bsdf;
                    const V3 fs = eval_bsdf(m, g, wi, ppL, pdf_bsdf);
                    const float G = geometry_term(g.p, g.sn, false, lp.p, lp.n, false);
                    const V3 Lel = emitted(lp.Le, lp.n, -ppL);
                    if (G != 0.0f && !is_zero(fs) && !is_zero(Lel)) {
                        float w = 1.0f;
                        if (TECH == LMGPU_RENDER_PT_MIS) {
                            const float pdf_dl = lp.pdf_area / G;
                            w = pdf_dl / (pdf_dl + pdf_bsdf);
                        }
                        sh_c = thr * fs * Lel * (w * G / lp.pdf_area);
                        sh_target = lp.p;
                        shadow = !is_zero(sh_c);
                    }
                }
            }
            if (alive) {
                const int kv = TECH == LMGPU_RENDER_PT ? k : v;
                if (TECH != LMGPU_RENDER_PT && rc.rr_depth != -1 && kv >= rc.rr_depth) {
                    const float p = fminf(0.5f, luminance(thr));
                    if (rng_uniform(key, dim_vertex(kv) + DIM_RR) > p) alive = false;
                    else thr = thr / p;
                }
                if (alive) {
                    bs = sample_bsdf(m, g, wi, rng_uniform(key, dim_vertex(kv) + DIM_BSDF),
                                     rng_uniform(key, dim_vertex(kv) + DIM_BSDF + 1), rng_uniform(key, dim_vertex(kv) + DIM_COMP));
                    if (is_zero(bs.weight)) alive = false;
                    else thr = thr * bs.weight;
                }
                if (alive && TECH == LMGPU_RENDER_PT && rc.rr_depth != -1 && k >= rc.rr_depth) {
                    const float p = fminf(0.5f, luminance(thr));
                    if (rng_uniform(key, dim_vertex(k) + DIM_RR) > p) alive = false;
                    else thr = thr / p;
                }
                if (alive && TECH == LMGPU_RENDER_PT && rc.max_pv != -1 && k + 1 >= rc.max_pv) alive = false;
            }
            st.L[i] = f4(L, 0.0f);
        }
        const uint32_t sslot = queue_append(&st.counters[2], shadow);
        if (shadow) write_shadow(st, sslot, g.p, sh_target, sh_c, i);
        const uint32_t slot = queue_append(&st.counters[qout], alive);
        if (alive) {
            st.thr[i] = f4(thr, 0.0f);
            st.ray_o[i] = f4(g.p, EPS_F);
            st.ray_d[i] = f4(bs.wo, 0.0f);
            if (TECH != LMGPU_RENDER_PT) {
                st.prev_p[i] = f4(g.p, bs.pdf);
                st.prev_n[i] = f4(g.sn, __uint_as_float(bs.specular ? PREV_SPECULAR : 0u));
            }
            st.queue[qout][slot] = i;
        }
    }
}

// Film splat of each path's radiance at its raster position.
template <class F>
__global__ void __launch_bounds__(128) k_pt_splat(const DeviceScene s, const PathState st, int64_t count, F* film)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const float2 r = st.raster[i];
    film_add(film, film_pixel(s.cam, r.x, r.y), f3(st.L[i]));
}

// ------------------------------------------------------------ driver ------

// Wave workspace (scratch), cached per scene and grown on demand.
struct Workspace {
    int64_t capacity = 0;
    void* mem = nullptr;
    uint32_t* host_counts = nullptr;   // pinned
    PathState st{};
};

int ensure_workspace(Workspace& ws, int64_t paths)
{
    if (!ws.host_counts) LMGPU_CUDA_TRY(cudaMallocHost(&ws.host_counts, 16));
    if (ws.capacity >= paths && ws.mem) return LMGPU_OK;
    if (ws.mem) { cudaFree(ws.mem); ws.mem = nullptr; ws.capacity = 0; }
    const size_t P = (size_t)paths;
    const size_t bytes = P * (16 * 10 + 8 + 4 * 2) + 256;
    cudaError_t e = cudaMalloc(&ws.mem, bytes);
    if (e != cudaSuccess) return e == cudaErrorMemoryAllocation ? fail(LMGPU_ERR_OOM, "render workspace allocation failed")
                                                                 : cuda_fail(e, "cudaMalloc(workspace)");
    char* p = static_cast<char*>(ws.mem);
    auto take = [&](size_t b) { char* r = p; p += b; return r; };
    PathState& st = ws.st;
    st.counters = reinterpret_cast<uint32_t*>(take(256));
    st.ray_o = reinterpret_cast<float4*>(take(16 * P));
    st.ray_d = reinterpret_cast<float4*>(take(16 * P));
    st.hit = reinterpret_cast<float4*>(take(16 * P));
    st.thr = reinterpret_cast<float4*>(take(16 * P));
    st.L = reinterpret_cast<float4*>(take(16 * P));
    st.prev_p = reinterpret_cast<float4*>(take(16 * P));
    st.prev_n = reinterpret_cast<float4*>(take(16 * P));
    st.sh_o = reinterpret_cast<float4*>(take(16 * P));
    st.sh_d = reinterpret_cast<float4*>(take(16 * P));
    st.sh_c = reinterpret_cast<float4*>(take(16 * P));
    st.raster = reinterpret_cast<float2*>(take(8 * P));
    st.queue[0] = reinterpret_cast<int32_t*>(take(4 * P));
    st.queue[1] = reinterpret_cast<int32_t*>(take(4 * P));
    ws.capacity = paths;
    return LMGPU_OK;
}

template <class F>
int shadow_pass(LmgpuScene* sc, const PathState& st, F* film, int64_t max_rays, cudaStream_t stream)
{
    ShadowIO<F> io{ st.counters + 2, st.sh_o, st.sh_d, st.sh_c, st.L, film, sc->dev };
    return launch_trace<true>(sc, io, max_rays, stream);
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
    const DeviceScene& s = sc->dev;
    const int64_t pixels = (int64_t)s.cam.width * s.cam.height;
    int64_t P = p.wave_paths > 0 ? p.wave_paths : (int64_t(1) << 22);
    P = std::min<int64_t>(P, p.num_samples);
    int rc = ensure_workspace(ws, P);
    if (rc != LMGPU_OK) return rc;
    const PathState& st = ws.st;
    RenderConsts c;
    c.technique = TECH;
    c.rr_depth = p.rr_depth;
    c.max_pv = p.max_path_vertices;
    c.sampling = p.sampling;
    c.seed = p.seed;
    c.pixels = pixels;
    const int shade_blocks = 148 * 8;
    for (int64_t base = 0; base < p.num_samples && rc == LMGPU_OK; base += P) {
        const int64_t cnt = std::min<int64_t>(P, p.num_samples - base);
        c.sample_base = p.sample_offset + base;
        stats.waves++;
        stats.paths += cnt;
        if (c.max_pv != -1 && c.max_pv <= 1) continue;   // no path vertex beyond the camera
        LMGPU_CUDA_TRY(cudaMemsetAsync(st.counters, 0, 16, stream));
        k_pt_init<TECH><<<(unsigned)((cnt + 127) / 128), 128, 0, stream>>>(s, c, st, cnt);
        LMGPU_CUDA_TRY(cudaGetLastError());
        if (TECH != LMGPU_RENDER_PT) {
            if ((rc = read_counts(ws, stream)) != LMGPU_OK) break;
            stats.shadow_rays += ws.host_counts[2];
            if (ws.host_counts[2]) rc = shadow_pass(sc, st, film, ws.host_counts[2], stream);
        }
        int qin = 0;
        for (int k = 1; rc == LMGPU_OK; k++) {
            if (c.max_pv != -1 && k >= c.max_pv) break;
            if ((rc = read_counts(ws, stream)) != LMGPU_OK) break;
            const uint32_t n = ws.host_counts[qin];
            if (n == 0) break;
            stats.rays_traced += n;
            stats.max_bounces_run = std::max(stats.max_bounces_run, k);
            PathRayIO io{ st.queue[qin], st.counters + qin, st.ray_o, st.ray_d, st.hit };
            rc = launch_trace<false>(sc, io, n, stream);
            if (rc != LMGPU_OK) break;
            LMGPU_CUDA_TRY(cudaMemsetAsync(st.counters + (1 - qin), 0, 4, stream));
            LMGPU_CUDA_TRY(cudaMemsetAsync(st.counters + 2, 0, 4, stream));
            const unsigned blocks = (unsigned)std::min<int64_t>((n + 127) / 128, shade_blocks);
            k_pt_shade<TECH><<<blocks, 128, 0, stream>>>(s, c, st, k, qin, 1 - qin);
            LMGPU_CUDA_TRY(cudaGetLastError());
            if (TECH != LMGPU_RENDER_PT) {
                if ((rc = read_counts(ws, stream)) != LMGPU_OK) break;
                stats.shadow_rays += ws.host_counts[2];
                if (ws.host_counts[2]) rc = shadow_pass(sc, st, film, ws.host_counts[2], stream);
            }
            qin = 1 - qin;
        }
        if (rc == LMGPU_OK) {
            k_pt_splat<F><<<(unsigned)((cnt + 127) / 128), 128, 0, stream>>>(s, st, cnt, film);
            LMGPU_CUDA_TRY(cudaGetLastError());
        }
    }
    stats.rays_traced += stats.shadow_rays;
    return rc;
}

template <class F>
int render_dispatch(LmgpuScene* sc, const LmgpuRenderParams& p, F* film, cudaStream_t stream, LmgpuRenderStats& stats)
{
    Workspace& ws = *static_cast<Workspace*>(sc->render_ws);
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
    if (!sc->dev.cam.valid) return fail(LMGPU_ERR_INVALID, "scene has no camera");
    if (p->num_samples <= 0) return fail(LMGPU_ERR_INVALID, "num_samples must be positive");
    if (p->sample_offset < 0) return fail(LMGPU_ERR_INVALID, "negative sample offset");
    if (p->technique < LMGPU_RENDER_PT || p->technique > LMGPU_RENDER_PT_MIS) return fail(LMGPU_ERR_INVALID, "unknown technique");
    if (p->sampling != LMGPU_SAMPLING_STRATIFIED && p->sampling != LMGPU_SAMPLING_UNIFORM) return fail(LMGPU_ERR_INVALID, "unknown sampling");
    if (p->wave_paths < 0) return fail(LMGPU_ERR_INVALID, "negative wave size");
    if (!sc->render_ws) sc->render_ws = new Workspace;
    return LMGPU_OK;
}

template <class F>
__global__ void k_rescale(const F* film, float* out, int64_t n, double scale)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = (float)((double)film[i] * scale);
}

// Bytes of wave workspace per path (ensure_workspace's layout) and the
// fixed header of counters.
constexpr size_t WS_BYTES_PER_PATH = 16 * 10 + 8 + 4 * 2;
constexpr size_t WS_HEADER_BYTES = 256;

// Points a Workspace at caller-owned memory (same layout as
// ensure_workspace, no allocation); host_counts is the caller's readback
// buffer for the queue counters.
void carve_workspace(Workspace& ws, void* mem, int64_t paths, uint32_t* host_counts)
{
    const size_t P = (size_t)paths;
    char* p = static_cast<char*>(mem);
    auto take = [&](size_t b) { char* r = p; p += b; return r; };
    PathState& st = ws.st;
    st.counters = reinterpret_cast<uint32_t*>(take(WS_HEADER_BYTES));
    st.ray_o = reinterpret_cast<float4*>(take(16 * P));
    st.ray_d = reinterpret_cast<float4*>(take(16 * P));
    st.hit = reinterpret_cast<float4*>(take(16 * P));
    st.thr = reinterpret_cast<float4*>(take(16 * P));
    st.L = reinterpret_cast<float4*>(take(16 * P));
    st.prev_p = reinterpret_cast<float4*>(take(16 * P));
    st.prev_n = reinterpret_cast<float4*>(take(16 * P));
    st.sh_o = reinterpret_cast<float4*>(take(16 * P));
    st.sh_d = reinterpret_cast<float4*>(take(16 * P));
    st.sh_c = reinterpret_cast<float4*>(take(16 * P));
    st.raster = reinterpret_cast<float2*>(take(8 * P));
    st.queue[0] = reinterpret_cast<int32_t*>(take(4 * P));
    st.queue[1] = reinterpret_cast<int32_t*>(take(4 * P));
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
    if (!film) return fail(LMGPU_ERR_INVALID, "null film");
    if (!sc->dev.cam.valid) return fail(LMGPU_ERR_INVALID, "scene has no camera");
    if (p.num_samples <= 0) return fail(LMGPU_ERR_INVALID, "num_samples must be positive");
    if (p.sample_offset < 0) return fail(LMGPU_ERR_INVALID, "negative sample offset");
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

// Frees a scene's render workspace (called by lmgpu_scene_destroy).
void release_render_workspace(LmgpuScene* sc)
{
    if (!sc->render_ws) return;
    Workspace* ws = static_cast<Workspace*>(sc->render_ws);
    if (ws->mem) cudaFree(ws->mem);
    if (ws->host_counts) cudaFreeHost(ws->host_counts);
    delete ws;
    sc->render_ws = nullptr;
}

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
    int rc = check_params(scene, params);
    if (rc != LMGPU_OK) return rc;
    if (!film_device) return fail(LMGPU_ERR_INVALID, "null film");
    LmgpuRenderStats st;
    std::memset(&st, 0, sizeof(st));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaEvent_t e0, e1;
    LMGPU_CUDA_TRY(cudaEventCreate(&e0));
    LMGPU_CUDA_TRY(cudaEventCreate(&e1));
    LMGPU_CUDA_TRY(cudaEventRecord(e0, s));
    if (params->film_fp64) rc = render_dispatch(scene, *params, static_cast<double*>(film_device), s, st);
    else rc = render_dispatch(scene, *params, static_cast<float*>(film_device), s, st);
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
    void* film = nullptr;
    float* out = nullptr;
    LMGPU_CUDA_TRY(cudaMalloc(&film, n * esize));
    cudaError_t e = cudaMalloc(&out, n * sizeof(float));
    if (e != cudaSuccess) { cudaFree(film); return cuda_fail(e, "cudaMalloc(film)"); }
    e = cudaMemset(film, 0, n * esize);
    if (e != cudaSuccess) rc = cuda_fail(e, "cudaMemset(film)");
    if (rc == LMGPU_OK) rc = lmgpu_render_device(scene, params, film, nullptr, stats);
    if (rc == LMGPU_OK) {
        // Rescale(W * H / num_samples) (sched.mt.cpp:250-256, hdrfilm.cpp:334-341).
        const double scale = double(scene->dev.cam.width) * scene->dev.cam.height / double(params->num_samples);
        const unsigned blocks = (unsigned)((n + 255) / 256);
        if (params->film_fp64) k_rescale<double><<<blocks, 256>>>(static_cast<double*>(film), out, n, scale);
        else k_rescale<float><<<blocks, 256>>>(static_cast<float*>(film), out, n, scale);
        e = cudaMemcpy(film_host, out, n * sizeof(float), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) rc = cuda_fail(e, "cudaMemcpy(film)");
    }
    cudaFree(film);
    cudaFree(out);
    return rc;
}

}  // extern "C"
