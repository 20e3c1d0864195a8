// Wavefront path-tracing kernels: wave initialisation, shading, film splat
// and the queue I/O of the traversal kernel.
//
// They follow the reference renderers' per-sample loops
//   pt         pathtrace.cpp:165-266
//   pt.direct  pathtrace.direct.cpp:170-338
//   pt.mis     pathtrace.mis.cpp:167-369
// restructured into waves of paths that advance one bounce per kernel
// sequence: trace (closest hit) -> shade (emission, next-event estimation,
// Russian roulette, BSDF sampling) -> shadow (any hit) -> ... -> splat.
//
// Every kernel is written against a context policy that gives, for a path,
// its scene, its render constants, its scene-local sample index and its film:
//   OneScene<F>    one scene and one set of constants in kernel parameters
//                  (lmgpu_render*, pathtrace.cu);
//   SceneTable<F>  a device table of scenes: a wave spans the samples of many
//                  scenes, each path records its scene index, and the wave's
//                  position comes from device memory, so one captured wave
//                  replays unchanged (the multi-scene batch, batch.cu);
//   StreamTable<F> the same table with path regeneration: a fixed pool of
//                  path slots, each path with its own sample index and
//                  depth; finished paths retire (splat, free their slot) and
//                  new camera paths take free slots every iteration, so the
//                  queues stay full until the samples run out.
// A sample's random numbers depend only on (seed, scene-local sample index,
// dimension), so a scene renders the same paths alone or in a batch.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

#include "../../include/lmgpu.h"
#include "pathtrace.cuh"
#include "rng.cuh"
#include "scene.cuh"
#include "shading.cuh"
#include "trace.cuh"

namespace lmgpu {

constexpr uint32_t PREV_DEGENERATED = 1u;   // previous vertex is the pinhole
constexpr uint32_t PREV_SPECULAR = 2u;      // last BSDF sample was specular

// Device pointers of one wave's path state (capacity paths). The two ray
// queues hold each live path's ray and its state between bounces in queue
// order (see queue_ray), so the traversal and the shading read them, and
// the hits, contiguously; the ray's origin is the previous vertex.
struct PathState {
    float4* qo[2];     // queued ray: origin, scene index (int bits)
    float4* qd[2];     // direction, path slot | QUEUE_TMIN_ZERO (uint bits)
    float4* qt[2];     // throughput, previous vertex's BSDF pdf (projected solid angle)
    float4* qn[2];     // previous vertex's shading normal, flags (uint bits); pt.direct / pt.mis
    float4* hit;       // by slot of the traced queue: tri (int bits), t, u, v
    float4* L;         // radiance to splat at the path's raster position
    float2* raster;
    float4* sh_o;      // shadow ray origin, maxT
    float4* sh_d;      // direction, target (int bits: path index, or ~pixel)
    float4* sh_c;      // contribution, scene index (int bits)
    uint32_t* counters;   // [0], [1] ray queues; [2] shadow queue
    int32_t* scene;    // per path scene index (SceneTable, StreamTable)
    int64_t* sample;   // per path batch-global sample index (StreamTable)
    int32_t* depth;    // per path index k of its next bounce (StreamTable)
    int32_t* free_slots;   // free path slots (StreamTable)
    int32_t* retire;   // paths finished this iteration (StreamTable; counters[3])
    // Bounds-checked build: the queues' capacities (queue_append) and the
    // status word that records an append beyond one.
    uint32_t cap[4];
    int32_t* status;
};

struct RenderConsts {
    int32_t technique;
    int32_t rr_depth;
    int32_t max_pv;
    int32_t sampling;
    uint64_t seed;
    int64_t sample_base;   // OneScene: sample index of the wave's path 0; SceneTable: the scene's sample offset
    int64_t pixels;
    double inv_pixels;     // 1 / pixels
};

// ------------------------------------------------------------ contexts ----

template <class F>
struct OneScene {
    static constexpr bool TABLE = false;
    DeviceScene s;
    RenderConsts rc;
    F* film;
    __device__ __forceinline__ const DeviceScene& scene(int) const { return s; }
    __device__ __forceinline__ const RenderConsts& consts(int) const { return rc; }
    __device__ __forceinline__ int64_t wave_count(int64_t n) const { return n; }
    // Scene index and scene-local sample index of wave path i.
    __device__ __forceinline__ int locate(int64_t i, int64_t& sample) const
    {
        sample = rc.sample_base + i;
        return 0;
    }
    __device__ __forceinline__ int path_scene(const PathState&, int64_t) const { return 0; }
    __device__ __forceinline__ int64_t sample_of(int, int64_t i) const { return rc.sample_base + i; }
    __device__ __forceinline__ F* film_of(int) const { return film; }
    // New path number j of this launch: its slot i and scene-local sample.
    __device__ __forceinline__ int begin_path(const PathState&, int64_t j, int64_t& i, int64_t& sample) const
    {
        i = j;
        return locate(j, sample);
    }
    __device__ __forceinline__ int path_depth(const PathState&, int64_t, int k) const { return k; }
    static constexpr bool STREAM = false;
};

// One scene of a batch as the kernels see it.
struct BatchEntry {
    DeviceScene s;
    RenderConsts rc;       // rc.sample_base = the scene's sample_offset
    int64_t begin;         // batch-global index of the scene's first sample
    void* film;            // the scene's device film (float or double)
};

// Position of the current wave in the batch's sample sequence; advanced on
// the device at the end of each wave.
struct WaveCtl {
    int64_t base;          // batch-global sample index of path 0
    int64_t count;         // paths in this wave
    int64_t total;         // samples of the whole batch
    int64_t step;          // wave capacity
    int64_t stride;        // samples between this pool's consecutive waves (step × pools)
};

template <class F>
struct SceneTable {
    static constexpr bool TABLE = true;
    const BatchEntry* table;
    const int64_t* begins;   // num_scenes + 1 ascending sample boundaries
    int32_t num_scenes;
    const WaveCtl* wave;
    __device__ __forceinline__ const DeviceScene& scene(int sid) const { return table[sid].s; }
    __device__ __forceinline__ const RenderConsts& consts(int sid) const { return table[sid].rc; }
    __device__ __forceinline__ int64_t wave_count(int64_t) const { return wave->count; }
    __device__ __forceinline__ int locate(int64_t i, int64_t& sample) const
    {
        const int64_t g = wave->base + i;
        int lo = 0, hi = num_scenes;    // begins[lo] <= g < begins[hi]
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (begins[mid] <= g) lo = mid;
            else hi = mid;
        }
        sample = table[lo].rc.sample_base + (g - begins[lo]);
        return lo;
    }
    __device__ __forceinline__ int path_scene(const PathState& st, int64_t i) const { return st.scene[i]; }
    __device__ __forceinline__ int64_t sample_of(int sid, int64_t i) const
    {
        return table[sid].rc.sample_base + (wave->base + i - table[sid].begin);
    }
    __device__ __forceinline__ F* film_of(int sid) const { return static_cast<F*>(table[sid].film); }
    __device__ __forceinline__ int begin_path(const PathState& st, int64_t j, int64_t& i, int64_t& sample) const
    {
        i = j;
        const int sid = locate(j, sample);
        st.scene[i] = sid;
        return sid;
    }
    __device__ __forceinline__ int path_depth(const PathState&, int64_t, int k) const { return k; }
    static constexpr bool STREAM = false;
};

// Plan of one regenerating iteration, written by a one-thread kernel.
struct StreamCtl {
    int64_t next;          // next batch-global sample to start
    int64_t total;         // samples of the whole batch
    int64_t free_count;    // free slots (free_slots[0, free_count))
    int64_t n_new;         // paths started this iteration
    int64_t free_base;     // they take free_slots[free_base, free_base + n_new)
    int64_t g0;            // batch-global sample of the first of them
    int64_t capacity;      // path slots
    int64_t iterations;
    int64_t done;          // all samples started and every slot free
};

template <class F>
struct StreamTable {
    static constexpr bool TABLE = true;
    static constexpr bool STREAM = true;
    const BatchEntry* table;
    const int64_t* begins;
    int32_t num_scenes;
    const StreamCtl* ctl;
    const int64_t* sample;            // PathState::sample
    unsigned long long* max_depth;    // statistics: deepest bounce reached
    __device__ __forceinline__ const DeviceScene& scene(int sid) const { return table[sid].s; }
    __device__ __forceinline__ const RenderConsts& consts(int sid) const { return table[sid].rc; }
    __device__ __forceinline__ int64_t wave_count(int64_t) const { return ctl->n_new; }
    __device__ __forceinline__ int path_scene(const PathState& st, int64_t i) const { return st.scene[i]; }
    __device__ __forceinline__ int64_t sample_of(int sid, int64_t i) const
    {
        return table[sid].rc.sample_base + (sample[i] - table[sid].begin);
    }
    __device__ __forceinline__ F* film_of(int sid) const { return static_cast<F*>(table[sid].film); }
    __device__ __forceinline__ int begin_path(const PathState& st, int64_t j, int64_t& i, int64_t& local) const
    {
        i = st.free_slots[ctl->free_base + j];
        const int64_t g = ctl->g0 + j;
        int lo = 0, hi = num_scenes;    // begins[lo] <= g < begins[hi]
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (begins[mid] <= g) lo = mid;
            else hi = mid;
        }
        local = table[lo].rc.sample_base + (g - begins[lo]);
        st.scene[i] = lo;
        st.sample[i] = g;
        st.depth[i] = 1;
        return lo;
    }
    __device__ __forceinline__ int path_depth(const PathState& st, int64_t i, int) const { return st.depth[i]; }
};

// ------------------------------------------------------------- helpers ----

// Warp-aggregated append to queue q (counters[q]): returns this lane's slot
// (the whole warp must reach the call). In the bounds-checked build a slot
// at or beyond the queue's capacity is not handed out: the lane gets
// NO_SLOT (slot_ok is false), the status word records
// STATUS_QUEUE_OVERFLOW, and the counter is brought back to the capacity.
// The counter then never drops below the capacity again, so every slot
// below it is handed out exactly once and no later kernel reads past it.
constexpr uint32_t NO_SLOT = 0xffffffffu;
__device__ __forceinline__ bool slot_ok(uint32_t slot) { return !LMGPU_BOUNDS_CHECK || slot != NO_SLOT; }

__device__ __forceinline__ uint32_t queue_append(const PathState& st, int q, bool want)
{
    uint32_t* counter = &st.counters[q];
    const unsigned active = __activemask();
    const unsigned mask = __ballot_sync(active, want);
    if (!want) return NO_SLOT;
    const unsigned lane = threadIdx.x & 31u;
    const int leader = __ffs(mask) - 1;
    uint32_t base = 0;
    if ((int)lane == leader) base = atomicAdd(counter, (uint32_t)__popc(mask));
    base = __shfl_sync(mask, base, leader);
    const uint32_t slot = base + __popc(mask & ((1u << lane) - 1u));
#if LMGPU_BOUNDS_CHECK
    const uint32_t cap = st.cap[q];
    if ((int)lane == leader && base + __popc(mask) > cap) {
        atomicMin(counter, cap);
        atomicOr(st.status, STATUS_QUEUE_OVERFLOW);
    }
    if (slot >= cap) return NO_SLOT;
#endif
    return slot;
}

__device__ __forceinline__ V3 f3(float4 q) { return v3(q.x, q.y, q.z); }
__device__ __forceinline__ float4 f4(V3 v, float w) { return make_float4(v.x, v.y, v.z, w); }

// A queued ray's minT is Eps, except pt's camera rays (minT 0,
// pathtrace.cpp:187, 245); the flag shares the word of the path slot
// (slots < 2^31).
constexpr uint32_t QUEUE_TMIN_ZERO = 0x80000000u;

template <int TECH>
__device__ __forceinline__ void queue_ray(const PathState& st, int q, uint32_t slot, V3 o, V3 d, int64_t i, int sid,
                                          bool tmin_zero, V3 thr, float pdf, V3 n, uint32_t flags)
{
    st.qo[q][slot] = f4(o, __int_as_float(sid));
    st.qd[q][slot] = f4(d, __uint_as_float((uint32_t)i | (tmin_zero ? QUEUE_TMIN_ZERO : 0u)));
    st.qt[q][slot] = f4(thr, pdf);
    if (TECH != LMGPU_RENDER_PT) st.qn[q][slot] = f4(n, __uint_as_float(flags));
}
__device__ __forceinline__ int32_t queued_path(float4 d) { return (int32_t)(__float_as_uint(d.w) & ~QUEUE_TMIN_ZERO); }
__device__ __forceinline__ float queued_tmin(float4 d)
{
    return (__float_as_uint(d.w) & QUEUE_TMIN_ZERO) ? 0.0f : EPS_F;
}
__device__ __forceinline__ int queued_scene(float4 o) { return __float_as_int(o.w); }

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
__device__ __forceinline__ void write_shadow(const PathState& st, uint32_t slot, V3 p, V3 target, V3 c, int32_t dest,
                                             int sid)
{
    const V3 d = target - p;
    const float len = sqrtf(length2(d));
    st.sh_o[slot] = f4(p, len * (1.0f - EPS_F));
    st.sh_d[slot] = f4(d / len, __int_as_float(dest));
    st.sh_c[slot] = f4(c, __int_as_float(sid));
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

// ------------------------------------------------------------- kernels ----

// Wave initialisation: raster sample and camera ray; for pt.direct / pt.mis
// the whole camera vertex (light sample, Russian roulette). `count` is the
// wave's path count for OneScene (the tables read it from the device); new
// rays join ray queue q.
template <int TECH, class Ctx>
__global__ void __launch_bounds__(128) k_pt_init(const Ctx ctx, const PathState st, int64_t count, int q)
{
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= ctx.wave_count(count)) return;
    int64_t sample, i;
    const int sid = ctx.begin_path(st, j, i, sample);
    const DeviceScene& s = ctx.scene(sid);
    const RenderConsts& rc = ctx.consts(sid);
    const uint64_t key = sample_key(rc.seed, (uint64_t)sample);
    const float u0 = rng_uniform(key, DIM_RASTER), u1 = rng_uniform(key, DIM_RASTER + 1);
    float rx, ry;
    if (rc.sampling == LMGPU_SAMPLING_STRATIFIED) {
        stratified_raster(sample, rc.pixels, rc.inv_pixels, s.cam.width, s.cam.height, u0, u1, rx, ry);
    } else {
        rx = u0; ry = u1;
    }
    float pdf_cam;
    const V3 dir = camera_direction(s.cam, rx, ry, pdf_cam);
    const V3 cp = load3(s.cam.position);
    st.raster[i] = make_float2(rx, ry);
    st.L[i] = make_float4(0, 0, 0, 0);
    V3 thr = v3(1, 1, 1);
    // No vertex beyond the camera: the path contributes nothing (the
    // one-scene driver skips such waves before launching).
    bool alive = rc.max_pv == -1 || rc.max_pv > 1;
    if (TECH != LMGPU_RENDER_PT && alive) {
        V3 target, c;
        int32_t dest;
        const bool shadow = camera_nee<TECH>(s, key, target, c, dest);
        const uint32_t sslot = queue_append(st, 2, shadow);
        if (shadow && slot_ok(sslot)) write_shadow(st, sslot, cp, target, c, dest, sid);
        if (rc.rr_depth != -1 && 1 >= rc.rr_depth) {
            const float p = fminf(0.5f, luminance(thr));
            if (rng_uniform(key, dim_vertex(1) + DIM_RR) > p) alive = false;
            else thr = thr / p;
        }
    }
    const uint32_t slot = queue_append(st, q, alive);
    if (alive && slot_ok(slot))
        queue_ray<TECH>(st, q, slot, cp, dir, i, sid, TECH == LMGPU_RENDER_PT, thr, pdf_cam, v3(0, 0, 1), PREV_DEGENERATED);
    if (Ctx::STREAM) {                           // a path that ends at the camera retires at once
        const uint32_t r = queue_append(st, 3, !alive);
        if (!alive && slot_ok(r)) st.retire[r] = (int32_t)i;
    }
}

// Closest-hit traversal of the queued rays (writes hit records). With a
// scene table each ray is traced in its own path's scene.
// Both path-tracer queues refill traversal lanes once 20 are idle and pause
// a descent once fewer than 16 lanes still descend. Measured with the render
// walks (1080p terrain frame / 64-scene batch): 166.7 / 793.9 ms against
// 171.0 / 804.6 ms at (24, 24); pausing below 20 lanes or refilling 16 at a
// time was slower, pausing below 28 slower still.
#ifndef LMGPU_PT_REFILL_MIN
#define LMGPU_PT_REFILL_MIN 20
#endif
#ifndef LMGPU_PT_EXIT_BELOW
#define LMGPU_PT_EXIT_BELOW 16
#endif
constexpr int PATH_QUEUE_REFILL_MIN = LMGPU_PT_REFILL_MIN;
constexpr int PATH_QUEUE_EXIT_BELOW = LMGPU_PT_EXIT_BELOW;
// The shadow queue's speculative any-hit walk refills at 12 idle lanes
// (shadow traversal of the 1080p frame 45.3 -> 44.2 ms; 8 and 28 were
// slower, and pausing below 8, 12 or 24 lanes instead of 16 did not help).
#ifndef LMGPU_PT_SHADOW_REFILL_MIN
#define LMGPU_PT_SHADOW_REFILL_MIN 12
#endif
#ifndef LMGPU_PT_SHADOW_EXIT_BELOW
#define LMGPU_PT_SHADOW_EXIT_BELOW LMGPU_PT_EXIT_BELOW
#endif

template <bool TABLE>
struct PathRayIO {
    static constexpr bool PER_RAY_SCENE = TABLE;
    static constexpr bool RENDER = true;
    static constexpr int REFILL_MIN = PATH_QUEUE_REFILL_MIN;
    static constexpr int EXIT_BELOW = PATH_QUEUE_EXIT_BELOW;
    const uint32_t* count_ptr;
    const float4* qo;
    const float4* qd;
    float4* hit;
    const BatchEntry* table;      // TABLE only
    __device__ int64_t count() const { return (int64_t)*count_ptr; }
    __device__ const DeviceScene& ray_scene(int64_t j) const { return table[queued_scene(qo[j])].s; }
    __device__ RayIn load(int64_t j) const
    {
        const float4 o = qo[j], d = qd[j];
        RayIn r;
        r.o[0] = o.x; r.o[1] = o.y; r.o[2] = o.z;
        r.d[0] = d.x; r.d[1] = d.y; r.d[2] = d.z;
        r.tmin = queued_tmin(d); r.tmax = FLT_MAX;
        return r;
    }
    __device__ void store(int64_t j, const Hit& h, const TraversalRay&) const
    {
        hit[j] = make_float4(__int_as_float(h.tri), h.t, h.u, h.v);
    }
};

// Shadow rays: visible iff neither a triangle nor the environment's emitter
// shape is hit within [Eps, maxT] (Scene::Intersect inside Visible); visible
// contributions go to the path's radiance or straight to the film.
template <class Ctx>
struct ShadowIO {
    static constexpr bool PER_RAY_SCENE = Ctx::TABLE;
    static constexpr bool RENDER = true;
    static constexpr int REFILL_MIN = LMGPU_PT_SHADOW_REFILL_MIN;
    static constexpr int EXIT_BELOW = LMGPU_PT_SHADOW_EXIT_BELOW;
    const uint32_t* count_ptr;
    const float4* sh_o;
    const float4* sh_d;
    const float4* sh_c;
    float4* L;
    Ctx ctx;
    __device__ int64_t count() const { return (int64_t)*count_ptr; }
    __device__ const DeviceScene& ray_scene(int64_t j) const { return ctx.scene(__float_as_int(sh_c[j].w)); }
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
        const float4 c4 = sh_c[j];
        const int sid = __float_as_int(c4.w);
        const DeviceScene& s = ctx.scene(sid);
        const V3 o = v3(r.o[0], r.o[1], r.o[2]), d = v3(r.d[0], r.d[1], r.d[2]);
        float te;
        if (s.has_env && env_sphere_intersect(s, o, d, r.tmin, sh_o[j].w, te)) return;
        const V3 c = f3(c4);
        const int32_t dest = __float_as_int(sh_d[j].w);
        if (dest >= 0) {
            const float4 l = L[dest];
            L[dest] = make_float4(l.x + c.x, l.y + c.y, l.z + c.z, 0.0f);
        } else {
            film_add(ctx.film_of(sid), ~dest, c);
        }
    }
};

// Shading of the hits of iteration k: emission at the hit (vertex k + 1),
// then for pt.direct / pt.mis next-event estimation at it, Russian roulette
// and BSDF sampling; pt samples the BSDF first and applies Russian roulette
// with numPathVertices = k (pathtrace.cpp:223-260).
// 8 resident blocks per SM (64 registers, a few spilled bytes): on the
// 1080p terrain frame 6, 7 and 10 blocks took 159.6, 159.7 and 164.0 ms
// against 156.7 ms; the 64-scene batch was within 0.5 % for all four.
#ifndef LMGPU_PT_SHADE_MIN_BLOCKS
#define LMGPU_PT_SHADE_MIN_BLOCKS 8
#endif
template <int TECH, class Ctx>
__global__ void __launch_bounds__(128, LMGPU_PT_SHADE_MIN_BLOCKS) k_pt_shade(const Ctx ctx, const PathState st, int kw,
                                                                            int qin, int qout)
{
    const int64_t count = (int64_t)st.counters[qin];
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    // Whole warps iterate together so that the queue appends stay warp-wide.
    const int64_t rounds = (count + stride - 1) / stride;
    for (int64_t r = 0; r < rounds; r++) {
        const int64_t j = r * stride + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
        const bool valid = j < count;
        const float4 o4 = valid ? st.qo[qin][j] : make_float4(0, 0, 0, 0);
        const float4 d4 = valid ? st.qd[qin][j] : make_float4(0, 0, 0, 0);
        const int32_t i = queued_path(d4);
        const int sid = queued_scene(o4);
        const int k = valid ? ctx.path_depth(st, i, kw) : kw;   // this bounce's index
        bool alive = false, shadow = false;
        V3 thr = v3(0, 0, 0);
        Geom g;
        BsdfSample bs;
        V3 sh_target = v3(0, 0, 0), sh_c = v3(0, 0, 0);
        if (valid) {
            const DeviceScene& s = ctx.scene(sid);
            const RenderConsts& rc = ctx.consts(sid);
            const uint64_t key = sample_key(rc.seed, (uint64_t)ctx.sample_of(sid, i));
            const float4 h4 = st.hit[j];
            const V3 ro = f3(o4), rd = f3(d4);
            const V3 wi = -rd;
            const float4 t4 = st.qt[qin][j];
            thr = f3(t4);
            const int32_t tri = __float_as_int(h4.x);
            V3 Le = v3(0, 0, 0);
            float light_pdf_area = 0.0f;   // EvaluatePositionPDF of the light that was hit
            bool hit_surface = false;
            Material m;
            m.type = LMGPU_BSDF_BLACK;
            m.R = v3(0, 0, 0);
            if (tri < 0) {
                float t;
                if (s.has_env && env_sphere_intersect(s, ro, rd, queued_tmin(d4), FLT_MAX, t)) {
                    env_surface(s, ro, rd, t, g);
                    Le = emitted(load3(s.env_Le), g.sn, wi);
                    light_pdf_area = s.env_inv_area;
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
            // ---- emission reached by BSDF sampling (the path's radiance is
            // read and written only here; shadow rays add to it later)
            if (!is_zero(Le)) {
                bool add = true;
                V3 c = thr * Le;
                if (TECH != LMGPU_RENDER_PT) {
                    const float4 pn = st.qn[qin][j];   // previous vertex: position ro, pdf t4.w
                    const uint32_t flags = __float_as_uint(pn.w);
                    if (flags & PREV_SPECULAR) {
                    } else if (TECH == LMGPU_RENDER_PT_MIS) {
                        const float G = geometry_term(ro, f3(pn), (flags & PREV_DEGENERATED) != 0, g.p, g.sn, false);
                        const float pdf_dl = G == 0.0f ? 0.0f : light_pdf_area / (float(s.num_lights) * G);
                        c = thr * Le * (t4.w / (t4.w + pdf_dl));
                    } else {
                        add = false;
                    }
                }
                if (add) {
                    const V3 L = f3(st.L[i]) + c;
                    st.L[i] = f4(L, 0.0f);
                }
            }
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
        }
        const uint32_t sslot = queue_append(st, 2, shadow);
        if (shadow && slot_ok(sslot)) write_shadow(st, sslot, g.p, sh_target, sh_c, i, sid);
        const uint32_t slot = queue_append(st, qout, alive);
        if (alive && slot_ok(slot)) {
            queue_ray<TECH>(st, qout, slot, g.p, bs.wo, i, sid, false, thr, bs.pdf, g.sn, bs.specular ? PREV_SPECULAR : 0u);
            if (Ctx::STREAM) st.depth[i] = k + 1;
        }
        if constexpr (Ctx::STREAM) {
            const bool done = valid && !alive;
            const uint32_t r = queue_append(st, 3, done);
            if (done && slot_ok(r)) st.retire[r] = i;
            const unsigned m = __reduce_max_sync(__activemask(), valid ? (unsigned)k : 0u);
            if ((threadIdx.x & 31u) == (unsigned)(__ffs(__activemask()) - 1)) atomicMax(ctx.max_depth, (unsigned long long)m);
        }
    }
}

// Retirement of the paths that finished this iteration (after the shadow
// pass, whose contributions they have received): splat their radiance and
// return their slots to the free list after the slots still free.
template <class Ctx>
__global__ void __launch_bounds__(128) k_pt_retire(const Ctx ctx, const PathState st)
{
    const int64_t n = (int64_t)st.counters[3];
    const int64_t base = ctx.ctl->free_count;
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x) {
        const int32_t i = st.retire[j];
        const int sid = ctx.path_scene(st, i);
        const float2 r = st.raster[i];
        film_add(ctx.film_of(sid), film_pixel(ctx.scene(sid).cam, r.x, r.y), f3(st.L[i]));
        st.free_slots[base + j] = i;
    }
}

// Film splat of each path's radiance at its raster position.
template <class Ctx>
__global__ void __launch_bounds__(128) k_pt_splat(const Ctx ctx, const PathState st, int64_t count)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ctx.wave_count(count)) return;
    const int sid = ctx.path_scene(st, i);
    const float2 r = st.raster[i];
    film_add(ctx.film_of(sid), film_pixel(ctx.scene(sid).cam, r.x, r.y), f3(st.L[i]));
}

}  // namespace lmgpu
