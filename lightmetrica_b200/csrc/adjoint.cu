// Differentiable rendering: a forward / adjoint pair over the path tracer
// with per-triangle diffuse albedo and per-light emission as parameters.
//
// Both passes run the same per-sample path (the reference's pt / pt.direct /
// pt.mis loops, pathtrace*.cpp) one thread per sample. The adjoint pass does
// not store path vertices from the forward pass: it replays every path from
// its counter-based random numbers (recomputation instead of checkpointing)
// and, for each radiance contribution c splatted at pixel p, adds
// dL/dI_p * c / R_t to the gradient of the albedo R of every diffuse vertex t
// on the contribution's prefix (c is linear in each of them) and
// dL/dI_p * c / Le to the emission of its light. A path's contributions come
// in order of non-decreasing prefix length ("depth"), so the replay keeps,
// for the first RECORDED_VERTS vertices, the sum of the weights
// w = dL/dI_p * c whose prefix ends there and turns them into suffix sums
// once the path is done: one set of atomics per vertex instead of one per
// (contribution, vertex). Emission gradients are summed per thread and per
// block before they reach global memory, since every path adds to the same
// few lights. Russian-roulette probabilities and MIS weights are held at
// their sampled values, which keeps the estimator unbiased for the diffuse
// BSDFs (their sampling densities do not depend on R).
//
// Paths deeper than RECORDED_VERTS vertices: the weights of all
// contributions deeper than that are summed into one total W_tail while the
// path runs, and the path's state on arrival at that depth is kept as a
// checkpoint (position, direction, throughput, previous vertex: a few
// registers' worth). When the path has ended, the first vertices' suffix
// sums start from W_tail, and the tail is replayed from the checkpoint a
// second time: a vertex i there is on the prefix of exactly the tail
// contributions deeper than i, so its weight is W_tail minus the running sum
// of the tail contributions met before it; no per-vertex record is needed.
// Only long paths pay for the second replay of their tail. A replay stops at
// MAX_PATH_VERTICES surface vertices and flags LMGPU_ERR_QUEUE_OVERFLOW: paths
// that long occur only in closed scenes without Russian roulette, where the
// reference's own loop (pathtrace*.cpp, `while (true)` with
// max_path_vertices = -1) does not end either.
#include <cuda_runtime.h>
#include <algorithm>
#include <cstring>

#include "../../include/lmgpu.h"
#include "internal.h"
#include "pathtrace.cuh"
#include "rng.cuh"
#include "trace.cuh"
#include "trace4.cuh"

namespace lmgpu {
namespace {

constexpr int RECORDED_VERTS = 32;          // vertices with a per-vertex record
constexpr int MAX_PATH_VERTICES = 4096;     // replay bound (surface vertices)

struct DiffConsts {
    int32_t technique, rr_depth, max_pv, sampling;
    uint64_t seed;
    int64_t sample_offset, num_samples, pixels;
    double inv_pixels;       // 1 / pixels
    float scale;             // film rescale W*H/num_samples
    const float* albedo;     // 3 per triangle or null
    const float* emission;   // 3 per area light or null
};

template <int LAYOUT, bool ANY, int STACK>
__device__ __forceinline__ int32_t cast_ray(const DeviceScene& s, V3 o, V3 d, float tmin, float tmax, Hit& h,
                                            int2* stack, int32_t* status)
{
    RayIn in;
    in.o[0] = o.x; in.o[1] = o.y; in.o[2] = o.z;
    in.d[0] = d.x; in.d[1] = d.y; in.d[2] = d.z;
    in.tmin = tmin; in.tmax = tmax;
    TraversalRay r;
    setup_ray<LAYOUT != LMGPU_LAYOUT_NAIVE>(r, in);   // a render ray (the naive scan keeps the exact setup)
    h.tri = -1;
    if (s.num_tris == 0) return -1;
    bool ok;
    const int cap = s.stack_cap < STACK ? s.stack_cap : STACK;
    // The renderers' walks and triangle test: the wavefront kernels' own.
    if (LAYOUT == LMGPU_LAYOUT_BVH2 && ANY && LMGPU_TRACE_ANYHIT_WALK)   // visibility: the any-hit walk
        ok = trace_bvh2_any<true>(s.bvh2, s.tris, s.root_ref, s.root_box, r, h, reinterpret_cast<int*>(stack), cap, nullptr);
    else if (LAYOUT == LMGPU_LAYOUT_BVH2) ok = trace_bvh2<ANY, true>(s.bvh2, s.tris, s.root_ref, s.root_box, r, h, stack, cap, nullptr);
    else if (LAYOUT == LMGPU_LAYOUT_BVH4) ok = trace_bvh4<ANY, true>(s.bvh4, s.tris, s.root_ref4, s.root_box, r, h, stack, cap, nullptr);
    else { trace_naive<ANY>(s.tris_by_id, s.num_tris, r, h, nullptr); ok = true; }
    if (!ok) { atomicOr(status, STATUS_STACK_OVERFLOW); h.tri = -1; }
    return h.tri;
}

template <int LAYOUT, int STACK>
__device__ __forceinline__ bool visible(const DeviceScene& s, V3 a, V3 b, int2* stack, int32_t* status)
{
    const V3 d = b - a;
    const float len = sqrtf(length2(d));
    const V3 dn = d / len;
    const float maxt = len * (1.0f - EPS_F);
    Hit h;
    if (cast_ray<LAYOUT, true, STACK>(s, a, dn, EPS_F, maxt, h, stack, status) >= 0) return false;
    float t;
    if (s.has_env && env_sphere_intersect(s, a, dn, EPS_F, maxt, t)) return false;
    return true;
}

__device__ __forceinline__ Material diff_material(const DeviceScene& s, const DiffConsts& c, int tri)
{
    Material m = material_of(s, s.tri_prim[tri]);
    if (c.albedo && m.type == LMGPU_BSDF_DIFFUSE) m.R = load3(c.albedo + 3 * (int64_t)tri);
    return m;
}

__device__ __forceinline__ V3 light_Le(const DeviceScene& s, const DiffConsts& c, int li)
{
    if (li >= s.num_area_lights) return load3(s.env_Le);
    return c.emission ? load3(c.emission + 3 * li) : load3(s.area_lights[li].Le);
}

// Per-path records of the adjoint. w[i] (i < RECORDED_VERTS): the weights
// of the contributions whose prefix ends at vertex i; w[TAIL_SUM]: all
// contributions deeper than RECORDED_VERTS; w[RUN_SUM]: in the tail replay,
// the tail contributions met so far. (One array, indexed at run time, so
// that the sums stay in local memory rather than in registers.)
constexpr int TAIL_SUM = RECORDED_VERTS, RUN_SUM = RECORDED_VERTS + 1;
struct Replay {
    int32_t tri[RECORDED_VERTS];
    V3 w[RECORDED_VERTS + 2];
};

// A path between two bounces: everything the bounce loop carries, so that
// the loop can resume from it.
struct PathPoint {
    V3 ro, rd, thr, prev_p, prev_n;
    float tmin, prev_pdf;
    int k;                    // index of the next bounce
    int nv;                   // surface vertices so far
    bool prev_deg, prev_spec;
};

// Emission gradient of one light summed by a thread; flushed into the
// block's shared sums (lights below SHARED_LIGHTS) or to global memory.
constexpr int SHARED_LIGHTS = 32;
struct EmissionSum {
    int light;
    V3 g;
};

__device__ __forceinline__ void flush_emission(EmissionSum& e, float* s_de, float* d_emission)
{
    if (e.light < 0) return;
    float* dst = e.light < SHARED_LIGHTS ? s_de + 3 * e.light : d_emission + 3 * e.light;
    if (e.g.x != 0.0f) atomicAdd(dst, e.g.x);
    if (e.g.y != 0.0f) atomicAdd(dst + 1, e.g.y);
    if (e.g.z != 0.0f) atomicAdd(dst + 2, e.g.z);
    e.light = -1;
    e.g = v3(0, 0, 0);
}

// One contribution: forward splats it, the adjoint records dL/dI . c for the
// albedos of its prefix (prefix length `depth`) and for its light. In the
// tail replay (`tail`) only contributions deeper than RECORDED_VERTS count,
// into the running sum; their light's gradient was added by the main replay.
template <bool BACKWARD>
__device__ __forceinline__ void contribute(const DiffConsts& c, const DeviceScene& s, Replay& rp, bool tail, int depth,
                                           int light, int pixel, V3 contrib, float* image, const float* dL,
                                           EmissionSum& es, float* s_de, float* d_emission)
{
    if (pixel < 0 || is_zero(contrib)) return;
    if (!BACKWARD) {
        atomicAdd(image + 3 * pixel, contrib.x * c.scale);
        atomicAdd(image + 3 * pixel + 1, contrib.y * c.scale);
        atomicAdd(image + 3 * pixel + 2, contrib.z * c.scale);
        return;
    }
    const V3 w = v3(dL[3 * pixel] * contrib.x, dL[3 * pixel + 1] * contrib.y, dL[3 * pixel + 2] * contrib.z) * c.scale;
    if (is_zero(w)) return;
    if (tail) {
        if (depth > RECORDED_VERTS) rp.w[RUN_SUM] = rp.w[RUN_SUM] + w;
        return;
    }
    if (depth > 0) {
        const int slot = depth > RECORDED_VERTS ? TAIL_SUM : depth - 1;
        rp.w[slot] = rp.w[slot] + w;
    }
    if (light >= 0 && light < s.num_area_lights) {
        const V3 Le = light_Le(s, c, light);
        const V3 g = v3(Le.x != 0.0f ? w.x / Le.x : 0.0f, Le.y != 0.0f ? w.y / Le.y : 0.0f,
                        Le.z != 0.0f ? w.z / Le.z : 0.0f);
        if (es.light != light) flush_emission(es, s_de, d_emission);
        es.light = light;
        es.g = es.g + g;
    }
}

// Adds weight S / R to the albedo gradient of triangle t (diffuse only).
__device__ __forceinline__ void add_albedo_grad(const DiffConsts& c, const DeviceScene& s, int t, V3 S, float* d_albedo)
{
    if (is_zero(S)) return;
    const Material m = diff_material(s, c, t);
    if (m.type != LMGPU_BSDF_DIFFUSE) return;
    if (m.R.x != 0.0f) atomicAdd(d_albedo + 3 * (int64_t)t, S.x / m.R.x);
    if (m.R.y != 0.0f) atomicAdd(d_albedo + 3 * (int64_t)t + 1, S.y / m.R.y);
    if (m.R.z != 0.0f) atomicAdd(d_albedo + 3 * (int64_t)t + 2, S.z / m.R.z);
}

// End of a replayed path: the albedo gradient weight of recorded vertex i is
// the sum of the weights of every contribution whose prefix contains it: the
// suffix sum of the recorded weights plus every deeper contribution.
__device__ __forceinline__ void flush_albedo(const DiffConsts& c, const DeviceScene& s, const Replay& rp, int n,
                                             float* d_albedo)
{
    V3 S = rp.w[TAIL_SUM];
    for (int i = n - 1; i >= 0; i--) {
        S = S + rp.w[i];
        add_albedo_grad(c, s, rp.tri[i], S, d_albedo);
    }
}

// Light sample with the parameterised emission; returns the light index.
__device__ __forceinline__ int sample_light_diff(const DeviceScene& s, const DiffConsts& c, float u0, float u1, LightPoint& lp)
{
    if (!sample_light(s, u0, u1, lp)) return -1;
    const int nl = s.num_lights;
    const int li = min(static_cast<int>(u0 * float(nl)), nl - 1);
    lp.Le = light_Le(s, c, li);
    return li;
}

// Saves the checkpoint. Kept out of line: the copy runs once per deep path,
// and inlined it costs the bounce loop registers (backward 36.6 -> 34.5 ms
// on the refined Cornell box out of line).
__device__ __noinline__ void save_point(PathPoint* dst, const PathPoint& src) { *dst = src; }

// The bounce loop from `pp` until the path ends. TAIL is the adjoint's
// second replay of a deep path's tail; otherwise, in the adjoint, the state
// on arrival at depth RECORDED_VERTS is saved in *ck and *deep set. Both
// instantiations compute the same path from the same state.
template <int TECH, int LAYOUT, int STACK, bool BACKWARD, bool TAIL>
__device__ __forceinline__ void bounce_loop(const DeviceScene& s, const DiffConsts& c, uint64_t key, int path_pixel,
                                            PathPoint& pp, PathPoint* ck, bool* deep, Replay& rp, int2* stack,
                                            float* image, const float* dL, float* d_albedo, EmissionSum& es,
                                            float* s_de, float* d_emission, int32_t* status)
{
    for (;;) {
        if (c.max_pv != -1 && pp.k >= c.max_pv) break;
        if (BACKWARD && !TAIL && pp.nv == RECORDED_VERTS) { save_point(ck, pp); *deep = true; }
        Hit h;
        const int tri = cast_ray<LAYOUT, false, STACK>(s, pp.ro, pp.rd, pp.tmin, FLT_MAX, h, stack, status);
        Geom g;
        const V3 wi = -pp.rd;
        V3 Le = v3(0, 0, 0);
        float lpdf = 0.0f;
        int light = -1;
        bool surface = false;
        Material m;
        m.type = LMGPU_BSDF_BLACK;
        m.R = v3(0, 0, 0);
        if (tri < 0) {
            float t;
            if (!(s.has_env && env_sphere_intersect(s, pp.ro, pp.rd, pp.tmin, FLT_MAX, t))) break;
            env_surface(s, pp.ro, pp.rd, t, g);
            Le = emitted(load3(s.env_Le), g.sn, wi);
            lpdf = s.env_inv_area;
            light = s.num_area_lights;
        } else {
            surface_from_hit(s, tri, h.u, h.v, pp.ro, pp.rd, h.t, g);
            const int li = s.prim_light[s.tri_prim[tri]];
            if (li >= 0) {
                Le = emitted(light_Le(s, c, li), g.sn, wi);
                lpdf = s.area_lights[li].inv_area;
                light = li;
            }
            m = diff_material(s, c, tri);
            surface = true;
            if (pp.nv == MAX_PATH_VERTICES) {
                atomicOr(status, STATUS_QUEUE_OVERFLOW);
                break;
            }
            if (BACKWARD && !TAIL && pp.nv < RECORDED_VERTS) {
                rp.tri[pp.nv] = tri;
                rp.w[pp.nv] = v3(0, 0, 0);
            }
            pp.nv++;
        }
        const int depth_here = pp.nv - (surface ? 1 : 0);
        if (!is_zero(Le)) {
            const V3 contrib = pp.thr * Le;
            if (TECH == LMGPU_RENDER_PT || pp.prev_spec) {
                contribute<BACKWARD>(c, s, rp, TAIL, depth_here, light, path_pixel, contrib, image, dL, es, s_de,
                                     d_emission);
            } else if (TECH == LMGPU_RENDER_PT_MIS) {
                const float G = geometry_term(pp.prev_p, pp.prev_n, pp.prev_deg, g.p, g.sn, false);
                const float pdl = G == 0.0f ? 0.0f : lpdf / (float(s.num_lights) * G);
                contribute<BACKWARD>(c, s, rp, TAIL, depth_here, light, path_pixel,
                                     contrib * (pp.prev_pdf / (pp.prev_pdf + pdl)), image, dL, es, s_de, d_emission);
            }
        }
        if (!surface) break;
        // Tail replay: every tail contribution no deeper than this vertex
        // has been met; the rest have it on their prefix.
        if (BACKWARD && TAIL && pp.nv > RECORDED_VERTS) add_albedo_grad(c, s, tri, rp.w[TAIL_SUM] - rp.w[RUN_SUM], d_albedo);
        const int v = pp.k + 1;
        if (TECH != LMGPU_RENDER_PT && c.max_pv != -1 && v >= c.max_pv) break;
        if (TECH != LMGPU_RENDER_PT && has_non_delta(m.type)) {
            LightPoint lp;
            const int li = sample_light_diff(s, c, rng_uniform(key, dim_vertex(v) + DIM_LIGHT),
                                             rng_uniform(key, dim_vertex(v) + DIM_LIGHT + 1), lp);
            if (li >= 0) {
                const V3 ppL = normalize(lp.p - g.p);
                float pb;
                const V3 fs = eval_bsdf(m, g, wi, ppL, pb);
                const float G = geometry_term(g.p, g.sn, false, lp.p, lp.n, false);
                const V3 Lel = emitted(lp.Le, lp.n, -ppL);
                if (G != 0.0f && !is_zero(fs) && !is_zero(Lel) && visible<LAYOUT, STACK>(s, g.p, lp.p, stack, status)) {
                    float w = 1.0f;
                    if (TECH == LMGPU_RENDER_PT_MIS) { const float pdl = lp.pdf_area / G; w = pdl / (pdl + pb); }
                    contribute<BACKWARD>(c, s, rp, TAIL, pp.nv, li, path_pixel, pp.thr * fs * Lel * (w * G / lp.pdf_area),
                                         image, dL, es, s_de, d_emission);
                }
            }
        }
        const int kv = TECH == LMGPU_RENDER_PT ? pp.k : v;
        if (TECH != LMGPU_RENDER_PT && c.rr_depth != -1 && kv >= c.rr_depth) {
            const float p = fminf(0.5f, luminance(pp.thr));
            if (rng_uniform(key, dim_vertex(kv) + DIM_RR) > p) break;
            pp.thr = pp.thr / p;
        }
        const BsdfSample bs = sample_bsdf(m, g, wi, rng_uniform(key, dim_vertex(kv) + DIM_BSDF),
                                          rng_uniform(key, dim_vertex(kv) + DIM_BSDF + 1),
                                          rng_uniform(key, dim_vertex(kv) + DIM_COMP));
        if (is_zero(bs.weight)) break;
        pp.thr = pp.thr * bs.weight;
        if (TECH == LMGPU_RENDER_PT && c.rr_depth != -1 && pp.k >= c.rr_depth) {
            const float p = fminf(0.5f, luminance(pp.thr));
            if (rng_uniform(key, dim_vertex(pp.k) + DIM_RR) > p) break;
            pp.thr = pp.thr / p;
        }
        if (TECH == LMGPU_RENDER_PT && c.max_pv != -1 && pp.k + 1 >= c.max_pv) break;
        pp.prev_p = g.p; pp.prev_n = g.sn; pp.prev_deg = false; pp.prev_spec = bs.specular; pp.prev_pdf = bs.pdf;
        pp.ro = g.p; pp.rd = bs.wo; pp.tmin = EPS_F;
        pp.k++;
    }
}

template <int TECH, int LAYOUT, int STACK, bool BACKWARD>
// 8 resident blocks per SM (64 registers, some spills): on the refined
// Cornell box, forward / backward 22.2 / 33.1 ms against 24.9 / 36.2 ms at the
// unconstrained 94-96 registers (5 blocks); 6, 10 and 12 blocks were slower
// in total. The passes are latency-bound and gain more from resident warps
// than they lose to spills.
__global__ void __launch_bounds__(128, 8) k_diff(const DeviceScene s, const DiffConsts c, float* image, const float* dL,
                                              float* d_albedo, float* d_emission, int32_t* status)
{
    int2 stack[STACK];
    Replay rp;
    __shared__ float s_de[3 * SHARED_LIGHTS];
    EmissionSum es;
    es.light = -1;
    es.g = v3(0, 0, 0);
    if (BACKWARD) {
        for (int i = threadIdx.x; i < 3 * SHARED_LIGHTS; i += blockDim.x) s_de[i] = 0.0f;
        __syncthreads();
    }
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < c.num_samples; j += stride) {
        const uint64_t sample = (uint64_t)(c.sample_offset + j);
        const uint64_t key = sample_key(c.seed, sample);
        if (BACKWARD) {
            rp.w[TAIL_SUM] = v3(0, 0, 0);
            rp.w[RUN_SUM] = v3(0, 0, 0);
        }
        const float u0 = rng_uniform(key, DIM_RASTER), u1 = rng_uniform(key, DIM_RASTER + 1);
        float rx, ry;
        if (c.sampling == LMGPU_SAMPLING_STRATIFIED) {
            stratified_raster((int64_t)sample, c.pixels, c.inv_pixels, s.cam.width, s.cam.height, u0, u1, rx, ry);
        } else {
            rx = u0; ry = u1;
        }
        const int path_pixel = film_pixel(s.cam, rx, ry);
        float pdf_cam;
        const V3 dir = camera_direction(s.cam, rx, ry, pdf_cam);
        const V3 cp = load3(s.cam.position);
        if (c.max_pv != -1 && c.max_pv <= 1) continue;
        PathPoint pp;
        pp.ro = cp; pp.rd = dir; pp.thr = v3(1, 1, 1);
        pp.prev_p = cp; pp.prev_n = v3(0, 0, 1);
        pp.prev_deg = true; pp.prev_spec = false;
        pp.prev_pdf = pdf_cam;
        pp.tmin = TECH == LMGPU_RENDER_PT ? 0.0f : EPS_F;
        pp.k = 1;
        pp.nv = 0;
        bool alive = true;
        if (TECH != LMGPU_RENDER_PT) {
            LightPoint lp;
            const int li = sample_light_diff(s, c, rng_uniform(key, dim_vertex(1) + DIM_LIGHT),
                                             rng_uniform(key, dim_vertex(1) + DIM_LIGHT + 1), lp);
            if (li >= 0) {
                const V3 ppL = normalize(lp.p - cp);
                float lrx, lry, We;
                if (camera_project(s.cam, cp, ppL, lrx, lry, We) && We > 0.0f) {
                    const float G = geometry_term(cp, v3(0, 0, 1), true, lp.p, lp.n, false);
                    const V3 Le = emitted(lp.Le, lp.n, -ppL);
                    if (G != 0.0f && !is_zero(Le) && visible<LAYOUT, STACK>(s, cp, lp.p, stack, status)) {
                        float w = 1.0f;
                        if (TECH == LMGPU_RENDER_PT_MIS) { const float pdl = lp.pdf_area / G; w = pdl / (pdl + We); }
                        contribute<BACKWARD>(c, s, rp, false, 0, li, film_pixel(s.cam, lrx, lry),
                                             Le * (w * We * G / lp.pdf_area), image, dL, es, s_de, d_emission);
                    }
                }
            }
            if (c.rr_depth != -1 && 1 >= c.rr_depth) {
                const float p = fminf(0.5f, luminance(pp.thr));
                if (rng_uniform(key, dim_vertex(1) + DIM_RR) > p) alive = false;
                else pp.thr = pp.thr / p;
            }
        }
        PathPoint ck;
        bool deep = false;
        if (alive)
            bounce_loop<TECH, LAYOUT, STACK, BACKWARD, false>(s, c, key, path_pixel, pp, &ck, &deep, rp, stack, image, dL,
                                                              d_albedo, es, s_de, d_emission, status);
        if (BACKWARD) {
            flush_albedo(c, s, rp, min(pp.nv, RECORDED_VERTS), d_albedo);
            // The tail of a path deeper than RECORDED_VERTS: replayed from the
            // checkpoint taken on arrival at that depth.
            if (deep)
                bounce_loop<TECH, LAYOUT, STACK, BACKWARD, true>(s, c, key, path_pixel, ck, nullptr, nullptr, rp, stack,
                                                                 image, dL, d_albedo, es, s_de, d_emission, status);
        }
    }
    if (BACKWARD) {
        flush_emission(es, s_de, d_emission);
        __syncthreads();
        const int n = 3 * min(s.num_area_lights, SHARED_LIGHTS);
        for (int i = threadIdx.x; i < n; i += blockDim.x)
            if (s_de[i] != 0.0f) atomicAdd(d_emission + i, s_de[i]);
    }
}

template <int TECH, int LAYOUT, int STACK>
int launch_diff_l(LmgpuScene* sc, const DiffConsts& c, bool backward, float* image, const float* dL, float* da,
                  float* de, cudaStream_t st)
{
    const int64_t blocks = std::max<int64_t>(1, std::min<int64_t>((c.num_samples + 127) / 128, 148 * 16));
    if (backward) k_diff<TECH, LAYOUT, STACK, true><<<blocks, 128, 0, st>>>(sc->rdev, c, image, dL, da, de, sc->d_status);
    else k_diff<TECH, LAYOUT, STACK, false><<<blocks, 128, 0, st>>>(sc->rdev, c, image, dL, da, de, sc->d_status);
    LMGPU_CUDA_TRY(cudaGetLastError());
    return LMGPU_OK;
}

template <int TECH, int STACK>
int launch_diff_s(LmgpuScene* sc, const DiffConsts& c, bool backward, float* image, const float* dL, float* da,
                  float* de, cudaStream_t st)
{
    switch (sc->dev.layout) {
    case LMGPU_LAYOUT_BVH2: return launch_diff_l<TECH, LMGPU_LAYOUT_BVH2, STACK>(sc, c, backward, image, dL, da, de, st);
    case LMGPU_LAYOUT_BVH4: return launch_diff_l<TECH, LMGPU_LAYOUT_BVH4, STACK>(sc, c, backward, image, dL, da, de, st);
    default: return launch_diff_l<TECH, LMGPU_LAYOUT_NAIVE, 1>(sc, c, backward, image, dL, da, de, st);
    }
}

template <int TECH>
int launch_diff_t(LmgpuScene* sc, const DiffConsts& c, bool backward, float* image, const float* dL, float* da,
                  float* de, cudaStream_t st)
{
    const int cap = sc->rdev.stack_cap;
    if (cap <= 32) return launch_diff_s<TECH, 32>(sc, c, backward, image, dL, da, de, st);
    if (cap <= 64) return launch_diff_s<TECH, 64>(sc, c, backward, image, dL, da, de, st);
    if (cap <= 128) return launch_diff_s<TECH, 128>(sc, c, backward, image, dL, da, de, st);
    return fail(LMGPU_ERR_UNSUPPORTED, "BVH too deep for the differentiable path (stack 128)");
}

int launch_diff(LmgpuScene* sc, const LmgpuRenderParams* p, const LmgpuDiffParams* dp, bool backward, float* image,
                const float* dL, float* da, float* de, cudaStream_t st, LmgpuRenderStats* stats)
{
    if (!sc || !p) return fail(LMGPU_ERR_INVALID, "null argument");
    if (const int rc = check_scene_device(sc)) return rc;
    if (!sc->dev.cam.valid) return fail(LMGPU_ERR_INVALID, "scene has no camera");
    if (p->num_samples <= 0) return fail(LMGPU_ERR_INVALID, "num_samples must be positive");
    if (p->sample_offset < 0) return fail(LMGPU_ERR_INVALID, "negative sample offset");
    if (!sample_range_ok(p->sample_offset, p->num_samples)) return fail(LMGPU_ERR_INVALID, "sample indices reach 2^53");
    if (p->technique < LMGPU_RENDER_PT || p->technique > LMGPU_RENDER_PT_MIS) return fail(LMGPU_ERR_INVALID, "unknown technique");
    DiffConsts c;
    std::memset(&c, 0, sizeof(c));
    c.technique = p->technique;
    c.rr_depth = p->rr_depth;
    c.max_pv = p->max_path_vertices;
    c.sampling = p->sampling;
    c.seed = p->seed;
    c.sample_offset = p->sample_offset;
    c.num_samples = p->num_samples;
    c.pixels = (int64_t)sc->dev.cam.width * sc->dev.cam.height;
    c.inv_pixels = 1.0 / double(c.pixels);
    c.scale = float(double(c.pixels) / double(p->num_samples));
    c.albedo = dp ? dp->albedo : nullptr;
    c.emission = dp ? dp->emission : nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (stats) {
        LMGPU_CUDA_TRY(cudaEventCreate(&e0));
        LMGPU_CUDA_TRY(cudaEventCreate(&e1));
        LMGPU_CUDA_TRY(cudaEventRecord(e0, st));
    }
    int rc;
    switch (p->technique) {
    case LMGPU_RENDER_PT: rc = launch_diff_t<LMGPU_RENDER_PT>(sc, c, backward, image, dL, da, de, st); break;
    case LMGPU_RENDER_PT_DIRECT: rc = launch_diff_t<LMGPU_RENDER_PT_DIRECT>(sc, c, backward, image, dL, da, de, st); break;
    default: rc = launch_diff_t<LMGPU_RENDER_PT_MIS>(sc, c, backward, image, dL, da, de, st); break;
    }
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        stats->paths = p->num_samples;
        if (rc == LMGPU_OK) {
            cudaEventRecord(e1, st);
            cudaEventSynchronize(e1);
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, e0, e1);
            stats->device_ms = ms;
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    }
    return rc;
}

}  // namespace
}  // namespace lmgpu

using namespace lmgpu;

extern "C" {

int lmgpu_adjoint_forward(LmgpuScene* scene, const LmgpuRenderParams* params, const LmgpuDiffParams* diff,
                          float* image_device, void* stream, LmgpuRenderStats* stats)
{
    if (!image_device) return fail(LMGPU_ERR_INVALID, "null image");
    return launch_diff(scene, params, diff, false, image_device, nullptr, nullptr, nullptr,
                       static_cast<cudaStream_t>(stream), stats);
}

int lmgpu_adjoint_backward(LmgpuScene* scene, const LmgpuRenderParams* params, const LmgpuDiffParams* diff,
                           const float* dL_dimage_device, float* d_albedo_device, float* d_emission_device,
                           void* stream, LmgpuRenderStats* stats)
{
    if (!dL_dimage_device || !d_albedo_device || !d_emission_device)
        return fail(LMGPU_ERR_INVALID, "null gradient buffer");
    return launch_diff(scene, params, diff, true, nullptr, dL_dimage_device, d_albedo_device, d_emission_device,
                       static_cast<cudaStream_t>(stream), stats);
}

}  // extern "C"
