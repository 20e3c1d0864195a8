// Device-side ray traversal for sm_100a.
//
// Exactness contract: for LMGPU_LAYOUT_BVH2 the closest hit (triangle id, t,
// u, v) is bit-identical to the reference BVHScene::Intersect
// (scene.bvh.cpp:405-473, TriAccel::Intersect triaccel.h:100-160):
//   * same tree (host builder) and the same near-first depth-first order
//     (the right child first iff the ray direction is negative along the
//     node's split axis);
//   * the slab test's maxT-independent part is evaluated when a node is
//     first seen; its `tmin < maxT` part is re-evaluated when the far child is
//     popped, i.e. with the same maxT the recursive reference sees there;
//   * every float operation uses an explicit round-to-nearest intrinsic
//     (__fadd_rn, __fmul_rn, __fdiv_rn, ...), so nvcc cannot fuse them into
//     FMAs and each rounds once, like the reference's float SSE build.
#pragma once
#include <cfloat>
#include <cstdint>
#include "layout.h"

namespace lmgpu {

struct RayIn {
    float o[3], d[3];
    float tmin, tmax;
};

struct TraversalRay {
    float o[3];
    float d[3];
    float inv_min[3];   // 1/d, or 0 where d == 0      (scene.bvh.cpp:124-127)
    float inv_max[3];   // 1/d, or FLT_MAX where d == 0 (scene.bvh.cpp:129-132)
    uint32_t neg;       // bit c set iff d[c] < 0        (scene.bvh.cpp:134-137);
                        // bit 3: finite origin, every d[c] != 0 with a finite 1/d
                        // (RAY_FINITE_INV)
    float tmin, tmax;
};

constexpr uint32_t RAY_FINITE_INV = 8u;

// Render rays (RENDER_SLAB) keep inv_min = 1/d, clamped to +-1e18 so that it
// stays finite, and inv_max = -o/d: a plane distance is then one
// multiply-add, (lo - o)/d = fma(lo, 1/d, -o/d) (slab_render).
#ifndef LMGPU_RENDER_FMA_SLAB
#define LMGPU_RENDER_FMA_SLAB 1
#endif

template <bool RENDER = false>
__device__ __forceinline__ void setup_ray(TraversalRay& r, const RayIn& in)
{
    if (RENDER && LMGPU_RENDER_FMA_SLAB) {
        r.neg = RAY_FINITE_INV;
#pragma unroll
        for (int c = 0; c < 3; c++) {
            r.o[c] = in.o[c];
            r.d[c] = in.d[c];
            float inv = __frcp_rn(in.d[c]);
            if (!(fabsf(inv) <= 1e18f)) inv = copysignf(1e18f, in.d[c]);
            r.inv_min[c] = inv;
            r.inv_max[c] = -(in.o[c] * inv);
            r.neg |= (in.d[c] < 0.0f ? 1u : 0u) << c;
        }
        r.tmin = in.tmin;
        r.tmax = in.tmax;
        return;
    }
    r.neg = RAY_FINITE_INV;
#pragma unroll
    for (int c = 0; c < 3; c++) {
        r.o[c] = in.o[c];
        r.d[c] = in.d[c];
        const bool z = in.d[c] == 0.0f;
        const float inv = __frcp_rn(in.d[c]);  // correctly rounded 1/d == 1.0f/d
        r.inv_min[c] = z ? 0.0f : inv;
        r.inv_max[c] = z ? FLT_MAX : inv;
        r.neg |= (in.d[c] < 0.0f ? 1u : 0u) << c;
        const float inf = __int_as_float(0x7f800000);
        if (z || !(fabsf(inv) < inf) || !(fabsf(in.o[c]) < inf)) r.neg &= ~RAY_FINITE_INV;
    }
    r.tmin = in.tmin;
    r.tmax = in.tmax;
}

// Slab test of one box, split into the maxT-independent verdict (`pass`)
// and the entry distance `t_enter`; the box is hit iff pass && t_enter < maxT.
// lo/hi are the box's per-axis bounds.
__device__ __forceinline__ bool slab_intrinsic(const TraversalRay& r,
                                               float lox, float hix, float loy, float hiy,
                                               float loz, float hiz, float& t_enter)
{
    const float nx = (r.neg & 1u) ? hix : lox, fx = (r.neg & 1u) ? lox : hix;
    const float ny = (r.neg & 2u) ? hiy : loy, fy = (r.neg & 2u) ? loy : hiy;
    const float nz = (r.neg & 4u) ? hiz : loz, fz = (r.neg & 4u) ? loz : hiz;
    float tmin = __fmul_rn(__fsub_rn(nx, r.o[0]), r.inv_min[0]);
    float tmax = __fmul_rn(__fsub_rn(fx, r.o[0]), r.inv_max[0]);
    const float tymin = __fmul_rn(__fsub_rn(ny, r.o[1]), r.inv_min[1]);
    const float tymax = __fmul_rn(__fsub_rn(fy, r.o[1]), r.inv_max[1]);
    if ((tmin > tymax) || (tymin > tmax)) return false;
    if (tymin > tmin) tmin = tymin;
    if (tymax < tmax) tmax = tymax;
    const float tzmin = __fmul_rn(__fsub_rn(nz, r.o[2]), r.inv_min[2]);
    const float tzmax = __fmul_rn(__fsub_rn(fz, r.o[2]), r.inv_max[2]);
    if ((tmin > tzmax) || (tzmin > tmax)) return false;
    if (tzmin > tmin) tmin = tzmin;
    if (tzmax < tmax) tmax = tzmax;
    t_enter = tmin;
    return tmax > r.tmin;
}

// The same slab test for a ray with RAY_FINITE_INV and a box with finite
// lo <= hi on every axis (every binary node's child box). Then inv_min == inv_max,
// the near/far plane distances of an axis are min/max of its two plane
// distances (a float subtraction and multiplication round monotonically),
// no value is NaN, and the reference's pairwise comparison chain fails
// exactly when max(near) > min(far); its final tmin is max(near). The verdict
// and t_enter therefore equal slab_intrinsic's (t_enter up to the sign of a
// zero, which no comparison distinguishes).
#ifndef LMGPU_TRACE_FAST_SLAB
#define LMGPU_TRACE_FAST_SLAB 1
#endif
#ifndef LMGPU_TRACE_F32X2
#define LMGPU_TRACE_F32X2 1
#endif
// (lo - o) * inv and (hi - o) * inv: with LMGPU_TRACE_F32X2 as one packed
// sub.rn.f32x2 and one mul.rn.f32x2 (sm_100), each lane rounded to nearest
// on its own, i.e. the same two results as the scalar __fsub_rn/__fmul_rn.
__device__ __forceinline__ void plane_pair(float lo, float hi, float o, float inv, float& a, float& b)
{
#if LMGPU_TRACE_F32X2
    asm("{\n\t.reg .b64 p, q;\n\t"
        "mov.b64 p, {%2, %3};\n\t"
        "mov.b64 q, {%4, %4};\n\t"
        "sub.rn.f32x2 p, p, q;\n\t"
        "mov.b64 q, {%5, %5};\n\t"
        "mul.rn.f32x2 p, p, q;\n\t"
        "mov.b64 {%0, %1}, p;\n\t}"
        : "=f"(a), "=f"(b) : "f"(lo), "f"(hi), "f"(o), "f"(inv));
#else
    a = __fmul_rn(__fsub_rn(lo, o), inv);
    b = __fmul_rn(__fsub_rn(hi, o), inv);
#endif
}

__device__ __forceinline__ bool slab_finite(const TraversalRay& r,
                                            float lox, float hix, float loy, float hiy,
                                            float loz, float hiz, float& t_enter)
{
    float ax, bx, ay, by, az, bz;
    plane_pair(lox, hix, r.o[0], r.inv_min[0], ax, bx);
    plane_pair(loy, hiy, r.o[1], r.inv_min[1], ay, by);
    plane_pair(loz, hiz, r.o[2], r.inv_min[2], az, bz);
    const float tn = fmaxf(fmaxf(fminf(ax, bx), fminf(ay, by)), fminf(az, bz));
    const float tf = fminf(fminf(fmaxf(ax, bx), fmaxf(ay, by)), fmaxf(az, bz));
    t_enter = tn;
    return tn <= tf && tf > r.tmin;
}

// The slab test of render rays (setup_ray<true>): plane distances by packed
// multiply-adds fma.rn.f32x2 (sm_100), near/far by min/max as slab_finite.
// It rounds differently from the reference's test near box faces, which
// renders (same expected image, not bit-exact hits) tolerate.
__device__ __forceinline__ void plane_pair_fma(float lo, float hi, float inv, float noinv, float& a, float& b)
{
    asm("{\n\t.reg .b64 p, q, r;\n\t"
        "mov.b64 p, {%2, %3};\n\t"
        "mov.b64 q, {%4, %4};\n\t"
        "mov.b64 r, {%5, %5};\n\t"
        "fma.rn.f32x2 p, p, q, r;\n\t"
        "mov.b64 {%0, %1}, p;\n\t}"
        : "=f"(a), "=f"(b) : "f"(lo), "f"(hi), "f"(inv), "f"(noinv));
}

// Entry and exit of a box from its six plane distances (x lo, x hi, y lo, ...).
__device__ __forceinline__ bool slab_interval(const TraversalRay& r, const float* t, float& t_enter)
{
    const float tn = fmaxf(fmaxf(fminf(t[0], t[1]), fminf(t[2], t[3])), fminf(t[4], t[5]));
    const float tf = fminf(fminf(fmaxf(t[0], t[1]), fmaxf(t[2], t[3])), fmaxf(t[4], t[5]));
    t_enter = tn;
    return tn <= tf && tf > r.tmin;
}

__device__ __forceinline__ bool slab_render(const TraversalRay& r,
                                            float lox, float hix, float loy, float hiy,
                                            float loz, float hiz, float& t_enter)
{
    float t[6];
    plane_pair_fma(lox, hix, r.inv_min[0], r.inv_max[0], t[0], t[1]);
    plane_pair_fma(loy, hiy, r.inv_min[1], r.inv_max[1], t[2], t[3]);
    plane_pair_fma(loz, hiz, r.inv_min[2], r.inv_max[2], t[4], t[5]);
    return slab_interval(r, t, t_enter);
}

// Both child boxes of a binary node (render rays or the exact test).
template <bool RENDER>
__device__ __forceinline__ void slab_pair(const TraversalRay& r, float4 bx, float4 by, float4 bz,
                                          bool& pl, float& tl, bool& pr, float& tr)
{
    if (RENDER && LMGPU_RENDER_FMA_SLAB) {
        pl = slab_render(r, bx.x, bx.y, by.x, by.y, bz.x, bz.y, tl);
        pr = slab_render(r, bx.z, bx.w, by.z, by.w, bz.z, bz.w, tr);
    } else if (LMGPU_TRACE_FAST_SLAB && (r.neg & RAY_FINITE_INV)) {
        pl = slab_finite(r, bx.x, bx.y, by.x, by.y, bz.x, bz.y, tl);
        pr = slab_finite(r, bx.z, bx.w, by.z, by.w, bz.z, bz.w, tr);
    } else {
        pl = slab_intrinsic(r, bx.x, bx.y, by.x, by.y, bz.x, bz.y, tl);
        pr = slab_intrinsic(r, bx.z, bx.w, by.z, by.w, bz.z, bz.w, tr);
    }
}

// One box (the root's) for render rays or the exact test.
template <bool RENDER>
__device__ __forceinline__ bool slab_box(const TraversalRay& r, float lox, float hix, float loy, float hiy,
                                         float loz, float hiz, float& t_enter)
{
    if (RENDER && LMGPU_RENDER_FMA_SLAB) return slab_render(r, lox, hix, loy, hiy, loz, hiz, t_enter);
    return slab_intrinsic(r, lox, hix, loy, hiy, loz, hiz, t_enter);
}

// TriAccel::Intersect (triaccel.h:100-160) in the reference's order.
// Returns true on a hit within [mint, maxt]; u, v, t are then valid.
__device__ __forceinline__ bool triaccel_intersect(const float4 q0, const float4 q1, const float4 q2,
                                                   const TraversalRay& r, float maxt,
                                                   float& u, float& v, float& t)
{
    const uint32_t k = __float_as_uint(q0.x) & TRI_AXIS_MASK;
    if (k == 3u) return false;
    // (u, v, k) axis permutation: k=0 -> (1,2,0), k=1 -> (2,0,1), k=2 -> (0,1,2)
    const float o_u = k == 0 ? r.o[1] : (k == 1 ? r.o[2] : r.o[0]);
    const float o_v = k == 0 ? r.o[2] : (k == 1 ? r.o[0] : r.o[1]);
    const float o_k = k == 0 ? r.o[0] : (k == 1 ? r.o[1] : r.o[2]);
    const float d_u = k == 0 ? r.d[1] : (k == 1 ? r.d[2] : r.d[0]);
    const float d_v = k == 0 ? r.d[2] : (k == 1 ? r.d[0] : r.d[1]);
    const float d_k = k == 0 ? r.d[0] : (k == 1 ? r.d[1] : r.d[2]);
    const float n_u = q0.y, n_v = q0.z, n_d = q0.w;
    const float a_u = q1.x, a_v = q1.y, b_nu = q1.z, b_nv = q1.w;
    const float c_nu = q2.x, c_nv = q2.y;
    float num = __fsub_rn(n_d, __fmul_rn(o_u, n_u));
    num = __fsub_rn(num, __fmul_rn(o_v, n_v));
    num = __fsub_rn(num, o_k);
    float den = __fadd_rn(__fmul_rn(d_u, n_u), __fmul_rn(d_v, n_v));
    den = __fadd_rn(den, d_k);
    t = __fdiv_rn(num, den);
    if (t < r.tmin || t > maxt) return false;
    const float hu = __fsub_rn(__fadd_rn(o_u, __fmul_rn(t, d_u)), a_u);
    const float hv = __fsub_rn(__fadd_rn(o_v, __fmul_rn(t, d_v)), a_v);
    u = __fadd_rn(__fmul_rn(hv, b_nu), __fmul_rn(hu, b_nv));
    v = __fadd_rn(__fmul_rn(hu, c_nu), __fmul_rn(hv, c_nv));
    return u >= 0.0f && v >= 0.0f && __fadd_rn(u, v) <= 1.0f;
}

// The same TriAccel test for renders, which need the same expected image,
// not bit-identical hits: multiply-adds and an approximate division
// (div.approx: a reciprocal and a multiply) in place of the separately
// rounded products and the correctly rounded division. Hits may differ
// from the exact test's only within rounding of the edges and of t.
__device__ __forceinline__ bool triaccel_intersect_fast(const float4 q0, const float4 q1, const float4 q2,
                                                        const TraversalRay& r, float maxt,
                                                        float& u, float& v, float& t)
{
    const uint32_t k = __float_as_uint(q0.x) & TRI_AXIS_MASK;
    if (k == 3u) return false;
    const float o_u = k == 0 ? r.o[1] : (k == 1 ? r.o[2] : r.o[0]);
    const float o_v = k == 0 ? r.o[2] : (k == 1 ? r.o[0] : r.o[1]);
    const float o_k = k == 0 ? r.o[0] : (k == 1 ? r.o[1] : r.o[2]);
    const float d_u = k == 0 ? r.d[1] : (k == 1 ? r.d[2] : r.d[0]);
    const float d_v = k == 0 ? r.d[2] : (k == 1 ? r.d[0] : r.d[1]);
    const float d_k = k == 0 ? r.d[0] : (k == 1 ? r.d[1] : r.d[2]);
    const float num = __fmaf_rn(-o_v, q0.z, __fmaf_rn(-o_u, q0.y, q0.w)) - o_k;
    const float den = __fmaf_rn(d_v, q0.z, __fmaf_rn(d_u, q0.y, d_k));
    t = __fdividef(num, den);
    if (!(t >= r.tmin && t <= maxt)) return false;
    const float hu = __fmaf_rn(t, d_u, o_u) - q1.x;
    const float hv = __fmaf_rn(t, d_v, o_v) - q1.y;
    u = __fmaf_rn(hv, q1.z, hu * q1.w);
    v = __fmaf_rn(hu, q2.x, hv * q2.y);
    return u >= 0.0f && v >= 0.0f && u + v <= 1.0f;
}

struct Hit {
    int32_t tri;   // reference TriAccel index, -1 = miss
    float t, u, v;
};

struct TraceStats {
    uint32_t nodes;   // binary-node slab tests (reference count)
    uint32_t tris;    // TriAccel tests
};

// Leaf loop: every record of the leaf is tested against the running maxT;
// a hit sets maxT = t so later records need t <= new maxT (scene.bvh.cpp:416-427).
// FAST selects triaccel_intersect_fast (render rays); otherwise the
// reference's exact test.
#ifndef LMGPU_RENDER_FAST_TRI
#define LMGPU_RENDER_FAST_TRI 1
#endif
template <bool ANY_HIT, bool FAST = false>
__device__ __forceinline__ bool trace_leaf(const TriRecord* __restrict__ tris, int32_t first,
                                           TraversalRay& r, Hit& h, TraceStats* st)
{
    const float4* p = reinterpret_cast<const float4*>(tris + first);
    for (;;) {
        const float4 q0 = __ldg(p), q1 = __ldg(p + 1), q2 = __ldg(p + 2);
        if (st) st->tris++;
        float u, v, t;
        if ((FAST && LMGPU_RENDER_FAST_TRI) ? triaccel_intersect_fast(q0, q1, q2, r, r.tmax, u, v, t)
                                            : triaccel_intersect(q0, q1, q2, r, r.tmax, u, v, t)) {
            r.tmax = t;
            h.tri = static_cast<int32_t>(__float_as_uint(q2.z));
            h.t = t; h.u = u; h.v = v;
            if (ANY_HIT) return true;
        }
        if (__float_as_uint(q0.x) & TRI_LAST_IN_LEAF) break;
        p += 3;
    }
    return false;
}

// Resumable traversal state: the current reference (internal node >= 0,
// leaf < 0, or REF_DONE) and the deferred far children.
constexpr int32_t REF_DONE = 0x7fffffff;

struct TravState {
    int32_t ref;
    int sp;
};

// Traversal stack storage: a per-thread array (local memory), or a split
// stack whose first S entries live in shared memory ([S][128] per block of
// 128 threads: lanes hit distinct banks) and the rest in local memory, so
// the stack's bottom no longer competes with tree nodes for L1.
__device__ __forceinline__ void stack_put(int2* s, int i, int2 v) { s[i] = v; }
__device__ __forceinline__ int2 stack_get(const int2* s, int i) { return s[i]; }

template <int S>
struct SplitStack {
    int2 (*sh)[128];
    int2* local;
};
template <int S>
__device__ __forceinline__ void stack_put(const SplitStack<S>& s, int i, int2 v)
{
    if (i < S) s.sh[i][threadIdx.x] = v;
    else s.local[i - S] = v;
}
template <int S>
__device__ __forceinline__ int2 stack_get(const SplitStack<S>& s, int i)
{
    return i < S ? s.sh[i][threadIdx.x] : s.local[i - S];
}

// Pops the next deferred child whose box is still entered before maxT
// (the reference's far-child test, evaluated with the current maxT).
template <class Stack>
__device__ __forceinline__ void pop_next(TravState& ts, Stack stack, const TraversalRay& r, TraceStats* st)
{
    while (ts.sp > 0) {
        const int2 e = stack_get(stack, --ts.sp);
        if (st) st->nodes++;
        if (__int_as_float(e.y) < r.tmax) { ts.ref = e.x; return; }
    }
    ts.ref = REF_DONE;
}

// Root box test (the reference tests every node's own box on entry).
template <bool RENDER = false>
__device__ __forceinline__ void trav_begin(TravState& ts, int32_t root_ref, const float* root_box,
                                           const TraversalRay& r, TraceStats* st)
{
    ts.sp = 0;
    float te;
    if (st) st->nodes++;
    ts.ref = (slab_box<RENDER>(r, root_box[0], root_box[3], root_box[1], root_box[4], root_box[2], root_box[5], te) &&
              te < r.tmax) ? root_ref : REF_DONE;
}

// Binary children-in-parent nodes: descends until the state reaches a leaf
// or finishes. Returns false on stack overflow. With EXIT_BELOW > 0 and
// `may_exit`, it also returns (state intact, at an internal node) once fewer
// than EXIT_BELOW lanes of the warp are still descending, after at least one
// step: the caller resumes it later, so the ray's walk is unchanged.
// Speculative descent (SPEC, render rays of the persistent kernel): a lane
// that reaches a leaf while it holds none postpones it (*pend) and goes on
// with its next deferred node, so it keeps descending with the rest of the
// warp; the descent ends once every lane still descending holds a leaf (or
// by the pause rule). The caller tests the postponed leaf first. Every leaf
// is still tested against the current maxT, so a closest hit is as close;
// the walk may visit nodes that the postponed leaf's hit would have culled.
// LMGPU_TRACE_SPECULATIVE: 0 off; 1 visibility (any-hit) walks, whose
// verdict does not depend on the order of leaf tests; 2 closest-hit walks
// too. On the terrain frame and the 64-scene batch, 1 took the shadow-ray
// traversal from 47.8 to 45.3 ms and from 113.1 to 105.6 ms; 2 made the
// bounce-ray traversal 1 % slower, and between triangles hit at exactly the
// same distance the one found first, hence the hit, then depends on when
// the warp's other rays break the descent.
#ifndef LMGPU_TRACE_SPECULATIVE
#define LMGPU_TRACE_SPECULATIVE 1
#endif

// Slab tests of both children of binary node `ref`: pass bits and entry
// distances (left: pl, tl; right: pr, tr); returns (left, right, split axis).
template <bool RENDER>
__device__ __forceinline__ int3 node_children(const Bvh2Node* __restrict__ nodes, int32_t ref, const TraversalRay& r,
                                              bool& pl, float& tl, bool& pr, float& tr)
{
    const float4* np = reinterpret_cast<const float4*>(nodes + ref);
    const float4 bx = __ldg(np), by = __ldg(np + 1), bz = __ldg(np + 2);
    const int4 meta = __ldg(reinterpret_cast<const int4*>(np + 3));
    slab_pair<RENDER>(r, bx, by, bz, pl, tl, pr, tr);
    return make_int3(meta.x, meta.y, meta.z);
}

// The same for a quantised node (render rays). A plane at grid index q of
// axis k lies at origin_k + q * step_k, so its distance along the ray is
// q * (step_k / d_k) + (origin_k - o_k) / d_k: one multiply-add per plane,
// two planes per packed fma.rn.f32x2 as in slab_render. q becomes a float
// as 2^23 + q (its 16 bits under the exponent of 2^23, one byte permute);
// the 2^23 * step_k / d_k this adds is taken off the per-axis bias. That
// subtraction rounds at about half a grid step along the axis, inside the
// two-step margin quantize_bvh2 leaves around every box.
__device__ __forceinline__ float grid_plane(uint32_t word, bool hi)
{
    return __uint_as_float(__byte_perm(word, 0x4b00u, hi ? 0x5432u : 0x5410u));
}
template <bool RENDER>
__device__ __forceinline__ int3 node_children(const Bvh2QNode* __restrict__ nodes, int32_t ref, const TraversalRay& r,
                                              bool& pl, float& tl, bool& pr, float& tr)
{
    static_assert(RENDER && LMGPU_RENDER_FMA_SLAB, "quantised nodes serve render rays only");
    const uint4* np = reinterpret_cast<const uint4*>(nodes + ref);
    const uint4 a = __ldg(np), b = __ldg(np + 1), c = __ldg(np + 2);
    const uint32_t words[6] = { b.x, b.y, b.z, b.w, c.x, c.y };
    const float origin[3] = { __uint_as_float(a.x), __uint_as_float(a.y), __uint_as_float(a.z) };
    float t[2][6];   // [child][lo/hi of x, y, z]
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const float step = __uint_as_float(((a.w >> (8 * k)) & 0xffu) << 23);
        const float s = step * r.inv_min[k];
        const float bias = fmaf(-8388608.0f, s, fmaf(origin[k], r.inv_min[k], r.inv_max[k]));
#pragma unroll
        for (int ch = 0; ch < 2; ch++) {
            const uint32_t w = words[2 * k + ch];
            plane_pair_fma(grid_plane(w, false), grid_plane(w, true), s, bias, t[ch][2 * k], t[ch][2 * k + 1]);
        }
    }
    pl = slab_interval(r, t[0], tl);
    pr = slab_interval(r, t[1], tr);
    return make_int3((int)c.z, (int)c.w, (int)(a.w >> 24));
}

// Child order of render walks: LMGPU_RENDER_NEAR_FIRST 1 visits the child
// with the nearer entry distance first; 0 the reference's order (right
// child first iff the ray points down the split axis), which the exact
// walks keep. LMGPU_RENDER_ANY_NEAR_FIRST: the same for visibility walks,
// whose verdict does not depend on the order. A ray's walk still depends on
// the ray alone. On the 1080p terrain frame the bounce-ray traversal went
// from 89.1 to 86.4 ms (the order is decided from the two pass bits, with
// fewer branches) and the shadow traversal from 44.2 to 42.8 ms; on the
// 64-scene batch from 500.3 / 105.5 to 497.0 / 99.7 ms.
#ifndef LMGPU_RENDER_NEAR_FIRST
#define LMGPU_RENDER_NEAR_FIRST 1
#endif
#ifndef LMGPU_RENDER_ANY_NEAR_FIRST
#define LMGPU_RENDER_ANY_NEAR_FIRST 1
#endif

template <int EXIT_BELOW = 0, bool RENDER = false, bool SPEC = false, class Node, class Stack>
__device__ __forceinline__ bool bvh2_descend(const Node* __restrict__ nodes, TravState& ts, Stack stack,
                                             int stack_cap, const TraversalRay& r, TraceStats* st,
                                             bool may_exit = false, int32_t* pend = nullptr)
{
    bool stepped = false;
    for (;;) {
        if (SPEC && ts.ref < 0 && *pend == 0) {     // a leaf: postpone it, go on with the next deferred node
            *pend = ts.ref;
            pop_next(ts, stack, r, st);
        }
        if (!(ts.ref >= 0 && ts.ref != REF_DONE)) break;
        if (SPEC && __all_sync(__activemask(), *pend != 0)) break;
        if (EXIT_BELOW > 0 && may_exit && stepped && __popc(__activemask()) < EXIT_BELOW) break;
        stepped = true;
        float tl = 0.f, tr = 0.f;
        bool pl, pr;
        const int3 meta = node_children<RENDER>(nodes, ts.ref, r, pl, tl, pr, tr);
        const bool right_first = (RENDER && LMGPU_RENDER_NEAR_FIRST) ? (pr && (!pl || tr < tl))
                                                                     : bool((r.neg >> meta.z) & 1u);
        const int32_t near_ref = right_first ? meta.y : meta.x;
        const int32_t far_ref = right_first ? meta.x : meta.y;
        const bool near_pass = right_first ? pr : pl;
        const bool far_pass = right_first ? pl : pr;
        const float near_t = right_first ? tr : tl;
        const float far_t = right_first ? tl : tr;
        if (st) st->nodes++;                         // near child's slab test
        if (near_pass && near_t < r.tmax) {
            if (far_pass) {
                if (ts.sp >= stack_cap) return false;
                stack_put(stack, ts.sp++, make_int2(far_ref, __float_as_int(far_t)));
            } else if (st) {
                st->nodes++;                         // far child's (failing) test
            }
            ts.ref = near_ref;
            continue;
        }
        if (st) st->nodes++;                         // far child's test, same maxT
        if (far_pass && far_t < r.tmax) { ts.ref = far_ref; continue; }
        pop_next(ts, stack, r, st);
    }
    return true;
}

// Closest hit (or any hit) through the binary children-in-parent BVH.
// `stack` is per-thread scratch of `stack_cap` (ref, t_enter) pairs.
// Returns false if the stack bound was exceeded (the caller flags an error).
// RENDER: a render ray (setup_ray<true>) with the renders' arithmetic.
template <bool ANY_HIT, bool RENDER = false>
__device__ __forceinline__ bool trace_bvh2(const Bvh2Node* __restrict__ nodes,
                                           const TriRecord* __restrict__ tris,
                                           int32_t root_ref, const float* root_box,
                                           TraversalRay& r, Hit& h, int2* stack, int stack_cap,
                                           TraceStats* st)
{
    h.tri = -1;
    TravState ts;
    trav_begin<RENDER>(ts, root_ref, root_box, r, st);
    for (;;) {
        if (!bvh2_descend<0, RENDER>(nodes, ts, stack, stack_cap, r, st)) return false;
        if (ts.ref == REF_DONE) return true;
        if (trace_leaf<ANY_HIT, RENDER>(tris, ~ts.ref, r, h, st) && ANY_HIT) return true;
        pop_next(ts, stack, r, st);
    }
}

// ---------------------------------------------------------------- any hit
// Visibility queries (shadow rays) stop at their first hit, so their maxT
// never changes while they walk: a far child can be tested against maxT
// when it is pushed instead of when it is popped. The stack then holds
// node references only (4 bytes), and a pop needs no test. Every box test
// uses the same arithmetic and the same maxT as the closest-hit walk's, so
// the walk reaches a hit exactly when the closest-hit walk would find one:
// the visibility verdict is the same.
#ifndef LMGPU_TRACE_ANYHIT_WALK
#define LMGPU_TRACE_ANYHIT_WALK 1     // 0: visibility queries take the closest-hit walk
#endif
__device__ __forceinline__ void ref_put(int* s, int i, int v) { s[i] = v; }
__device__ __forceinline__ int ref_get(const int* s, int i) { return s[i]; }

template <int S>
struct SplitRefStack {
    int (*sh)[128];
    int* local;
};
template <int S>
__device__ __forceinline__ void ref_put(const SplitRefStack<S>& s, int i, int v)
{
    if (i < S) s.sh[i][threadIdx.x] = v;
    else s.local[i - S] = v;
}
template <int S>
__device__ __forceinline__ int ref_get(const SplitRefStack<S>& s, int i)
{
    return i < S ? s.sh[i][threadIdx.x] : s.local[i - S];
}

template <class Stack>
__device__ __forceinline__ void pop_any(TravState& ts, Stack stack)
{
    ts.ref = ts.sp > 0 ? ref_get(stack, --ts.sp) : REF_DONE;
}

// Any-hit descent through the binary nodes (exact walks: the right child
// first iff the ray direction is negative on the split axis; render walks:
// LMGPU_RENDER_ANY_NEAR_FIRST). Returns false on stack overflow;
// EXIT_BELOW / may_exit as in bvh2_descend.
template <int EXIT_BELOW = 0, bool RENDER = false, bool SPEC = false, class Node, class Stack>
__device__ __forceinline__ bool bvh2_descend_any(const Node* __restrict__ nodes, TravState& ts, Stack stack,
                                                 int stack_cap, const TraversalRay& r, TraceStats* st,
                                                 bool may_exit = false, int32_t* pend = nullptr)
{
    bool stepped = false;
    for (;;) {
        if (SPEC && ts.ref < 0 && *pend == 0) {     // postpone the leaf (bvh2_descend's SPEC)
            *pend = ts.ref;
            pop_any(ts, stack);
        }
        if (!(ts.ref >= 0 && ts.ref != REF_DONE)) break;
        if (SPEC && __all_sync(__activemask(), *pend != 0)) break;
        if (EXIT_BELOW > 0 && may_exit && stepped && __popc(__activemask()) < EXIT_BELOW) break;
        stepped = true;
        float tl = 0.f, tr = 0.f;
        bool pl, pr;
        const int3 meta = node_children<RENDER>(nodes, ts.ref, r, pl, tl, pr, tr);
        if (st) st->nodes += 2;
        const bool hl = pl && tl < r.tmax, hr = pr && tr < r.tmax;
        if (hl && hr) {
            const bool right_first = (RENDER && LMGPU_RENDER_ANY_NEAR_FIRST) ? tr < tl : bool((r.neg >> meta.z) & 1u);
            if (ts.sp >= stack_cap) return false;
            ref_put(stack, ts.sp++, right_first ? meta.x : meta.y);
            ts.ref = right_first ? meta.y : meta.x;
        } else if (hl || hr) {
            ts.ref = hl ? meta.x : meta.y;
        } else {
            pop_any(ts, stack);
        }
    }
    return true;
}

// Any hit through the binary nodes with a per-thread reference stack of
// `stack_cap` entries; h.tri >= 0 iff some triangle is hit in [tmin, tmax].
template <bool RENDER>
__device__ __forceinline__ bool trace_bvh2_any(const Bvh2Node* __restrict__ nodes, const TriRecord* __restrict__ tris,
                                               int32_t root_ref, const float* root_box, TraversalRay& r, Hit& h,
                                               int* stack, int stack_cap, TraceStats* st)
{
    h.tri = -1;
    TravState ts;
    trav_begin<RENDER>(ts, root_ref, root_box, r, st);
    for (;;) {
        if (!bvh2_descend_any<0, RENDER>(nodes, ts, stack, stack_cap, r, st)) return false;
        if (ts.ref == REF_DONE) return true;
        if (trace_leaf<true, RENDER>(tris, ~ts.ref, r, h, st)) return true;
        pop_any(ts, stack);
    }
}

// Brute force over all records in TriAccel order (reference scene.naive.cpp:98-121).
template <bool ANY_HIT>
__device__ __forceinline__ void trace_naive(const TriRecord* __restrict__ tris_in_id_order, int64_t n,
                                            TraversalRay& r, Hit& h, TraceStats* st)
{
    h.tri = -1;
    const float4* p = reinterpret_cast<const float4*>(tris_in_id_order);
    for (int64_t i = 0; i < n; i++, p += 3) {
        const float4 q0 = __ldg(p), q1 = __ldg(p + 1), q2 = __ldg(p + 2);
        if (st) st->tris++;
        float u, v, t;
        if (triaccel_intersect(q0, q1, q2, r, r.tmax, u, v, t)) {
            r.tmax = t;
            h.tri = static_cast<int32_t>(__float_as_uint(q2.z));
            h.t = t; h.u = u; h.v = v;
            if (ANY_HIT) return;
        }
    }
}

}  // namespace lmgpu
