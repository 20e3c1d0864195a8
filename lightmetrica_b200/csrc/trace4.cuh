// 4-wide traversal of the collapsed reference tree (LMGPU_LAYOUT_BVH4).
//
// Exact by construction, like the binary traversal: a 4-node holds the
// grandchildren of one binary node and the kernel visits them in the
// reference's depth-first order for this ray (recovered from the three stored
// split axes). The skipped intermediate boxes never change a decision: the
// float slab test is monotone under box containment (every subtraction and
// multiplication rounds monotonically and a parent's box is the exact min/max
// union of its children's), so whenever a grandchild's box is entered before
// maxT its parent's box is too.
#pragma once
#include "trace.cuh"

namespace lmgpu {

// 4-wide nodes: descends until the state reaches a leaf or finishes.
// Returns false on stack overflow. EXIT_BELOW / may_exit as in bvh2_descend.
template <int EXIT_BELOW = 0, bool RENDER = false, class Stack>
__device__ __forceinline__ bool bvh4_descend(const Bvh4Node* __restrict__ nodes, TravState& ts, Stack stack,
                                             int stack_cap, const TraversalRay& r, TraceStats* st,
                                             bool may_exit = false)
{
    bool stepped = false;
    while (ts.ref >= 0 && ts.ref != REF_DONE) {
        if (EXIT_BELOW > 0 && may_exit && stepped && __popc(__activemask()) < EXIT_BELOW) break;
        stepped = true;
        const float4* np = reinterpret_cast<const float4*>(nodes + ts.ref);
        const float4 lox = __ldg(np + 0), hix = __ldg(np + 1);
        const float4 loy = __ldg(np + 2), hiy = __ldg(np + 3);
        const float4 loz = __ldg(np + 4), hiz = __ldg(np + 5);
        const int4 child = __ldg(reinterpret_cast<const int4*>(np + 6));
        const int4 axes = __ldg(reinterpret_cast<const int4*>(np + 7));
        float t0 = 0.f, t1 = 0.f, t2 = 0.f, t3 = 0.f;
        // Empty slots hold lo > hi on every axis, which the exact test
        // rejects; the render test's min/max form does not, so their
        // reference (BVH4_EMPTY) excludes them below.
        const bool p0 = slab_box<RENDER>(r, lox.x, hix.x, loy.x, hiy.x, loz.x, hiz.x, t0);
        const bool p1 = slab_box<RENDER>(r, lox.y, hix.y, loy.y, hiy.y, loz.y, hiz.y, t1);
        const bool p2 = slab_box<RENDER>(r, lox.z, hix.z, loy.z, hiy.z, loz.z, hiz.z, t2);
        const bool p3 = slab_box<RENDER>(r, lox.w, hix.w, loy.w, hiy.w, loz.w, hiz.w, t3);
        if (st) st->nodes += 4;
        // Visit order, 4 bits per slot.
        uint32_t order = 0;
        int cnt = 0;
        const int first_pair = (r.neg >> axes.x) & 1u;
#pragma unroll
        for (int q = 0; q < 2; q++) {
            const int p = q == 0 ? first_pair : 1 - first_pair;
            const int a = p == 0 ? axes.y : axes.z;
            if (a < 0) {
                order |= uint32_t(2 * p) << (4 * cnt); cnt++;
            } else {
                const bool sw = (r.neg >> a) & 1u;
                order |= uint32_t(sw ? 2 * p + 1 : 2 * p) << (4 * cnt); cnt++;
                order |= uint32_t(sw ? 2 * p : 2 * p + 1) << (4 * cnt); cnt++;
            }
        }
        // Passing children in visit order; the first one entered before maxT
        // is descended now (same maxT as the reference), later ones are
        // deferred with their entry distance.
        int32_t refs[4];
        float ts4[4];
        int np_ = 0;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            if (j < cnt) {
                const uint32_t sl = (order >> (4 * j)) & 0xFu;
                const bool ps = sl == 0 ? p0 : sl == 1 ? p1 : sl == 2 ? p2 : p3;
                const float tt = sl == 0 ? t0 : sl == 1 ? t1 : sl == 2 ? t2 : t3;
                const int32_t cr = sl == 0 ? child.x : sl == 1 ? child.y : sl == 2 ? child.z : child.w;
                if (ps && cr != BVH4_EMPTY) { refs[np_] = cr; ts4[np_] = tt; np_++; }
            }
        }
        int first = -1;
#pragma unroll
        for (int j = 0; j < 4; j++)
            if (first < 0 && j < np_ && ts4[j] < r.tmax) first = j;
        if (first >= 0) {
            if (ts.sp + (np_ - 1 - first) > stack_cap) return false;
#pragma unroll
            for (int j = 3; j >= 0; j--)
                if (j > first && j < np_) stack_put(stack, ts.sp++, make_int2(refs[j], __float_as_int(ts4[j])));
            ts.ref = refs[first];
            continue;
        }
        pop_next(ts, stack, r, nullptr);
    }
    return true;
}

template <bool ANY_HIT, bool RENDER = false>
__device__ __forceinline__ bool trace_bvh4(const Bvh4Node* __restrict__ nodes,
                                           const TriRecord* __restrict__ tris,
                                           int32_t root_ref, const float* root_box,
                                           TraversalRay& r, Hit& h, int2* stack, int stack_cap,
                                           TraceStats* st)
{
    h.tri = -1;
    TravState ts;
    trav_begin<RENDER>(ts, root_ref, root_box, r, st);
    for (;;) {
        if (!bvh4_descend<0, RENDER>(nodes, ts, stack, stack_cap, r, st)) return false;
        if (ts.ref == REF_DONE) return true;
        if (trace_leaf<ANY_HIT, RENDER>(tris, ~ts.ref, r, h, st) && ANY_HIT) return true;
        pop_next(ts, stack, r, nullptr);
    }
}

}  // namespace lmgpu
