// Persistent traversal kernel shared by the intersection API and the path
// tracer's ray and shadow queues. The I/O policy supplies the ray count, the
// rays and what to do with each result.
#pragma once
#include <cuda_runtime.h>
#include <algorithm>
#include <mutex>
#include <type_traits>
#include <unordered_map>
#include "internal.h"
#include "trace.cuh"
#include "trace4.cuh"

namespace lmgpu {

// Scheduling constants of the persistent traversal kernel. They change only
// when lanes take new rays and when a descent pauses, never a ray's walk.
#ifndef LMGPU_TRACE_REFILL_MIN
#define LMGPU_TRACE_REFILL_MIN 8      // idle lanes that trigger a refill
#endif
#ifndef LMGPU_TRACE_EXIT_BELOW
#define LMGPU_TRACE_EXIT_BELOW 24     // pause a descent when fewer lanes descend (0: never)
#endif
#ifndef LMGPU_TRACE_MIN_BLOCKS
#define LMGPU_TRACE_MIN_BLOCKS 10     // minimum resident blocks of 128 threads per SM (48 registers)
#endif
// Rays of many scenes keep their scene's node and triangle pointers per lane:
// at 10 blocks (48 registers) that spilled, at 9 (56 registers) it does not,
// and the 64-scene batch ran 939 -> 897 ms (8 blocks: 926 ms).
#ifndef LMGPU_TRACE_TABLE_MIN_BLOCKS
#define LMGPU_TRACE_TABLE_MIN_BLOCKS 9
#endif
#ifndef LMGPU_TRACE_API_MIN_BLOCKS
#define LMGPU_TRACE_API_MIN_BLOCKS 9   // intersection API: 2^24-ray soup 2,776 -> 2,837 Mrays/s against 10
#endif
#ifndef LMGPU_TRACE_SHARED_STACK
#define LMGPU_TRACE_SHARED_STACK 12   // stack entries per lane kept in shared memory (0: none)
#endif

// I/O policies whose rays each belong to their own scene (a multi-scene
// batch) declare PER_RAY_SCENE = true and supply ray_scene(j).
template <class IO, class = void>
struct per_ray_scene : std::false_type {};
template <class IO>
struct per_ray_scene<IO, std::void_t<decltype(IO::PER_RAY_SCENE)>> : std::bool_constant<IO::PER_RAY_SCENE> {};

// Idle lanes that trigger a refill: an I/O policy may declare its own
// REFILL_MIN (the path tracer's queues gather each ray through an index, so
// they refill in larger groups); the default suits rays read in order.
template <class IO, class = void>
struct refill_min : std::integral_constant<int, LMGPU_TRACE_REFILL_MIN> {};
template <class IO>
struct refill_min<IO, std::void_t<decltype(IO::REFILL_MIN)>> : std::integral_constant<int, IO::REFILL_MIN> {};

// Resident blocks of 128 threads per SM the kernel is bounded to (its
// register budget): an I/O policy may declare MIN_BLOCKS; rays of many
// scenes default to LMGPU_TRACE_TABLE_MIN_BLOCKS.
template <class IO, class = void>
struct min_blocks
    : std::integral_constant<int, per_ray_scene<IO>::value ? LMGPU_TRACE_TABLE_MIN_BLOCKS : LMGPU_TRACE_MIN_BLOCKS> {};
template <class IO>
struct min_blocks<IO, std::void_t<decltype(IO::MIN_BLOCKS)>> : std::integral_constant<int, IO::MIN_BLOCKS> {};

// Render rays (the path tracer's queues) declare RENDER = true: their
// triangle tests take triaccel_intersect_fast; the intersection API keeps
// the reference's exact arithmetic.
template <class IO, class = void>
struct render_rays : std::false_type {};
template <class IO>
struct render_rays<IO, std::void_t<decltype(IO::RENDER)>> : std::bool_constant<IO::RENDER> {};

// Pause threshold of a descent: an I/O policy may declare EXIT_BELOW.
template <class IO, class = void>
struct exit_below : std::integral_constant<int, LMGPU_TRACE_EXIT_BELOW> {};
template <class IO>
struct exit_below<IO, std::void_t<decltype(IO::EXIT_BELOW)>> : std::integral_constant<int, IO::EXIT_BELOW> {};

// Node and triangle arrays of the scene a lane is tracing.
struct LaneScene {
    const Bvh2Node* bvh2;
    const Bvh4Node* bvh4;
    const Bvh2QNode* bvh2q;
    const TriRecord* tris;
};


template <int LAYOUT, int EXIT, bool RENDER, bool SPEC, class Stack>
__device__ __forceinline__ bool descend(const LaneScene& s, TravState& ts, Stack stack, int cap,
                                        const TraversalRay& r, bool may_exit, TraceStats* st, int32_t* pend)
{
    if constexpr (LAYOUT == LMGPU_LAYOUT_BVH2)
        return bvh2_descend<EXIT, RENDER, SPEC>(s.bvh2, ts, stack, cap, r, st, may_exit, pend);
    else if constexpr (LAYOUT == LMGPU_LAYOUT_BVH2Q)
        return bvh2_descend<EXIT, RENDER, SPEC>(s.bvh2q, ts, stack, cap, r, st, may_exit, pend);
    else
        return bvh4_descend<EXIT, RENDER>(s.bvh4, ts, stack, cap, r, st, may_exit);
}

// Binary layouts (float or quantised nodes) share the walks and stacks.
constexpr bool binary_layout(int layout) { return layout == LMGPU_LAYOUT_BVH2 || layout == LMGPU_LAYOUT_BVH2Q; }

// Adds each lane's counts to counts[0] (binary-node slab tests; four per
// 4-wide node) and counts[1] (TriAccel tests); the whole warp calls it.
__device__ __forceinline__ void add_trace_stats(const TraceStats& st, unsigned long long* counts)
{
    unsigned long long a = st.nodes, b = st.tris;
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, o);
        b += __shfl_down_sync(0xffffffffu, b, o);
    }
    if ((threadIdx.x & 31u) == 0) { atomicAdd(counts, a); atomicAdd(counts + 1, b); }
}

// Persistent traversal with per-lane ray replacement: a warp keeps tracing
// until the batch is exhausted; lanes whose ray has finished take the next
// rays from a global counter (one warp-aggregated atomic per refill), so short
// rays do not idle behind long ones. Each ray's walk is the same exact
// depth-first traversal as trace_bvh2 / trace_bvh4; only the scheduling
// differs. Lanes alternate "descend to a leaf" and "test the leaf, pop"
// (while-while) and refill when refill_min<IO> lanes are idle. A descent
// pauses once fewer than LMGPU_TRACE_EXIT_BELOW lanes are still descending,
// so the lanes that reached a leaf or finished are not held up by the
// warp's longest descent; the paused lanes resume in the next round (on the
// 2^24-ray soup this raised the kernel from 1.48 to 2.29 Grays/s).
// For a multi-scene I/O policy each lane switches to its new ray's scene at
// refill (node and triangle arrays, root); an empty scene is a miss.
// The COUNT instantiation (measurement runs only) also adds the rays' slab
// and TriAccel tests to counts[0..1]; the walk is the same. The stack bound
// is the scene's stack_cap where that is below STACK.
// Shadow rays through binary nodes take the any-hit walk (bvh2_descend_any:
// a stack of node references, no pop-time tests), whose visibility verdicts
// equal the closest-hit walk's.
// Render shadow rays through binary nodes descend speculatively (SPEC in
// bvh2_descend_any; closest-hit render rays too with
// LMGPU_TRACE_SPECULATIVE=2): each round a lane tests at most one leaf, the
// one it postponed, and the warp's leaf tests fall in the same round.
template <int LAYOUT, bool ANY_HIT>
struct RefStackWalk : std::bool_constant<LMGPU_TRACE_ANYHIT_WALK && ANY_HIT && binary_layout(LAYOUT)> {};

template <int LAYOUT, int STACK, bool ANY_HIT, class IO, bool COUNT = false>
__global__ void __launch_bounds__(128, min_blocks<IO>::value)
k_trace_persistent(const DeviceScene s, const IO io, int32_t* status, unsigned long long* next_ray,
                   unsigned long long* counts)
{
    constexpr unsigned FULL = 0xffffffffu;
    constexpr bool REFS = RefStackWalk<LAYOUT, ANY_HIT>::value;
    constexpr bool RENDER = render_rays<IO>::value;
    constexpr bool SPEC = RENDER && binary_layout(LAYOUT) &&
                          (REFS ? LMGPU_TRACE_SPECULATIVE >= 1 : LMGPU_TRACE_SPECULATIVE >= 2);
#if LMGPU_TRACE_SHARED_STACK > 0
    // The shared part takes the same bytes either way: twice as many
    // 4-byte references as (reference, entry distance) pairs.
    constexpr int SH0 = REFS ? 2 * LMGPU_TRACE_SHARED_STACK : LMGPU_TRACE_SHARED_STACK;
    constexpr int SH = SH0 < STACK ? SH0 : STACK;
    using Entry = std::conditional_t<REFS, int, int2>;
    __shared__ Entry stack_sh[SH][128];
    Entry stack_local[STACK > SH ? STACK - SH : 1];
    using StackT = std::conditional_t<REFS, SplitRefStack<SH>, SplitStack<SH>>;
    const StackT stack{ stack_sh, stack_local };
#else
    std::conditional_t<REFS, int, int2> stack[STACK];
#endif
    const int64_t n = io.count();
    const unsigned lane = threadIdx.x & 31u;
    const int32_t root = binary_layout(LAYOUT) ? s.root_ref : s.root_ref4;
    const int cap = s.stack_cap < STACK ? s.stack_cap : STACK;
    LaneScene ls{ s.bvh2, s.bvh4, s.bvh2q, s.tris };
    TraceStats stats{ 0, 0 };
    TraceStats* const st = COUNT ? &stats : nullptr;
    TraversalRay r;
    Hit h;
    h.tri = -1;
    TravState ts;
    ts.ref = REF_DONE;
    ts.sp = 0;
    int32_t pend = 0;                          // postponed leaf (SPEC), 0: none
    int64_t idx = -1;
    bool exhausted = n <= 0;
    for (;;) {
        const bool idle = ts.ref == REF_DONE && pend == 0;
        const unsigned need = __ballot_sync(FULL, idle);
        if (!exhausted && (__popc(need) >= refill_min<IO>::value || need == FULL)) {
            const int leader = __ffs(need) - 1;
            unsigned long long base = 0;
            if ((int)lane == leader) base = atomicAdd(next_ray, (unsigned long long)__popc(need));
            base = __shfl_sync(FULL, base, leader);
            if (base + __popc(need) >= (unsigned long long)n) exhausted = true;
            if (idle) {
                idx = (int64_t)base + __popc(need & ((1u << lane) - 1u));
                if (idx < n) {
                    setup_ray<RENDER>(r, io.load(idx));
                    h.tri = -1;
                    if constexpr (per_ray_scene<IO>::value) {
                        const DeviceScene& rs = io.ray_scene(idx);
                        ls.bvh2 = rs.bvh2;
                        ls.bvh4 = rs.bvh4;
                        ls.bvh2q = rs.bvh2q;
                        ls.tris = rs.tris;
                        if (rs.num_tris > 0)
                            trav_begin<RENDER>(ts, binary_layout(LAYOUT) ? rs.root_ref : rs.root_ref4, rs.root_box, r, st);
                    } else {
                        trav_begin<RENDER>(ts, root, s.root_box, r, st);
                    }
                    if (ts.ref == REF_DONE) io.store(idx, h, r);
                }
            }
        } else if (exhausted && need == FULL) {
            break;
        }
        if (ts.ref != REF_DONE || pend != 0) {
            bool ok = true;
            if (ts.ref != REF_DONE) {
                if constexpr (REFS && LAYOUT == LMGPU_LAYOUT_BVH2Q)
                    ok = bvh2_descend_any<exit_below<IO>::value, RENDER, SPEC>(ls.bvh2q, ts, stack, cap, r, st,
                                                                             !exhausted, &pend);
                else if constexpr (REFS)
                    ok = bvh2_descend_any<exit_below<IO>::value, RENDER, SPEC>(ls.bvh2, ts, stack, cap, r, st,
                                                                             !exhausted, &pend);
                else
                    ok = descend<LAYOUT, exit_below<IO>::value, RENDER, SPEC>(ls, ts, stack, cap, r, !exhausted, st,
                                                                            &pend);
            }
            if (!ok) {
                atomicOr(status, STATUS_STACK_OVERFLOW);
                h.tri = -1;
                ts.ref = REF_DONE;
                pend = 0;
            } else if (SPEC) {
                // the postponed leaf; a leaf the descent stopped at is
                // postponed by the next round's descent
                if (pend != 0) {
                    const int32_t leaf = pend;
                    pend = 0;
                    if (trace_leaf<ANY_HIT, RENDER>(ls.tris, ~leaf, r, h, st) && ANY_HIT) ts.ref = REF_DONE;
                }
            } else if (ts.ref < 0) {           // at a leaf (a paused descent resumes next round)
                // (a binary pop is the reference's far-child test; 4-wide
                // nodes count their four slab tests when fetched)
                if (trace_leaf<ANY_HIT, RENDER>(ls.tris, ~ts.ref, r, h, st) && ANY_HIT) ts.ref = REF_DONE;
                else if constexpr (REFS) pop_any(ts, stack);
                else pop_next(ts, stack, r, binary_layout(LAYOUT) ? st : nullptr);
            }
            if (ts.ref == REF_DONE) io.store(idx, h, r);
        }
    }
    if (COUNT) add_trace_stats(stats, counts);
}

// Brute-force traversal for the naive layout (one thread per ray).
template <bool ANY_HIT, class IO>
__global__ void __launch_bounds__(128) k_trace_naive(const DeviceScene s, const IO io)
{
    const int64_t n = io.count();
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        TraversalRay r;
        setup_ray(r, io.load(i));
        Hit h;
        h.tri = -1;
        if (s.num_tris > 0) trace_naive<ANY_HIT>(s.tris_by_id, s.num_tris, r, h, nullptr);
        io.store(i, h, r);
    }
}

// Resident-grid size of a kernel (blocks of 128 threads), cached per kernel.
int resident_blocks_of(const void* kernel);
template <class K>
int resident_blocks(K kernel)
{
    return resident_blocks_of(reinterpret_cast<const void*>(kernel));
}

// Launches the traversal for `io` on `stream`: persistent kernel for the
// BVH layouts (with the scene's work counter reset first), brute force for
// the naive layout. `max_rays` bounds the grid (0 = resident grid). COUNT
// launches the counting instantiation, adding to `counts` (BVH layouts).
template <bool ANY_HIT, int STACK, bool COUNT, class IO>
int launch_trace_stack(LmgpuScene* sc, const DeviceScene& s, const IO& io, int64_t max_rays, cudaStream_t stream,
                       unsigned long long* counts)
{
    if (s.layout == LMGPU_LAYOUT_NAIVE || s.num_tris == 0) {
        if (COUNT) return fail(LMGPU_ERR_UNSUPPORTED, "traversal counters need a BVH layout");
        const int64_t blocks = std::max<int64_t>(1, std::min<int64_t>((max_rays + 127) / 128, 148 * 64));
        k_trace_naive<ANY_HIT, IO><<<blocks, 128, 0, stream>>>(s, io);
        LMGPU_CUDA_TRY(cudaGetLastError());
        return LMGPU_OK;
    }
    // Each launch takes its own counter from the scene's ring, so persistent
    // kernels queued on different streams never share one.
    unsigned long long* work = sc->d_work + (sc->work_slot++ % LmgpuScene::WORK_SLOTS);
    LMGPU_CUDA_TRY(cudaMemsetAsync(work, 0, sizeof(unsigned long long), stream));
    if (s.layout == LMGPU_LAYOUT_BVH2) {
        auto k = k_trace_persistent<LMGPU_LAYOUT_BVH2, STACK, ANY_HIT, IO, COUNT>;
        int64_t blocks = resident_blocks(k);
        if (max_rays > 0) blocks = std::max<int64_t>(1, std::min<int64_t>(blocks, (max_rays + 127) / 128));
        k<<<blocks, 128, 0, stream>>>(s, io, sc->d_status, work, counts);
    } else {
        auto k = k_trace_persistent<LMGPU_LAYOUT_BVH4, STACK, ANY_HIT, IO, COUNT>;
        int64_t blocks = resident_blocks(k);
        if (max_rays > 0) blocks = std::max<int64_t>(1, std::min<int64_t>(blocks, (max_rays + 127) / 128));
        k<<<blocks, 128, 0, stream>>>(s, io, sc->d_status, work, counts);
    }
    LMGPU_CUDA_TRY(cudaGetLastError());
    return LMGPU_OK;
}

// `render` traces the scene's render view (its render tree), else the
// reference's tree.
template <bool ANY_HIT, class IO, bool COUNT = false>
int launch_trace(LmgpuScene* sc, const IO& io, int64_t max_rays, cudaStream_t stream,
                 unsigned long long* counts = nullptr, bool render = false)
{
    const DeviceScene& s = render ? sc->rdev : sc->dev;
    const int cap = s.stack_cap;
    if (cap <= 32) return launch_trace_stack<ANY_HIT, 32, COUNT>(sc, s, io, max_rays, stream, counts);
    if (cap <= 64) return launch_trace_stack<ANY_HIT, 64, COUNT>(sc, s, io, max_rays, stream, counts);
    if (cap <= 128) return launch_trace_stack<ANY_HIT, 128, COUNT>(sc, s, io, max_rays, stream, counts);
    if (cap <= 256) return launch_trace_stack<ANY_HIT, 256, COUNT>(sc, s, io, max_rays, stream, counts);
    return fail(LMGPU_ERR_UNSUPPORTED, "BVH deeper than the largest compiled traversal stack (256)");
}

}  // namespace lmgpu
