// Multi-scene batch: many independent scenes rendered as one stream of
// waves, each wave captured once into a CUDA graph and replayed.
//
// The one-scene driver (pathtrace.cu) reads every queue count back to the
// host to size its next launch, so a small scene spends most of its time in
// launch gaps and host round trips, and the GPU renders one scene at a time.
// Here the waves run over the concatenated sample sequence of all scenes
// (SceneTable context: per-path scene index, per-ray scene in traversal),
// launches have fixed grids that read their counts on the device, and one
// wave (init, K bounces of trace / shade / shadow, splat, wave advance) is a
// fixed kernel sequence: captured into a graph once per configuration and
// launched once per wave with no host synchronisation. Scenes whose depth is
// unbounded (max_path_vertices = -1) finish their tail bounces with direct
// launches after the graph.
//
// Overlap mode keeps two pools of path state and runs each wave's
// latency-bound tail bounces beside the next wave's first bounces (two
// branches of one captured graph).
//
// Stream mode regenerates paths instead: the path slots form
// one pool, every iteration retires the paths that finished (splat, free the
// slot) and starts new camera paths in the free slots, so the ray queues
// stay full until the samples run out and only the batch's last paths run
// a latency-bound tail. Two iterations (both queue parities) are one
// captured graph, launched until a device-side flag reports that every
// sample has started and every slot is free.
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/lmgpu.h"
#include "internal.h"
#include "pt_kernels.cuh"
#include "trace_kernels.cuh"

using namespace lmgpu;

namespace {

constexpr int WORK_SLOTS = 160;            // traversal launches per wave: 2 per bounce + 1
constexpr int POOLS = 2;                   // path pools (overlap mode uses both)
constexpr int DEFAULT_OVERLAP_BOUNCE = 3;
constexpr int GRAPH_BOUNCES_UNBOUNDED = 24;
constexpr int MAX_BOUNDED_BOUNCES = 64;
// path state (two queues of 64-byte ray records, hits, radiance, shadow
// rays, raster) + sample index, scene index, depth, free list, retire queue;
// the shadow arrays hold 2 entries per path (in stream mode a new path's
// camera-vertex shadow ray and its first bounce's share one shadow pass).
constexpr size_t BYTES_PER_PATH = 16 * 13 + 16 * 3 + 8 + 8 + 4 + 4 + 4 + 4;
constexpr int STREAM_CHECK_EVERY = 8;      // graph launches between checks of the done flag

// Device totals of a render: [0] closest-hit rays, [1] shadow rays,
// [2] deepest bounce with a live ray.
constexpr int NSTATS = 4;

struct GraphKey {
    int tech = -1, fp64 = -1, layout = -1, stack = -1, bounces = -1, bounded = -1, shade_blocks = -1, mode = -1;
    int split = -1;
    int64_t paths = -1;
    int num_scenes = -1;
    bool operator==(const GraphKey& o) const
    {
        return tech == o.tech && fp64 == o.fp64 && layout == o.layout && stack == o.stack && bounces == o.bounces &&
               bounded == o.bounded && shade_blocks == o.shade_blocks && paths == o.paths && num_scenes == o.num_scenes &&
               mode == o.mode && split == o.split;
    }
};

// A measurement render's record (lmgpu_batch_profile): events around every
// traversal launch and, with `count`, the counting kernels' totals.
struct TraceProfileRun {
    bool count = false;
    std::vector<cudaEvent_t> events;          // start, end of each traversal launch
    std::vector<int> kinds;                   // 0 closest hit, 1 shadow
    unsigned long long* d_counts = nullptr;   // [kind][slab tests, TriAccel tests]
    cudaError_t error = cudaSuccess;
};

}  // namespace

struct LmgpuBatch {
    int device = 0;
    int sms = 148;
    std::vector<LmgpuScene*> scenes;
    LmgpuBatchConfig cfg{ LMGPU_LAYOUT_BVH2, 1 << 27, 16, 1, LMGPU_BATCH_WAVES, 0 };

    BatchEntry* d_table = nullptr;
    int64_t* d_begins = nullptr;
    WaveCtl* d_wave = nullptr;              // one per path pool
    StreamCtl* d_ctl = nullptr;
    int64_t* h_done = nullptr;              // pinned: StreamCtl::done and ::iterations
    unsigned long long* d_stats = nullptr;
    unsigned long long* d_work = nullptr;   // WORK_SLOTS per path pool
    int32_t* d_status = nullptr;
    BatchEntry* h_table = nullptr;          // pinned staging
    int64_t* h_begins = nullptr;
    unsigned long long* h_stats = nullptr;
    uint32_t* h_counts = nullptr;
    cudaEvent_t staged = nullptr;           // the staging buffers' last copy has run

    void* ws_mem = nullptr;
    int64_t ws_capacity = 0;                // paths per pool
    int ws_pools = 0;
    PathState st[POOLS]{};

    cudaStream_t cap_stream = nullptr;
    // Overlap period branches: heads at the highest stream priority, tails
    // at the lowest (captured kernel nodes keep their stream's priority).
    cudaStream_t cap_hi = nullptr, cap_lo = nullptr;    // for capture
    cudaStream_t hi = nullptr, lo = nullptr;            // for direct launches
    cudaEvent_t ev[5] = {};                 // overlap period: fork, tail 0, head 1, head branch end, tail branch end
    cudaGraphExec_t exec = nullptr;         // a wave, two stream iterations, or an overlap period
    cudaGraphExec_t exec_head = nullptr;    // overlap: pool 0's first head
    cudaGraphExec_t exec_tail = nullptr;    // overlap: pool 0's last tail
    GraphKey key;

    TraceProfileRun* prof = nullptr;        // set during lmgpu_batch_profile only

    // lmgpu_batch_render's films: device films of all scenes, their rescaled
    // float copies and a pinned host copy.
    void* hf_film = nullptr;
    size_t hf_film_bytes = 0;
    float* hf_out = nullptr;
    float* hf_pinned = nullptr;
    size_t hf_out_bytes = 0;
};

namespace {

// ------------------------------------------------------ small kernels ----

template <class F>
__global__ void k_rescale_film(const F* film, float* out, int64_t n, double scale)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = (float)((double)film[i] * scale);
}

// Pool l starts at wave l; each pool then advances by `pools` waves.
__global__ void k_batch_setup(WaveCtl* wave, int pools, int64_t total, int64_t step, unsigned long long* stats)
{
    for (int l = 0; l < pools; l++) {
        const int64_t base = l * step;
        const int64_t left = total - base;
        wave[l].base = base;
        wave[l].count = left <= 0 ? 0 : (left < step ? left : step);
        wave[l].total = total;
        wave[l].step = step;
        wave[l].stride = pools * step;
    }
    for (int i = 0; i < NSTATS; i++) stats[i] = 0;
}

// Start of a wave: clear the queue counters and this wave's traversal work
// counters.
__global__ void k_wave_begin(uint32_t* counters, unsigned long long* work, int slots)
{
    for (int i = threadIdx.x; i < slots; i += blockDim.x) work[i] = 0;
    if (threadIdx.x < 4) counters[threadIdx.x] = 0;
}

// Before bounce k: tally the rays about to be traced and the shadow rays of
// the previous pass, then clear the output queue and the shadow queue. The
// totals are shared by the path pools (atomics: pools run concurrently).
__global__ void k_bounce_prep(uint32_t* counters, int qin, int k, unsigned long long* stats)
{
    const uint32_t n = counters[qin];
    atomicAdd(stats + 0, (unsigned long long)n);
    atomicAdd(stats + 1, (unsigned long long)counters[2]);
    if (n > 0) atomicMax(stats + 2, (unsigned long long)k);
    counters[1 - qin] = 0;
    counters[2] = 0;
}

// End of a wave (after the splat): last shadow tally, advance the pool to
// its next wave.
__global__ void k_wave_end(WaveCtl* wave, uint32_t* counters, unsigned long long* stats)
{
    atomicAdd(stats + 1, (unsigned long long)counters[2]);
    counters[2] = 0;
    const int64_t base = wave->base + wave->stride;
    wave->base = base;
    const int64_t left = wave->total - base;
    wave->count = left <= 0 ? 0 : (left < wave->step ? left : wave->step);
}

// Stream mode: all slots free, nothing started.
__global__ void k_stream_setup(StreamCtl* ctl, int64_t total, int64_t capacity, int32_t* free_slots, uint32_t* counters,
                               unsigned long long* stats)
{
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    for (int64_t i = t; i < capacity; i += (int64_t)gridDim.x * blockDim.x) free_slots[i] = (int32_t)i;
    if (t == 0) {
        ctl->next = 0;
        ctl->total = total;
        ctl->free_count = capacity;
        ctl->n_new = 0;
        ctl->free_base = 0;
        ctl->g0 = 0;
        ctl->capacity = capacity;
        ctl->iterations = 0;
        ctl->done = 0;
        for (int i = 0; i < 4; i++) counters[i] = 0;
        for (int i = 0; i < NSTATS; i++) stats[i] = 0;
    }
}

// Start of a stream iteration with input queue q: tally the previous
// iteration (it traced queue 1 - q and shaded into q), return its retired
// slots, then start min(free slots, samples left) new paths.
__global__ void k_stream_plan(StreamCtl* ctl, uint32_t* counters, int q, unsigned long long* stats,
                              unsigned long long* work)
{
    stats[0] += counters[1 - q];
    stats[1] += counters[2];
    ctl->free_count += counters[3];
    counters[1 - q] = 0;
    counters[2] = 0;
    counters[3] = 0;
    const int64_t left = ctl->total - ctl->next;
    const int64_t n = left < ctl->free_count ? left : ctl->free_count;
    ctl->done = (left <= 0 && ctl->free_count == ctl->capacity) ? 1 : 0;
    ctl->n_new = n;
    ctl->free_base = ctl->free_count - n;
    ctl->free_count -= n;
    ctl->g0 = ctl->next;
    ctl->next += n;
    ctl->iterations++;
    work[0] = 0;
    work[1] = 0;
}

// ------------------------------------------------------- wave builder ----

// Kernel layout of each walk: LMGPU_LAYOUT_BVH2_QSHADOW traces bounce rays
// through the float binary nodes and shadow rays through the quantised ones.
constexpr int walk_layout(int layout, bool any_hit)
{
    return layout == LMGPU_LAYOUT_BVH2_QSHADOW ? (any_hit ? LMGPU_LAYOUT_BVH2Q : LMGPU_LAYOUT_BVH2) : layout;
}

// Launches one persistent traversal of `io`. During a measurement render
// (b->prof) the launch is bracketed by CUDA events and, when counting, runs
// the counting instantiation of the same kernel.
template <int LAYOUT, int STACK, bool ANY_HIT, class IO>
void launch_traversal(const LmgpuBatch* b, int blocks, const DeviceScene& proto, const IO& io,
                      unsigned long long* work, cudaStream_t s)
{
    TraceProfileRun* p = b->prof;
    if (!p) {
        k_trace_persistent<walk_layout(LAYOUT, ANY_HIT), STACK, ANY_HIT, IO><<<blocks, 128, 0, s>>>(proto, io, b->d_status, work, nullptr);
        return;
    }
    cudaEvent_t e[2] = { nullptr, nullptr };
    for (cudaEvent_t& x : e)
        if (p->error == cudaSuccess) p->error = cudaEventCreate(&x);
    if (p->error == cudaSuccess) p->error = cudaEventRecord(e[0], s);
    if (p->count)
        k_trace_persistent<walk_layout(LAYOUT, ANY_HIT), STACK, ANY_HIT, IO, true><<<blocks, 128, 0, s>>>(
            proto, io, b->d_status, work, p->d_counts + (ANY_HIT ? 2 : 0));
    else
        k_trace_persistent<walk_layout(LAYOUT, ANY_HIT), STACK, ANY_HIT, IO><<<blocks, 128, 0, s>>>(proto, io, b->d_status, work, nullptr);
    if (p->error == cudaSuccess) p->error = cudaEventRecord(e[1], s);
    for (cudaEvent_t x : e)
        if (x) p->events.push_back(x);
    if (e[0] && e[1]) p->kinds.push_back(ANY_HIT ? 1 : 0);
}

struct Launch {
    int64_t paths;             // wave capacity
    int shade_blocks;
    int trace_blocks;          // closest-hit grid
    int shadow_blocks;         // any-hit grid
    DeviceScene proto;         // template scene for the traversal kernel (layout only)
};

// One wave of path pool l: head = begin, init, camera shadow pass, bounces
// 1 .. T-1; tail = bounces T .. K, splat, advance. The traversal launches of
// bounce k use work slots slot_of(k) and slot_of(k) + 1 of the pool.
template <int TECH, class F, int LAYOUT, int STACK>
struct Wave {
    using Ctx = SceneTable<float>;     // init / shade use no film
    using FilmCtx = SceneTable<F>;

    static Ctx ctx(const LmgpuBatch* b, int l)
    {
        return Ctx{ b->d_table, b->d_begins, (int32_t)b->scenes.size(), b->d_wave + l };
    }
    static FilmCtx film_ctx(const LmgpuBatch* b, int l)
    {
        return FilmCtx{ b->d_table, b->d_begins, (int32_t)b->scenes.size(), b->d_wave + l };
    }
    static unsigned long long* work(const LmgpuBatch* b, int l) { return b->d_work + (size_t)l * WORK_SLOTS; }
    static int slot_of(int k) { return (TECH != LMGPU_RENDER_PT ? 1 : 0) + 2 * (k - 1); }

    static void shadow(const LmgpuBatch* b, const Launch& L, int l, int slot, cudaStream_t s)
    {
        const PathState& st = b->st[l];
        ShadowIO<FilmCtx> io{ st.counters + 2, st.sh_o, st.sh_d, st.sh_c, st.L, film_ctx(b, l) };
        launch_traversal<LAYOUT, STACK, true>(b, L.shadow_blocks, L.proto, io, work(b, l) + slot, s);
    }

    static void bounce(const LmgpuBatch* b, const Launch& L, int l, int k, int slot, cudaStream_t s)
    {
        const PathState& st = b->st[l];
        const int qin = (k - 1) & 1;
        k_bounce_prep<<<1, 1, 0, s>>>(st.counters, qin, k, b->d_stats);
        PathRayIO<true> io{ st.counters + qin, st.qo[qin], st.qd[qin], st.hit, b->d_table };
        launch_traversal<LAYOUT, STACK, false>(b, L.trace_blocks, L.proto, io, work(b, l) + slot, s);
        k_pt_shade<TECH, Ctx><<<L.shade_blocks, 128, 0, s>>>(ctx(b, l), st, k, qin, 1 - qin);
        if (TECH != LMGPU_RENDER_PT) shadow(b, L, l, slot + 1, s);
    }

    static void head(const LmgpuBatch* b, const Launch& L, int l, int T, cudaStream_t s)
    {
        const PathState& st = b->st[l];
        k_wave_begin<<<1, 128, 0, s>>>(st.counters, work(b, l), WORK_SLOTS);
        k_pt_init<TECH, Ctx><<<(unsigned)((L.paths + 127) / 128), 128, 0, s>>>(ctx(b, l), st, 0, 0);
        if (TECH != LMGPU_RENDER_PT) shadow(b, L, l, 0, s);
        for (int k = 1; k < T; k++) bounce(b, L, l, k, slot_of(k), s);
    }

    static void tail(const LmgpuBatch* b, const Launch& L, int l, int T, int K, cudaStream_t s)
    {
        for (int k = T; k <= K; k++) bounce(b, L, l, k, slot_of(k), s);
        tail_end(b, L, l, s);
    }

    // Pool 0: init + bounces 1..K (+ splat and wave advance when `finish`).
    static void body(const LmgpuBatch* b, const Launch& L, int K, bool finish, cudaStream_t s)
    {
        head(b, L, 0, K + 1, s);
        if (finish) tail_end(b, L, 0, s);
    }

    static void tail_end(const LmgpuBatch* b, const Launch& L, int l, cudaStream_t s)
    {
        k_pt_splat<FilmCtx><<<(unsigned)((L.paths + 127) / 128), 128, 0, s>>>(film_ctx(b, l), b->st[l], 0);
        k_wave_end<<<1, 1, 0, s>>>(b->d_wave + l, b->st[l].counters, b->d_stats);
    }

    static void warm(Launch& L)
    {
        L.trace_blocks = resident_blocks(k_trace_persistent<walk_layout(LAYOUT, false), STACK, false, PathRayIO<true>>);
        L.shadow_blocks = resident_blocks(k_trace_persistent<walk_layout(LAYOUT, true), STACK, true, ShadowIO<FilmCtx>>);
    }
};

template <int TECH, class F, int LAYOUT, int STACK>
struct Stream {
    using Ctx = StreamTable<float>;    // init / shade use no film
    using FilmCtx = StreamTable<F>;

    template <class C>
    static C make(const LmgpuBatch* b)
    {
        return C{ b->d_table, b->d_begins, (int32_t)b->scenes.size(), b->d_ctl, b->st[0].sample, b->d_stats + 2 };
    }

    // One iteration with input queue q; traversal work counters work[2q], work[2q + 1].
    static void iteration(const LmgpuBatch* b, const Launch& L, int q, cudaStream_t s)
    {
        const PathState& st = b->st[0];
        unsigned long long* work = b->d_work + 2 * q;
        k_stream_plan<<<1, 1, 0, s>>>(b->d_ctl, st.counters, q, b->d_stats, work);
        k_pt_init<TECH, Ctx><<<(unsigned)((L.paths + 127) / 128), 128, 0, s>>>(make<Ctx>(b), st, 0, q);
        PathRayIO<true> io{ st.counters + q, st.qo[q], st.qd[q], st.hit, b->d_table };
        launch_traversal<LAYOUT, STACK, false>(b, L.trace_blocks, L.proto, io, work, s);
        k_pt_shade<TECH, Ctx><<<L.shade_blocks, 128, 0, s>>>(make<Ctx>(b), st, 0, q, 1 - q);
        if (TECH != LMGPU_RENDER_PT) {
            ShadowIO<FilmCtx> sio{ st.counters + 2, st.sh_o, st.sh_d, st.sh_c, st.L, make<FilmCtx>(b) };
            launch_traversal<LAYOUT, STACK, true>(b, L.shadow_blocks, L.proto, sio, work + 1, s);
        }
        k_pt_retire<FilmCtx><<<L.shade_blocks, 128, 0, s>>>(make<FilmCtx>(b), st);
    }

    static void pair(const LmgpuBatch* b, const Launch& L, cudaStream_t s)
    {
        iteration(b, L, 0, s);
        iteration(b, L, 1, s);
    }

    static void warm(Launch& L)
    {
        L.trace_blocks = resident_blocks(k_trace_persistent<walk_layout(LAYOUT, false), STACK, false, PathRayIO<true>>);
        L.shadow_blocks = resident_blocks(k_trace_persistent<walk_layout(LAYOUT, true), STACK, true, ShadowIO<FilmCtx>>);
    }
};

// ------------------------------------------------------------ driver ------

void drop_graphs(LmgpuBatch* b)
{
    for (cudaGraphExec_t* g : { &b->exec, &b->exec_head, &b->exec_tail })
        if (*g) { cudaGraphExecDestroy(*g); *g = nullptr; }
    b->key = GraphKey{};
}

// Path state of `paths` paths in each of `pools` pools (at least the pools
// and capacity already held), one allocation; every pool starts on a
// 256-byte boundary.
int ensure_batch_workspace(LmgpuBatch* b, int64_t paths, int pools)
{
    if (b->ws_mem && b->ws_capacity >= paths && b->ws_pools >= pools) return LMGPU_OK;
    pools = std::max(pools, b->ws_pools);
    drop_graphs(b);
    if (b->ws_mem) { cudaFree(b->ws_mem); b->ws_mem = nullptr; b->ws_capacity = 0; b->ws_pools = 0; }
    const size_t P = (size_t)paths;
    const size_t pool_bytes = (256 + P * BYTES_PER_PATH + 255) / 256 * 256;
    cudaError_t e = cudaMalloc(&b->ws_mem, pool_bytes * pools);
    if (e != cudaSuccess) {
        b->ws_mem = nullptr;
        return e == cudaErrorMemoryAllocation ? fail(LMGPU_ERR_OOM, "batch workspace allocation failed")
                                              : cuda_fail(e, "cudaMalloc(batch workspace)");
    }
    for (int l = 0; l < pools; l++) {
        char* p = static_cast<char*>(b->ws_mem) + pool_bytes * l;
        auto take = [&](size_t n) { char* r = p; p += n; return r; };
        PathState& st = b->st[l];
        st.counters = reinterpret_cast<uint32_t*>(take(256));
        for (int q = 0; q < 2; q++) {
            st.qo[q] = reinterpret_cast<float4*>(take(16 * P));
            st.qd[q] = reinterpret_cast<float4*>(take(16 * P));
            st.qt[q] = reinterpret_cast<float4*>(take(16 * P));
            st.qn[q] = reinterpret_cast<float4*>(take(16 * P));
        }
        st.hit = reinterpret_cast<float4*>(take(16 * P));
        st.L = reinterpret_cast<float4*>(take(16 * P));
        st.sh_o = reinterpret_cast<float4*>(take(2 * 16 * P));
        st.sh_d = reinterpret_cast<float4*>(take(2 * 16 * P));
        st.sh_c = reinterpret_cast<float4*>(take(2 * 16 * P));
        st.sample = reinterpret_cast<int64_t*>(take(8 * P));      // 8-byte arrays first: alignment
        st.raster = reinterpret_cast<float2*>(take(8 * P));
        st.scene = reinterpret_cast<int32_t*>(take(4 * P));
        st.depth = reinterpret_cast<int32_t*>(take(4 * P));
        st.free_slots = reinterpret_cast<int32_t*>(take(4 * P));
        st.retire = reinterpret_cast<int32_t*>(take(4 * P));
        const uint32_t caps[4] = { (uint32_t)P, (uint32_t)P, (uint32_t)(2 * P), (uint32_t)P };
        for (int q = 0; q < 4; q++) {
            st.cap[q] = caps[q];
#if LMGPU_BOUNDS_CHECK
            st.cap[q] = (uint32_t)std::min<int64_t>(caps[q], check_limit_from_env("LMGPU_CHECK_QUEUE_LIMIT"));
#endif
        }
        st.status = b->d_status;
    }
    b->ws_capacity = paths;
    b->ws_pools = pools;
    return LMGPU_OK;
}

// Captures what `fn` launches on the capture stream into *out.
template <class Fn>
int capture(LmgpuBatch* b, Fn fn, cudaGraphExec_t* out, const char* what, unsigned long long flags = 0)
{
    LMGPU_CUDA_TRY(cudaStreamBeginCapture(b->cap_stream, cudaStreamCaptureModeThreadLocal));
    fn(b->cap_stream);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(b->cap_stream, &g);
    if (e != cudaSuccess) return cuda_fail(e, what);
    e = cudaGraphInstantiate(out, g, flags);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) { *out = nullptr; return cuda_fail(e, "cudaGraphInstantiate"); }
    return LMGPU_OK;
}

int consume_batch_status(LmgpuBatch* b, cudaStream_t s)
{
    int32_t v = 0;
    LMGPU_CUDA_TRY(cudaMemcpyAsync(&v, b->d_status, sizeof(v), cudaMemcpyDeviceToHost, s));
    LMGPU_CUDA_TRY(cudaStreamSynchronize(s));
    if (v == 0) return LMGPU_OK;
    LMGPU_CUDA_TRY(cudaMemsetAsync(b->d_status, 0, sizeof(int32_t), s));
    return status_error(v);
}

// Everything a render needs to know about its parameters.
struct Plan {
    int tech, fp64, stack, bounces;
    bool bounded;
    int64_t total;
};

int make_plan(LmgpuBatch* b, const LmgpuRenderParams* params, void* const* films, Plan& pl)
{
    const int n = (int)b->scenes.size();
    if (!params) return fail(LMGPU_ERR_INVALID, "null params");
    pl.tech = params[0].technique;
    pl.fp64 = params[0].film_fp64 ? 1 : 0;
    pl.total = 0;
    pl.bounded = true;
    int max_pv = 1, cap = 0;
    for (int i = 0; i < n; i++) {
        const LmgpuRenderParams& p = params[i];
        const LmgpuScene* sc = b->scenes[i];
        if (films && !films[i]) return fail(LMGPU_ERR_INVALID, "null film");
        if (p.technique != pl.tech) return fail(LMGPU_ERR_INVALID, "a batch renders with one technique");
        if ((p.film_fp64 ? 1 : 0) != pl.fp64) return fail(LMGPU_ERR_INVALID, "a batch uses one film type");
        if (p.technique < LMGPU_RENDER_PT || p.technique > LMGPU_RENDER_PT_MIS) return fail(LMGPU_ERR_INVALID, "unknown technique");
        if (p.sampling != LMGPU_SAMPLING_STRATIFIED && p.sampling != LMGPU_SAMPLING_UNIFORM) return fail(LMGPU_ERR_INVALID, "unknown sampling");
        if (p.num_samples <= 0) return fail(LMGPU_ERR_INVALID, "num_samples must be positive");
        if (p.sample_offset < 0) return fail(LMGPU_ERR_INVALID, "negative sample offset");
        if (!sample_range_ok(p.sample_offset, p.num_samples)) return fail(LMGPU_ERR_INVALID, "sample indices reach 2^53");
        if (!sc->dev.cam.valid) return fail(LMGPU_ERR_INVALID, "scene has no camera");
        pl.total += p.num_samples;
        if (p.max_path_vertices == -1) pl.bounded = false;
        else max_pv = std::max(max_pv, p.max_path_vertices);
        cap = std::max(cap, sc->rdev.stack_cap);
    }
    if (pl.total >= (int64_t(1) << 62)) return fail(LMGPU_ERR_INVALID, "sample count too large");
    pl.bounces = pl.bounded ? max_pv - 1 : GRAPH_BOUNCES_UNBOUNDED;
    if (pl.bounded && pl.bounces > MAX_BOUNDED_BOUNCES) {
        pl.bounded = false;
        pl.bounces = GRAPH_BOUNCES_UNBOUNDED;
    }
    if (cap <= 64) pl.stack = 64;
    else if (cap <= 128) pl.stack = 128;
    else if (cap <= 256) pl.stack = 256;
    else return fail(LMGPU_ERR_UNSUPPORTED, "BVH deeper than the largest compiled traversal stack (256)");
    return LMGPU_OK;
}

int upload_table(LmgpuBatch* b, const LmgpuRenderParams* params, void* const* films, cudaStream_t s)
{
    const int n = (int)b->scenes.size();
    // The previous call's copies read the same pinned buffers.
    LMGPU_CUDA_TRY(cudaEventSynchronize(b->staged));
    int64_t begin = 0;
    for (int i = 0; i < n; i++) {
        const LmgpuRenderParams& p = params[i];
        BatchEntry& e = b->h_table[i];
        e.s = b->scenes[i]->rdev;
        e.s.layout = b->cfg.layout;
        e.rc.technique = p.technique;
        e.rc.rr_depth = p.rr_depth;
        e.rc.max_pv = p.max_path_vertices;
        e.rc.sampling = p.sampling;
        e.rc.seed = p.seed;
        e.rc.sample_base = p.sample_offset;
        e.rc.pixels = (int64_t)e.s.cam.width * e.s.cam.height;
        e.rc.inv_pixels = 1.0 / double(e.rc.pixels);
        e.begin = begin;
        e.film = films[i];
        b->h_begins[i] = begin;
        begin += p.num_samples;
    }
    b->h_begins[n] = begin;
    LMGPU_CUDA_TRY(cudaMemcpyAsync(b->d_table, b->h_table, n * sizeof(BatchEntry), cudaMemcpyHostToDevice, s));
    LMGPU_CUDA_TRY(cudaMemcpyAsync(b->d_begins, b->h_begins, (n + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, s));
    LMGPU_CUDA_TRY(cudaEventRecord(b->staged, s));
    return LMGPU_OK;
}

// Stream mode: `iterations` returns the iterations run (including at most
// 2 * STREAM_CHECK_EVERY - 1 empty ones after the last path retired).
template <int TECH, class F, int LAYOUT, int STACK>
int run_stream(LmgpuBatch* b, const Plan& pl, int64_t P, cudaStream_t s, int64_t& iterations)
{
    using S = Stream<TECH, F, LAYOUT, STACK>;
    Launch L;
    L.paths = P;
    L.shade_blocks = std::max(1, b->cfg.shade_blocks_per_sm) * b->sms;
    L.proto = b->scenes[0]->rdev;
    L.proto.layout = LAYOUT;
    L.proto.stack_cap = STACK;        // every scene of the batch: the largest bound
    S::warm(L);
    const unsigned setup_blocks = (unsigned)std::min<int64_t>((P + 255) / 256, 148 * 16);
    k_stream_setup<<<setup_blocks, 256, 0, s>>>(b->d_ctl, pl.total, P, b->st[0].free_slots, b->st[0].counters, b->d_stats);
    LMGPU_CUDA_TRY(cudaGetLastError());
    if (b->cfg.use_graph) {
        GraphKey key;
        key.tech = TECH; key.fp64 = pl.fp64; key.layout = LAYOUT; key.stack = STACK; key.bounces = 0;
        key.bounded = 0; key.shade_blocks = L.shade_blocks; key.paths = P; key.num_scenes = (int)b->scenes.size();
        key.mode = LMGPU_BATCH_STREAM;
        if (!b->exec || !(b->key == key)) {
            drop_graphs(b);
            const int rc = capture(b, [&](cudaStream_t c) { S::pair(b, L, c); }, &b->exec,
                                   "graph capture of two stream iterations");
            if (rc != LMGPU_OK) return rc;
            b->key = key;
        }
    }
    // Every live path advances one bounce per iteration, so each slot's path
    // ends within max_len + 1 iterations and every such period starts at
    // least P samples: the bound below is never reached by a render that
    // ends (Russian roulette makes a 1024-bounce path vanishingly unlikely).
    const int64_t max_len = pl.bounded ? pl.bounces + 2 : 1024;
    const int64_t bound = 2 * (((pl.total + P - 1) / P + 1) * (max_len + 1)) + 4 * STREAM_CHECK_EVERY;
    int64_t launched = 0;
    for (;;) {
        for (int c = 0; c < STREAM_CHECK_EVERY; c++) {
            if (b->cfg.use_graph) LMGPU_CUDA_TRY(cudaGraphLaunch(b->exec, s));
            else S::pair(b, L, s);
            launched += 2;
        }
        LMGPU_CUDA_TRY(cudaGetLastError());
        LMGPU_CUDA_TRY(cudaMemcpyAsync(b->h_done, &b->d_ctl->iterations, 2 * sizeof(int64_t), cudaMemcpyDeviceToHost, s));
        LMGPU_CUDA_TRY(cudaStreamSynchronize(s));
        if (b->h_done[1]) break;
        if (launched > bound) return fail(LMGPU_ERR_TIMEOUT, "stream render did not end within its iteration bound");
    }
    iterations = b->h_done[0];
    return LMGPU_OK;
}

// Overlap mode: pool 0 renders waves 0, 2, 4, ..., pool 1 waves 1, 3, 5, ...;
// a wave splits at bounce T into head (init, bounces 1 .. T-1) and tail
// (bounces T .. K, splat). One period runs two branches,
//     heads (high priority):  head(2j + 1) -> head(2j + 2)   (after tail(2j): same pool)
//     tails (low priority):   tail(2j)     -> tail(2j + 1)   (after head(2j + 1))
// so each wave's latency-bound tail shares the GPU with the other pool's
// full-width head, and the block scheduler serves the head's kernels
// first. Pool 0's first head comes before the periods and its last tail
// after them; floor(W / 2) periods cover W waves (a wave past the last
// sample has no paths and costs only its launches). Depth must be
// bounded: the tail is a fixed sequence of bounces.
template <int TECH, class F, int LAYOUT, int STACK>
int run_overlap(LmgpuBatch* b, const Plan& pl, int64_t P, cudaStream_t s, int64_t& waves)
{
    using W = Wave<TECH, F, LAYOUT, STACK>;
    Launch L;
    L.paths = P;
    L.shade_blocks = std::max(1, b->cfg.shade_blocks_per_sm) * b->sms;
    L.proto = b->scenes[0]->rdev;
    L.proto.layout = LAYOUT;
    L.proto.stack_cap = STACK;        // every scene of the batch: the largest bound
    W::warm(L);
    const int K = pl.bounces;
    const int T = std::min(b->cfg.overlap_bounce > 0 ? b->cfg.overlap_bounce : DEFAULT_OVERLAP_BOUNCE, K + 1);
    waves = (pl.total + P - 1) / P;
    const int64_t periods = waves / 2;
    k_batch_setup<<<1, 1, 0, s>>>(b->d_wave, POOLS, pl.total, P, b->d_stats);
    LMGPU_CUDA_TRY(cudaGetLastError());

    auto head0 = [&](cudaStream_t a) { W::head(b, L, 0, T, a); };
    auto tail0 = [&](cudaStream_t a) { W::tail(b, L, 0, T, K, a); };
    // Returns the first failing event call (inside a capture, the capture's
    // end reports it too).
    auto period = [&](cudaStream_t a, cudaStream_t hi, cudaStream_t lo) -> cudaError_t {
        cudaEvent_t* ev = b->ev;
        cudaError_t e = cudaSuccess;
        auto chk = [&](cudaError_t r) { if (e == cudaSuccess) e = r; };
        chk(cudaEventRecord(ev[0], a));
        chk(cudaStreamWaitEvent(hi, ev[0], 0));
        chk(cudaStreamWaitEvent(lo, ev[0], 0));
        W::tail(b, L, 0, T, K, lo);
        chk(cudaEventRecord(ev[1], lo));
        W::head(b, L, 1, T, hi);
        chk(cudaEventRecord(ev[2], hi));
        chk(cudaStreamWaitEvent(hi, ev[1], 0));
        W::head(b, L, 0, T, hi);
        chk(cudaEventRecord(ev[3], hi));
        chk(cudaStreamWaitEvent(lo, ev[2], 0));
        W::tail(b, L, 1, T, K, lo);
        chk(cudaEventRecord(ev[4], lo));
        chk(cudaStreamWaitEvent(a, ev[3], 0));
        chk(cudaStreamWaitEvent(a, ev[4], 0));
        return e;
    };
    if (b->cfg.use_graph) {
        GraphKey key;
        key.tech = TECH; key.fp64 = pl.fp64; key.layout = LAYOUT; key.stack = STACK; key.bounces = K;
        key.bounded = 1; key.shade_blocks = L.shade_blocks; key.paths = P; key.num_scenes = (int)b->scenes.size();
        key.mode = LMGPU_BATCH_OVERLAP; key.split = T;
        if (!b->exec || !b->exec_head || !b->exec_tail || !(b->key == key)) {
            drop_graphs(b);
            int rc = capture(b, head0, &b->exec_head, "graph capture of a wave head");
            if (rc == LMGPU_OK)
                rc = capture(b, [&](cudaStream_t a) { (void)period(a, b->cap_hi, b->cap_lo); }, &b->exec,
                             "graph capture of an overlap period", cudaGraphInstantiateFlagUseNodePriority);
            if (rc == LMGPU_OK) rc = capture(b, tail0, &b->exec_tail, "graph capture of a wave tail");
            if (rc != LMGPU_OK) { drop_graphs(b); return rc; }
            b->key = key;
        }
        LMGPU_CUDA_TRY(cudaGraphLaunch(b->exec_head, s));
        for (int64_t j = 0; j < periods; j++) LMGPU_CUDA_TRY(cudaGraphLaunch(b->exec, s));
        LMGPU_CUDA_TRY(cudaGraphLaunch(b->exec_tail, s));
        return LMGPU_OK;
    }
    head0(s);
    LMGPU_CUDA_TRY(cudaGetLastError());
    for (int64_t j = 0; j < periods; j++) {
        cudaError_t e = period(s, b->hi, b->lo);
        if (e == cudaSuccess) e = cudaGetLastError();
        if (e != cudaSuccess) {
            // Nothing of this render may still run on the branch streams
            // once the call has returned.
            cudaStreamSynchronize(b->hi);
            cudaStreamSynchronize(b->lo);
            return cuda_fail(e, "overlap period (direct launches)");
        }
    }
    tail0(s);
    LMGPU_CUDA_TRY(cudaGetLastError());
    return LMGPU_OK;
}

template <int TECH, class F, int LAYOUT, int STACK>
int run_waves(LmgpuBatch* b, const Plan& pl, int64_t P, cudaStream_t s, int64_t& waves)
{
    if (b->cfg.mode == LMGPU_BATCH_STREAM) return run_stream<TECH, F, LAYOUT, STACK>(b, pl, P, s, waves);
    if (b->cfg.mode == LMGPU_BATCH_OVERLAP && pl.bounded) return run_overlap<TECH, F, LAYOUT, STACK>(b, pl, P, s, waves);
    using W = Wave<TECH, F, LAYOUT, STACK>;
    Launch L;
    L.paths = P;
    L.shade_blocks = std::max(1, b->cfg.shade_blocks_per_sm) * b->sms;
    L.proto = b->scenes[0]->rdev;
    L.proto.layout = LAYOUT;
    L.proto.stack_cap = STACK;        // every scene of the batch: the largest bound
    W::warm(L);
    waves = (pl.total + P - 1) / P;
    k_batch_setup<<<1, 1, 0, s>>>(b->d_wave, 1, pl.total, P, b->d_stats);
    LMGPU_CUDA_TRY(cudaGetLastError());

    if (b->cfg.use_graph) {
        GraphKey key;
        key.tech = TECH; key.fp64 = pl.fp64; key.layout = LAYOUT; key.stack = STACK; key.bounces = pl.bounces;
        key.bounded = pl.bounded; key.shade_blocks = L.shade_blocks; key.paths = P; key.num_scenes = (int)b->scenes.size();
        key.mode = LMGPU_BATCH_WAVES;
        if (!b->exec || !(b->key == key)) {
            drop_graphs(b);
            const int rc = capture(b, [&](cudaStream_t c) { W::body(b, L, pl.bounces, pl.bounded, c); }, &b->exec,
                                   "graph capture of a batch wave");
            if (rc != LMGPU_OK) return rc;
            b->key = key;
        }
    }
    for (int64_t w = 0; w < waves; w++) {
        if (b->cfg.use_graph) LMGPU_CUDA_TRY(cudaGraphLaunch(b->exec, s));
        else W::body(b, L, pl.bounces, pl.bounded, s);
        LMGPU_CUDA_TRY(cudaGetLastError());
        if (pl.bounded) continue;
        // Unbounded depth: finish the wave's remaining bounces directly.
        const int slot = (TECH != LMGPU_RENDER_PT ? 1 : 0);   // counters reused: clear before each launch
        for (int k = pl.bounces + 1;; k++) {
            const int qin = (k - 1) & 1;
            LMGPU_CUDA_TRY(cudaMemcpyAsync(b->h_counts, b->st[0].counters, 16, cudaMemcpyDeviceToHost, s));
            LMGPU_CUDA_TRY(cudaStreamSynchronize(s));
            if (b->h_counts[qin] == 0) break;
            LMGPU_CUDA_TRY(cudaMemsetAsync(b->d_work + slot, 0, 2 * sizeof(unsigned long long), s));
            W::bounce(b, L, 0, k, slot, s);
            LMGPU_CUDA_TRY(cudaGetLastError());
        }
        W::tail_end(b, L, 0, s);
        LMGPU_CUDA_TRY(cudaGetLastError());
    }
    return LMGPU_OK;
}

template <int TECH, class F, int LAYOUT>
int dispatch_stack(LmgpuBatch* b, const Plan& pl, int64_t P, cudaStream_t s, int64_t& waves)
{
    switch (pl.stack) {
    case 64: return run_waves<TECH, F, LAYOUT, 64>(b, pl, P, s, waves);
    case 128: return run_waves<TECH, F, LAYOUT, 128>(b, pl, P, s, waves);
    default: return run_waves<TECH, F, LAYOUT, 256>(b, pl, P, s, waves);
    }
}

template <int TECH, class F>
int dispatch_layout(LmgpuBatch* b, const Plan& pl, int64_t P, cudaStream_t s, int64_t& waves)
{
    switch (b->cfg.layout) {
    case LMGPU_LAYOUT_BVH4: return dispatch_stack<TECH, F, LMGPU_LAYOUT_BVH4>(b, pl, P, s, waves);
    case LMGPU_LAYOUT_BVH2Q: return dispatch_stack<TECH, F, LMGPU_LAYOUT_BVH2Q>(b, pl, P, s, waves);
    case LMGPU_LAYOUT_BVH2_QSHADOW: return dispatch_stack<TECH, F, LMGPU_LAYOUT_BVH2_QSHADOW>(b, pl, P, s, waves);
    default: return dispatch_stack<TECH, F, LMGPU_LAYOUT_BVH2>(b, pl, P, s, waves);
    }
}

template <class F>
int dispatch_tech(LmgpuBatch* b, const Plan& pl, int64_t P, cudaStream_t s, int64_t& waves)
{
    switch (pl.tech) {
    case LMGPU_RENDER_PT: return dispatch_layout<LMGPU_RENDER_PT, F>(b, pl, P, s, waves);
    case LMGPU_RENDER_PT_DIRECT: return dispatch_layout<LMGPU_RENDER_PT_DIRECT, F>(b, pl, P, s, waves);
    default: return dispatch_layout<LMGPU_RENDER_PT_MIS, F>(b, pl, P, s, waves);
    }
}

int check_config(const LmgpuBatchConfig& c)
{
    if (c.layout != LMGPU_LAYOUT_BVH2 && c.layout != LMGPU_LAYOUT_BVH4 && c.layout != LMGPU_LAYOUT_BVH2Q &&
        c.layout != LMGPU_LAYOUT_BVH2_QSHADOW)
        return fail(LMGPU_ERR_INVALID, "batch layout must be LMGPU_LAYOUT_BVH2, _BVH4, _BVH2Q or _BVH2_QSHADOW");
    if (c.wave_paths < 1024 || c.wave_paths > (1 << 27)) return fail(LMGPU_ERR_INVALID, "wave_paths must be in [1024, 2^27]");
    if (c.shade_blocks_per_sm < 1 || c.shade_blocks_per_sm > 64) return fail(LMGPU_ERR_INVALID, "shade_blocks_per_sm must be in [1, 64]");
    if (c.mode != LMGPU_BATCH_WAVES && c.mode != LMGPU_BATCH_STREAM && c.mode != LMGPU_BATCH_OVERLAP)
        return fail(LMGPU_ERR_INVALID, "unknown batch mode");
    if (c.overlap_bounce < 0 || c.overlap_bounce > MAX_BOUNDED_BOUNCES)
        return fail(LMGPU_ERR_INVALID, "overlap_bounce must be in [0, 64]");
    return LMGPU_OK;
}

// Renders with the batch's current configuration; device time in *ms when
// `ms` is given (synchronises).
int batch_render(LmgpuBatch* b, const LmgpuRenderParams* params, void* const* films, cudaStream_t s,
                 LmgpuRenderStats* stats)
{
    Plan pl;
    int rc = make_plan(b, params, films, pl);
    if (rc != LMGPU_OK) return rc;
    int cur = 0;
    LMGPU_CUDA_TRY(cudaGetDevice(&cur));
    if (cur != b->device) return fail(LMGPU_ERR_INVALID, "batch used on another device than it was created on");
    int64_t P = std::min<int64_t>(b->cfg.wave_paths, pl.total);
    const int pools = (b->cfg.mode == LMGPU_BATCH_OVERLAP && pl.bounded) ? 2 : 1;
    rc = ensure_batch_workspace(b, std::max<int64_t>(P, b->ws_capacity), pools);
    // A device short of memory gets smaller waves (the configuration stays).
    while (rc == LMGPU_ERR_OOM && P > (int64_t(1) << 20)) {
        P /= 2;
        rc = ensure_batch_workspace(b, P, pools);
    }
    if (rc != LMGPU_OK) return rc;
    if ((rc = upload_table(b, params, films, s)) != LMGPU_OK) return rc;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (stats) {
        LMGPU_CUDA_TRY(cudaEventCreate(&e0));
        LMGPU_CUDA_TRY(cudaEventCreate(&e1));
        LMGPU_CUDA_TRY(cudaEventRecord(e0, s));
    }
    int64_t waves = 0;
    rc = pl.fp64 ? dispatch_tech<double>(b, pl, P, s, waves) : dispatch_tech<float>(b, pl, P, s, waves);
    if (stats) {
        if (rc == LMGPU_OK) {
            cudaError_t e = cudaEventRecord(e1, s);
            if (e == cudaSuccess) e = cudaMemcpyAsync(b->h_stats, b->d_stats, NSTATS * sizeof(unsigned long long),
                                                      cudaMemcpyDeviceToHost, s);
            if (e == cudaSuccess) e = cudaStreamSynchronize(s);
            if (e != cudaSuccess) rc = cuda_fail(e, "batch completion");
        }
        float ms = 0.0f;
        if (rc == LMGPU_OK) cudaEventElapsedTime(&ms, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        std::memset(stats, 0, sizeof(*stats));
        if (rc == LMGPU_OK) {
            stats->shadow_rays = (int64_t)b->h_stats[1];
            stats->rays_traced = (int64_t)(b->h_stats[0] + b->h_stats[1]);
            stats->paths = pl.total;
            stats->waves = waves;
            stats->max_bounces_run = (int32_t)b->h_stats[2];
            stats->device_ms = ms;
        }
    }
    if (rc == LMGPU_OK && stats) rc = consume_batch_status(b, s);
    return rc;
}

}  // namespace

extern "C" {

int lmgpu_batch_create(LmgpuScene* const* scenes, int32_t num_scenes, LmgpuBatch** out)
{
    if (!out) return fail(LMGPU_ERR_INVALID, "null output");
    *out = nullptr;
    if (!scenes || num_scenes <= 0) return fail(LMGPU_ERR_INVALID, "a batch needs at least one scene");
    int dev = 0;
    LMGPU_CUDA_TRY(cudaGetDevice(&dev));
    for (int i = 0; i < num_scenes; i++) {
        if (!scenes[i]) return fail(LMGPU_ERR_INVALID, "null scene");
        if (scenes[i]->dev.layout == LMGPU_LAYOUT_NAIVE) return fail(LMGPU_ERR_INVALID, "batch scenes need a BVH layout");
        if (scenes[i]->device != dev) return fail(LMGPU_ERR_INVALID, "batch scenes must live on the current device");
    }
    LmgpuBatch* b = new (std::nothrow) LmgpuBatch;
    if (!b) return fail(LMGPU_ERR_OOM, "host allocation failed");
    b->device = dev;
    b->scenes.assign(scenes, scenes + num_scenes);
    cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, dev);
    const size_t n = (size_t)num_scenes;
    cudaError_t e = cudaSuccess;
    auto dm = [&](void** p, size_t bytes) { if (e == cudaSuccess) e = cudaMalloc(p, bytes); };
    auto hm = [&](void** p, size_t bytes) { if (e == cudaSuccess) e = cudaMallocHost(p, bytes); };
    dm(reinterpret_cast<void**>(&b->d_table), n * sizeof(BatchEntry));
    dm(reinterpret_cast<void**>(&b->d_begins), (n + 1) * sizeof(int64_t));
    dm(reinterpret_cast<void**>(&b->d_wave), POOLS * sizeof(WaveCtl));
    dm(reinterpret_cast<void**>(&b->d_ctl), sizeof(StreamCtl));
    hm(reinterpret_cast<void**>(&b->h_done), 2 * sizeof(int64_t));
    dm(reinterpret_cast<void**>(&b->d_stats), NSTATS * sizeof(unsigned long long));
    dm(reinterpret_cast<void**>(&b->d_work), POOLS * WORK_SLOTS * sizeof(unsigned long long));
    dm(reinterpret_cast<void**>(&b->d_status), sizeof(int32_t));
    hm(reinterpret_cast<void**>(&b->h_table), n * sizeof(BatchEntry));
    hm(reinterpret_cast<void**>(&b->h_begins), (n + 1) * sizeof(int64_t));
    hm(reinterpret_cast<void**>(&b->h_stats), NSTATS * sizeof(unsigned long long));
    hm(reinterpret_cast<void**>(&b->h_counts), 16);
    if (e == cudaSuccess) e = cudaMemset(b->d_status, 0, sizeof(int32_t));
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->cap_stream, cudaStreamNonBlocking);
    int least = 0, greatest = 0;
    if (e == cudaSuccess) e = cudaDeviceGetStreamPriorityRange(&least, &greatest);
    if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&b->cap_hi, cudaStreamNonBlocking, greatest);
    if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&b->cap_lo, cudaStreamNonBlocking, least);
    if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&b->hi, cudaStreamNonBlocking, greatest);
    if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&b->lo, cudaStreamNonBlocking, least);
    for (cudaEvent_t& ev : b->ev)
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->staged, cudaEventDisableTiming);
    if (e != cudaSuccess) {
        lmgpu_batch_destroy(b);
        return e == cudaErrorMemoryAllocation ? fail(LMGPU_ERR_OOM, "batch allocation failed") : cuda_fail(e, "batch creation");
    }
    *out = b;
    return LMGPU_OK;
}

int lmgpu_batch_destroy(LmgpuBatch* b)
{
    if (!b) return LMGPU_OK;
    drop_graphs(b);
    if (b->cap_stream) cudaStreamDestroy(b->cap_stream);
    for (cudaStream_t st : { b->cap_hi, b->cap_lo, b->hi, b->lo })
        if (st) cudaStreamDestroy(st);
    for (cudaEvent_t ev : b->ev)
        if (ev) cudaEventDestroy(ev);
    if (b->staged) cudaEventDestroy(b->staged);
    cudaFree(b->ws_mem);
    cudaFree(b->d_table);
    cudaFree(b->d_begins);
    cudaFree(b->d_wave);
    cudaFree(b->d_ctl);
    cudaFreeHost(b->h_done);
    cudaFree(b->d_stats);
    cudaFree(b->d_work);
    cudaFree(b->d_status);
    cudaFreeHost(b->h_table);
    cudaFreeHost(b->h_begins);
    cudaFreeHost(b->h_stats);
    cudaFreeHost(b->h_counts);
    cudaFree(b->hf_film);
    cudaFree(b->hf_out);
    cudaFreeHost(b->hf_pinned);
    delete b;
    return LMGPU_OK;
}

int lmgpu_batch_get_config(const LmgpuBatch* b, LmgpuBatchConfig* c)
{
    if (!b || !c) return fail(LMGPU_ERR_INVALID, "null argument");
    *c = b->cfg;
    return LMGPU_OK;
}

int lmgpu_batch_set_config(LmgpuBatch* b, const LmgpuBatchConfig* c)
{
    if (!b || !c) return fail(LMGPU_ERR_INVALID, "null argument");
    const int rc = check_config(*c);
    if (rc != LMGPU_OK) return rc;
    b->cfg = *c;
    b->cfg.use_graph = c->use_graph ? 1 : 0;
    return LMGPU_OK;
}

int lmgpu_batch_render_device(LmgpuBatch* b, const LmgpuRenderParams* params, void* const* films, void* stream,
                              LmgpuRenderStats* stats)
{
    if (!b || !params || !films) return fail(LMGPU_ERR_INVALID, "null argument");
    return batch_render(b, params, films, static_cast<cudaStream_t>(stream), stats);
}

int lmgpu_batch_render(LmgpuBatch* b, const LmgpuRenderParams* params, float* const* films_host,
                       LmgpuRenderStats* stats)
{
    if (!b || !params || !films_host) return fail(LMGPU_ERR_INVALID, "null argument");
    const size_t n = b->scenes.size();
    std::vector<int64_t> off(n + 1, 0);
    for (size_t i = 0; i < n; i++) {
        if (!films_host[i]) return fail(LMGPU_ERR_INVALID, "null film");
        const DeviceScene& d = b->scenes[i]->dev;
        off[i + 1] = off[i] + 3 * (int64_t)d.cam.width * d.cam.height;
    }
    const size_t esize = params[0].film_fp64 ? sizeof(double) : sizeof(float);
    const size_t film_bytes = (size_t)off[n] * esize, out_bytes = (size_t)off[n] * sizeof(float);
    if (b->hf_film_bytes < film_bytes) {
        cudaFree(b->hf_film);
        b->hf_film = nullptr;
        b->hf_film_bytes = 0;
        LMGPU_CUDA_TRY(cudaMalloc(&b->hf_film, film_bytes));
        b->hf_film_bytes = film_bytes;
    }
    if (b->hf_out_bytes < out_bytes) {
        cudaFree(b->hf_out);
        cudaFreeHost(b->hf_pinned);
        b->hf_out = nullptr;
        b->hf_pinned = nullptr;
        b->hf_out_bytes = 0;
        cudaError_t e = cudaMalloc(&b->hf_out, out_bytes);
        if (e == cudaSuccess) e = cudaMallocHost(&b->hf_pinned, out_bytes);
        if (e != cudaSuccess) {
            cudaFree(b->hf_out);
            b->hf_out = nullptr;
            b->hf_pinned = nullptr;
            return cuda_fail(e, "batch film buffers");
        }
        b->hf_out_bytes = out_bytes;
    }
    std::vector<void*> films(n);
    for (size_t i = 0; i < n; i++) films[i] = static_cast<char*>(b->hf_film) + (size_t)off[i] * esize;
    LMGPU_CUDA_TRY(cudaMemsetAsync(b->hf_film, 0, film_bytes, nullptr));
    LmgpuRenderStats local;
    int rc = batch_render(b, params, films.data(), nullptr, stats ? stats : &local);
    if (rc != LMGPU_OK) return rc;
    // Rescale(W * H / num_samples) per scene (sched.mt.cpp:250-256).
    for (size_t i = 0; i < n; i++) {
        const DeviceScene& d = b->scenes[i]->dev;
        const int64_t m = off[i + 1] - off[i];
        const double scale = double(d.cam.width) * d.cam.height / double(params[i].num_samples);
        const unsigned blocks = (unsigned)((m + 255) / 256);
        if (esize == sizeof(double))
            k_rescale_film<double><<<blocks, 256>>>(static_cast<const double*>(films[i]), b->hf_out + off[i], m, scale);
        else
            k_rescale_film<float><<<blocks, 256>>>(static_cast<const float*>(films[i]), b->hf_out + off[i], m, scale);
        LMGPU_CUDA_TRY(cudaGetLastError());
    }
    LMGPU_CUDA_TRY(cudaMemcpyAsync(b->hf_pinned, b->hf_out, out_bytes, cudaMemcpyDeviceToHost, nullptr));
    LMGPU_CUDA_TRY(cudaStreamSynchronize(nullptr));
    for (size_t i = 0; i < n; i++)
        std::memcpy(films_host[i], b->hf_pinned + off[i], (size_t)(off[i + 1] - off[i]) * sizeof(float));
    return LMGPU_OK;
}

int lmgpu_batch_profile(LmgpuBatch* b, const LmgpuRenderParams* params, void* const* films, void* stream,
                        int32_t count_tests, LmgpuTraceProfile* out)
{
    if (!b || !params || !films || !out) return fail(LMGPU_ERR_INVALID, "null argument");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    TraceProfileRun run;
    run.count = count_tests != 0;
    if (run.count) {
        LMGPU_CUDA_TRY(cudaMalloc(&run.d_counts, 4 * sizeof(unsigned long long)));
        cudaError_t e = cudaMemsetAsync(run.d_counts, 0, 4 * sizeof(unsigned long long), s);
        if (e != cudaSuccess) { cudaFree(run.d_counts); return cuda_fail(e, "profile counters"); }
    }
    const LmgpuBatchConfig saved = b->cfg;
    b->cfg.use_graph = 0;
    b->cfg.mode = LMGPU_BATCH_WAVES;
    b->prof = &run;
    LmgpuRenderStats st;
    std::memset(&st, 0, sizeof(st));
    int rc = batch_render(b, params, films, s, &st);
    b->prof = nullptr;
    b->cfg = saved;
    if (rc == LMGPU_OK && run.error != cudaSuccess) rc = cuda_fail(run.error, "profile events");
    std::memset(out, 0, sizeof(*out));
    out->rays[0] = st.rays_traced - st.shadow_rays;
    out->rays[1] = st.shadow_rays;
    out->render_ms = st.device_ms;
    for (size_t k = 0; k < run.kinds.size() && rc == LMGPU_OK; k++) {
        float ms = 0.0f;
        const cudaError_t e = cudaEventElapsedTime(&ms, run.events[2 * k], run.events[2 * k + 1]);
        if (e != cudaSuccess) { rc = cuda_fail(e, "profile event times"); break; }
        out->trace_ms[run.kinds[k]] += ms;
        out->launches[run.kinds[k]]++;
    }
    for (cudaEvent_t e : run.events) cudaEventDestroy(e);
    if (run.count) {
        unsigned long long h[4] = {};
        if (rc == LMGPU_OK) {
            const cudaError_t e = cudaMemcpy(h, run.d_counts, sizeof(h), cudaMemcpyDeviceToHost);
            if (e != cudaSuccess) rc = cuda_fail(e, "profile counters");
        }
        out->node_tests[0] = h[0]; out->tri_tests[0] = h[1];
        out->node_tests[1] = h[2]; out->tri_tests[1] = h[3];
        cudaFree(run.d_counts);
    }
    return rc;
}

int lmgpu_batch_autotune(LmgpuBatch* b, const LmgpuRenderParams* params, double fraction, void* stream,
                         LmgpuBatchConfig* chosen, double* best_ms)
{
    if (!b || !params) return fail(LMGPU_ERR_INVALID, "null argument");
    if (!(fraction > 0.0 && fraction <= 1.0)) return fail(LMGPU_ERR_INVALID, "sample_fraction must be in (0, 1]");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const size_t n = b->scenes.size();
    // Scaled budgets, one scratch film shared by all scenes (its contents are discarded).
    std::vector<LmgpuRenderParams> p(params, params + n);
    auto scale = [&](double f) {
        int64_t t = 0;
        for (size_t i = 0; i < n; i++) {
            p[i].num_samples = std::max<int64_t>(1, (int64_t)std::llround((double)params[i].num_samples * f));
            t += p[i].num_samples;
        }
        return t;
    };
    int64_t px = 0, full = 0;
    for (size_t i = 0; i < n; i++) {
        full += params[i].num_samples;
        px = std::max<int64_t>(px, (int64_t)b->scenes[i]->dev.cam.width * b->scenes[i]->dev.cam.height);
    }
    const int64_t total = scale(fraction);
    Plan pl;
    int rc = make_plan(b, p.data(), nullptr, pl);
    if (rc != LMGPU_OK) return rc;
    void* film = nullptr;
    const size_t esize = pl.fp64 ? sizeof(double) : sizeof(float);
    LMGPU_CUDA_TRY(cudaMalloc(&film, std::max<int64_t>(px, 1) * 3 * esize));
    std::vector<void*> films(n, film);

    const LmgpuBatchConfig start = b->cfg;
    // A candidate is timed on at least four of its own waves (or the whole
    // render), so that large waves are not judged on a render that one wave
    // holds, and is compared by device time per sample. Overlap mode gets
    // four of its periods (eight waves): its first head and last tail run
    // alone, and on a four-wave trial of the 64-scene batch that hid its
    // gain (overlap 780 ms, fixed waves 816 ms on the whole batch).
    auto trial = [&](const LmgpuBatchConfig& c, double& ms_per_sample) -> int {
        int r = check_config(c);
        if (r != LMGPU_OK) return r;
        ms_per_sample = 1e30;
        b->cfg = c;
        const double waves_needed = c.mode == LMGPU_BATCH_OVERLAP ? 8.0 : 4.0;
        const double f = std::min(1.0, std::max(fraction, waves_needed * (double)c.wave_paths / (double)full));
        const int64_t samples = scale(f);
        LmgpuRenderStats st;
        if ((r = batch_render(b, p.data(), films.data(), s, &st)) != LMGPU_OK) return r;   // warm-up (capture)
        double best = 1e30;
        for (int k = 0; k < 2; k++) {
            if ((r = batch_render(b, p.data(), films.data(), s, &st)) != LMGPU_OK) return r;
            best = std::min(best, st.device_ms);
        }
        ms_per_sample = best / (double)samples;
        return LMGPU_OK;
    };
    // A candidate replaces the incumbent only if it is more than 0.5 % faster:
    // trial-to-trial noise is ~0.3 %, and without the margin the descent
    // drifted from the defaults on ties (for the 1080p frame into waves of
    // 2^26 paths, 0.3 % slower in the timed frames).
    auto better = [](double t, double incumbent) { return t < incumbent * 0.995; };
    LmgpuBatchConfig best = start;
    best.use_graph = 1;
    double best_t = 1e30;
    rc = trial(best, best_t);
    // Coordinate descent: mode, layout, then paths in flight, shading grid
    // and (overlap mode) the first tail bounce.
    for (int m : { LMGPU_BATCH_WAVES, LMGPU_BATCH_STREAM, LMGPU_BATCH_OVERLAP }) {
        if (rc != LMGPU_OK || m == best.mode) continue;
        LmgpuBatchConfig c = best;
        c.mode = m;
        double t;
        if ((rc = trial(c, t)) == LMGPU_OK && better(t, best_t)) { best = c; best_t = t; }
    }
    const int layouts[] = { LMGPU_LAYOUT_BVH2, LMGPU_LAYOUT_BVH4, LMGPU_LAYOUT_BVH2Q, LMGPU_LAYOUT_BVH2_QSHADOW };
    const int waves[] = { 1 << 21, 1 << 22, 1 << 23, 1 << 24, 1 << 25, 1 << 26, 1 << 27 };
    const int grids[] = { 4, 8, 16 };
    for (int l : layouts) {
        if (rc != LMGPU_OK || l == best.layout) continue;
        LmgpuBatchConfig c = best;
        c.layout = l;
        double t;
        if ((rc = trial(c, t)) == LMGPU_OK && better(t, best_t)) { best = c; best_t = t; }
    }
    int64_t largest = 0;
    for (int w : waves) {
        // Waves beyond the sample count behave like a wave of the sample count.
        if (rc != LMGPU_OK || w == best.wave_paths || (w > full && largest >= full)) continue;
        largest = std::max<int64_t>(largest, w);
        LmgpuBatchConfig c = best;
        c.wave_paths = w;
        double t;
        if ((rc = trial(c, t)) == LMGPU_OK && better(t, best_t)) { best = c; best_t = t; }
    }
    for (int g : grids) {
        if (rc != LMGPU_OK || g == best.shade_blocks_per_sm) continue;
        LmgpuBatchConfig c = best;
        c.shade_blocks_per_sm = g;
        double t;
        if ((rc = trial(c, t)) == LMGPU_OK && better(t, best_t)) { best = c; best_t = t; }
    }
    if (best.mode == LMGPU_BATCH_OVERLAP) {
        const int current = best.overlap_bounce > 0 ? best.overlap_bounce : DEFAULT_OVERLAP_BOUNCE;
        for (int t0 : { 2, 3, 4, 5 }) {
            if (rc != LMGPU_OK || t0 == current) continue;
            LmgpuBatchConfig c = best;
            c.overlap_bounce = t0;
            double t;
            if ((rc = trial(c, t)) == LMGPU_OK && better(t, best_t)) { best = c; best_t = t; }
        }
    }
    cudaFree(film);
    b->cfg = rc == LMGPU_OK ? best : start;
    if (rc != LMGPU_OK) return rc;
    if (chosen) *chosen = best;
    if (best_ms) *best_ms = best_t * (double)total;
    return LMGPU_OK;
}

}  // extern "C"
