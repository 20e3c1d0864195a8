// Host scene builder. Compiled by g++ with -ffp-contract=off so that every
// float operation rounds separately, as in the reference's float SSE build.
//
// Reference algorithms restated here (own code, same steps):
//   vertex transform    Mat4f * Vec4f, math.matrix.inl:692-702
//   TriAccel::Load      triaccel.h:57-98
//   BVHScene::Build     scene.bvh.cpp:202-388 (12-bucket binned SAH, cost
//                       0.125 + (n1 A1 + n2 A2) / A, leaf if cost >= n and
//                       n <= 255, 1-triangle and degenerate-centroid leaves)
// The tree is built in parallel over subtrees; its shape does not depend on
// the threading (every node's split is a function of its triangle set only).
#include "builder.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cfloat>
#include <cstring>
#include <functional>
#include <limits>
#include <thread>

namespace lmgpu {
namespace {

// _mm_min_ps / _mm_max_ps semantics (second operand unless strictly smaller).
inline float min_sse(float a, float b) { return a < b ? a : b; }
inline float max_sse(float a, float b) { return a > b ? a : b; }

inline HostAabb aabb_empty()
{
    HostAabb b;
    for (int i = 0; i < 3; i++) { b.mn[i] = FLT_MAX; b.mx[i] = -FLT_MAX; }
    return b;
}
inline void aabb_grow(HostAabb& a, const HostAabb& b)
{
    for (int i = 0; i < 3; i++) { a.mn[i] = min_sse(a.mn[i], b.mn[i]); a.mx[i] = max_sse(a.mx[i], b.mx[i]); }
}
inline void aabb_grow_p(HostAabb& a, const float* p)
{
    for (int i = 0; i < 3; i++) { a.mn[i] = min_sse(a.mn[i], p[i]); a.mx[i] = max_sse(a.mx[i], p[i]); }
}
inline float aabb_area(const HostAabb& b)
{
    float dx = b.mx[0] - b.mn[0], dy = b.mx[1] - b.mn[1], dz = b.mx[2] - b.mn[2];
    float s = dx * dy;
    s = s + dy * dz;
    s = s + dz * dx;
    return 2.0f * s;
}
inline int aabb_longest(const HostAabb& b)
{
    float dx = b.mx[0] - b.mn[0], dy = b.mx[1] - b.mn[1], dz = b.mx[2] - b.mn[2];
    return (dx > dy && dx > dz) ? 0 : (dy > dz ? 1 : 2);
}

// Column-major 4x4 times (x, y, z, 1) in the SSE order (c0 x + c1 y) + (c2 z + c3).
inline void xform_point(const float* m, const float* p, float* out)
{
    for (int r = 0; r < 3; r++) {
        float a = m[0 + r] * p[0];
        float b = m[4 + r] * p[1];
        float c = m[8 + r] * p[2];
        float d = m[12 + r] * 1.0f;
        float ab = a + b;
        float cd = c + d;
        out[r] = ab + cd;
    }
}

// TriAccel constants in the reference's evaluation order.
void load_triaccel(TriRecord& t, const float* A, const float* B, const float* C)
{
    static const int wald_modulo[4] = { 1, 2, 0, 1 };
    float b[3], c[3], N[3];
    for (int i = 0; i < 3; i++) { b[i] = C[i] - A[i]; c[i] = B[i] - A[i]; }
    N[0] = c[1] * b[2] - c[2] * b[1];
    N[1] = c[2] * b[0] - c[0] * b[2];
    N[2] = c[0] * b[1] - c[1] * b[0];
    uint32_t k = 0;
    for (int j = 0; j < 3; j++)
        if (std::fabs(N[j]) > std::fabs(N[k])) k = static_cast<uint32_t>(j);
    const int u = wald_modulo[k], v = wald_modulo[k + 1];
    const float n_k = N[k];
    const float denom = b[u] * c[v] - b[v] * c[u];
    std::memset(&t, 0, sizeof(t));
    if (denom == 0.0f) { t.k_flags = 3; return; }
    t.k_flags = k;
    t.n_u = N[u] / n_k;
    t.n_v = N[v] / n_k;
    float dot = A[0] * N[0] + A[1] * N[1];
    dot = dot + A[2] * N[2];
    t.n_d = dot / n_k;
    t.b_nu = b[u] / denom;
    t.b_nv = -b[v] / denom;
    t.a_u = A[u];
    t.a_v = A[v];
    t.c_nu = c[v] / denom;
    t.c_nv = -c[u] / denom;
}

struct Builder {
    BuiltScene& s;
    std::vector<HostAabb> tri_bounds;
    std::vector<float> centroids;
    std::vector<BuildNode> pool;
    std::atomic<int32_t> pool_next{0};
    std::atomic<int64_t> leaves{0};
    std::atomic<int32_t> depth{0};
    int spawn_depth = 0;

    explicit Builder(BuiltScene& out) : s(out) {}

    int32_t alloc_node() { return pool_next.fetch_add(1); }

    inline int bucket_of(int32_t tri, int axis, const HostAabb& cb) const
    {
        float c = centroids[3 * (size_t)tri + axis];
        float num = c - cb.mn[axis];
        float den = cb.mx[axis] - cb.mn[axis];
        float x = 12.0f * (num / den);
        int b = static_cast<int>(x);
        return b < 11 ? b : 11;
    }

    int32_t make_leaf(int begin, int end, const HostAabb& bound)
    {
        int32_t id = alloc_node();
        BuildNode& n = pool[id];
        n.leaf = true; n.begin = begin; n.end = end; n.bound = bound;
        leaves.fetch_add(1);
        return id;
    }

    int32_t build(int begin, int end, int d)
    {
        int32_t cur = depth.load();
        while (d > cur && !depth.compare_exchange_weak(cur, d)) {}
        int32_t* order = s.tri_order.data();
        HostAabb bound = aabb_empty();
        for (int i = begin; i < end; i++) aabb_grow(bound, tri_bounds[order[i]]);
        const int n = end - begin;
        if (n == 1) return make_leaf(begin, end, bound);

        HostAabb cb = aabb_empty();
        for (int i = begin; i < end; i++) aabb_grow_p(cb, &centroids[3 * (size_t)order[i]]);
        const int axis = aabb_longest(cb);
        if (cb.mn[axis] == cb.mx[axis]) return make_leaf(begin, end, bound);

        HostAabb bb[12];
        int bc[12];
        for (int i = 0; i < 12; i++) { bb[i] = aabb_empty(); bc[i] = 0; }
        for (int i = begin; i < end; i++) {
            const int32_t t = order[i];
            const int b = bucket_of(t, axis, cb);
            bc[b]++;
            aabb_grow(bb[b], tri_bounds[t]);
        }
        // Prefix/suffix sweeps give the same unions as the reference's
        // per-split loops: min/max are exact and order-independent.
        HostAabb left[11], right[11];
        int lc[11], rc[11];
        {
            HostAabb acc = aabb_empty(); int c = 0;
            for (int i = 0; i < 11; i++) { aabb_grow(acc, bb[i]); c += bc[i]; left[i] = acc; lc[i] = c; }
            acc = aabb_empty(); c = 0;
            for (int i = 11; i >= 1; i--) { aabb_grow(acc, bb[i]); c += bc[i]; right[i - 1] = acc; rc[i - 1] = c; }
        }
        const float area = aabb_area(bound);
        float costs[11];
        for (int i = 0; i < 11; i++) {
            float num = static_cast<float>(lc[i]) * aabb_area(left[i]) + static_cast<float>(rc[i]) * aabb_area(right[i]);
            costs[i] = 0.125f + num / area;
        }
        int min_idx = 0;
        double min_cost = costs[0];
        for (int i = 1; i < 11; i++)
            if (min_cost > costs[i]) { min_cost = costs[i]; min_idx = i; }

        if (min_cost < static_cast<float>(n) || n > 255) {
            // Two-pointer (Hoare) partition, the algorithm of std::partition
            // on bidirectional iterators: same leaf order as the reference.
            int first = begin, last = end;
            for (;;) {
                while (first != last && bucket_of(order[first], axis, cb) <= min_idx) ++first;
                if (first == last) break;
                --last;
                while (first != last && !(bucket_of(order[last], axis, cb) <= min_idx)) --last;
                if (first == last) break;
                std::swap(order[first], order[last]);
                ++first;
            }
            const int mid = first;
            int32_t l, r;
            if (d < spawn_depth && n > 4096) {
                int32_t lres = -1;
                std::thread th([&] { lres = build(begin, mid, d + 1); });
                r = build(mid, end, d + 1);
                th.join();
                l = lres;
            } else {
                l = build(begin, mid, d + 1);
                r = build(mid, end, d + 1);
            }
            int32_t id = alloc_node();
            BuildNode& nd = pool[id];
            nd.leaf = false; nd.axis = axis; nd.left = l; nd.right = r;
            nd.bound = pool[l].bound;
            aabb_grow(nd.bound, pool[r].bound);
            return id;
        }
        return make_leaf(begin, end, bound);
    }
};

// DFS pre-order flatten into Bvh2Node (internal nodes only).
int32_t flatten_bvh2(const std::vector<BuildNode>& nodes, int32_t ni, std::vector<Bvh2Node>& out)
{
    const BuildNode& n = nodes[ni];
    if (n.leaf) return ~n.begin;
    const int32_t id = static_cast<int32_t>(out.size());
    out.emplace_back();
    const BuildNode& L = nodes[n.left];
    const BuildNode& R = nodes[n.right];
    {
        Bvh2Node& o = out[id];
        o.bx[0] = L.bound.mn[0]; o.bx[1] = L.bound.mx[0]; o.bx[2] = R.bound.mn[0]; o.bx[3] = R.bound.mx[0];
        o.by[0] = L.bound.mn[1]; o.by[1] = L.bound.mx[1]; o.by[2] = R.bound.mn[1]; o.by[3] = R.bound.mx[1];
        o.bz[0] = L.bound.mn[2]; o.bz[1] = L.bound.mx[2]; o.bz[2] = R.bound.mn[2]; o.bz[3] = R.bound.mx[2];
        o.axis = n.axis;
        o.pad = 0;
    }
    const int32_t l = flatten_bvh2(nodes, n.left, out);
    const int32_t r = flatten_bvh2(nodes, n.right, out);
    out[id].left = l;
    out[id].right = r;
    return id;
}

// 4-wide collapse: each 4-node holds the (up to) four grandchildren of a
// binary internal node; a binary child that is a leaf occupies its slot pair
// alone.
int32_t flatten_bvh4(const std::vector<BuildNode>& nodes, int32_t ni, std::vector<Bvh4Node>& out)
{
    const BuildNode& n = nodes[ni];
    if (n.leaf) return ~n.begin;
    const int32_t id = static_cast<int32_t>(out.size());
    out.emplace_back();
    int32_t slot_node[4] = { -1, -1, -1, -1 };
    int32_t axis_pair[2] = { -1, -1 };
    const int32_t kids[2] = { n.left, n.right };
    for (int p = 0; p < 2; p++) {
        const BuildNode& c = nodes[kids[p]];
        if (c.leaf) { slot_node[2 * p] = kids[p]; }
        else { slot_node[2 * p] = c.left; slot_node[2 * p + 1] = c.right; axis_pair[p] = c.axis; }
    }
    {
        Bvh4Node& o = out[id];
        for (int k = 0; k < 4; k++) {
            if (slot_node[k] < 0) {
                // Empty slot: a box no ray can enter (lo > hi on every axis).
                o.lox[k] = o.loy[k] = o.loz[k] = FLT_MAX;
                o.hix[k] = o.hiy[k] = o.hiz[k] = -FLT_MAX;
                o.child[k] = BVH4_EMPTY;
                continue;
            }
            const HostAabb& b = nodes[slot_node[k]].bound;
            o.lox[k] = b.mn[0]; o.hix[k] = b.mx[0];
            o.loy[k] = b.mn[1]; o.hiy[k] = b.mx[1];
            o.loz[k] = b.mn[2]; o.hiz[k] = b.mx[2];
        }
        o.axis_top = n.axis;
        o.axis_l = axis_pair[0];
        o.axis_r = axis_pair[1];
        o.pad = 0;
    }
    for (int k = 0; k < 4; k++)
        if (slot_node[k] >= 0) out[id].child[k] = flatten_bvh4(nodes, slot_node[k], out);
    return id;
}

// ------------------------------------------------------------ render tree

// Render tree: binned SAH over all three axes (the reference bins only the
// longest axis of the centroid bounds, into 12 buckets), cost
// RTREE_NODE_COST + (nL AL + nR AR) / A in units of one triangle test
// against a leaf's n, leaves of at most RTREE_MAX_LEAF triangles (unless
// their centroids coincide).
#ifndef LMGPU_RTREE_BINS
#define LMGPU_RTREE_BINS 32
#endif
#ifndef LMGPU_RTREE_NODE_COST
#define LMGPU_RTREE_NODE_COST 0.5f    // a node visit costs about half a triangle test (measured)
#endif
#ifndef LMGPU_RTREE_MAX_LEAF
#define LMGPU_RTREE_MAX_LEAF 8
#endif

struct RenderBuilder {
    static constexpr int NB = LMGPU_RTREE_BINS;
    const std::vector<HostAabb>& tri_bounds;
    const std::vector<float>& centroids;
    std::vector<int32_t> order;
    std::vector<BuildNode> pool;
    std::atomic<int32_t> pool_next{0};
    std::atomic<int64_t> leaves{0};
    std::atomic<int32_t> depth{0};
    int spawn_depth = 0;

    RenderBuilder(const std::vector<HostAabb>& tb, const std::vector<float>& c) : tri_bounds(tb), centroids(c) {}

    int32_t alloc_node() { return pool_next.fetch_add(1); }

    int32_t make_leaf(int begin, int end, const HostAabb& bound)
    {
        int32_t id = alloc_node();
        BuildNode& n = pool[id];
        n.leaf = true; n.begin = begin; n.end = end; n.bound = bound;
        leaves.fetch_add(1);
        return id;
    }

    static int bin_of(float c, float lo, float scale)
    {
        const int b = static_cast<int>((c - lo) * scale);
        return b < 0 ? 0 : (b >= NB ? NB - 1 : b);
    }

    int32_t build(int begin, int end, int d)
    {
        int32_t cur = depth.load();
        while (d > cur && !depth.compare_exchange_weak(cur, d)) {}
        HostAabb bound = aabb_empty(), cb = aabb_empty();
        for (int i = begin; i < end; i++) {
            aabb_grow(bound, tri_bounds[order[i]]);
            aabb_grow_p(cb, &centroids[3 * (size_t)order[i]]);
        }
        const int n = end - begin;
        if (n == 1) return make_leaf(begin, end, bound);
        const float area = aabb_area(bound);
        float best = FLT_MAX;
        int best_axis = -1, best_bin = 0;
        for (int axis = 0; axis < 3; axis++) {
            const float lo = cb.mn[axis], ext = cb.mx[axis] - cb.mn[axis];
            if (!(ext > 0.0f)) continue;
            const float scale = float(NB) / ext;
            HostAabb bb[NB];
            int bc[NB];
            for (int i = 0; i < NB; i++) { bb[i] = aabb_empty(); bc[i] = 0; }
            for (int i = begin; i < end; i++) {
                const int32_t t = order[i];
                const int b = bin_of(centroids[3 * (size_t)t + axis], lo, scale);
                bc[b]++;
                aabb_grow(bb[b], tri_bounds[t]);
            }
            float right_area[NB];
            int right_count[NB];
            HostAabb acc = aabb_empty();
            int c = 0;
            for (int i = NB - 1; i >= 1; i--) {
                aabb_grow(acc, bb[i]);
                c += bc[i];
                right_area[i] = aabb_area(acc);
                right_count[i] = c;
            }
            acc = aabb_empty();
            c = 0;
            for (int i = 0; i < NB - 1; i++) {         // split after bin i
                aabb_grow(acc, bb[i]);
                c += bc[i];
                if (c == 0 || right_count[i + 1] == 0) continue;
                const float cost = LMGPU_RTREE_NODE_COST +
                                   (float(c) * aabb_area(acc) + float(right_count[i + 1]) * right_area[i + 1]) / area;
                if (cost < best) { best = cost; best_axis = axis; best_bin = i; }
            }
        }
        if (best_axis < 0 || (n <= LMGPU_RTREE_MAX_LEAF && float(n) <= best)) return make_leaf(begin, end, bound);
        const float lo = cb.mn[best_axis], scale = float(NB) / (cb.mx[best_axis] - cb.mn[best_axis]);
        int32_t* o = order.data();
        const int32_t* mid_ptr = std::partition(o + begin, o + end, [&](int32_t t) {
            return bin_of(centroids[3 * (size_t)t + best_axis], lo, scale) <= best_bin;
        });
        const int mid = static_cast<int>(mid_ptr - o);
        int32_t l, r;
        if (d < spawn_depth && n > 4096) {
            int32_t lres = -1;
            std::thread th([&] { lres = build(begin, mid, d + 1); });
            r = build(mid, end, d + 1);
            th.join();
            l = lres;
        } else {
            l = build(begin, mid, d + 1);
            r = build(mid, end, d + 1);
        }
        int32_t id = alloc_node();
        BuildNode& nd = pool[id];
        nd.leaf = false; nd.axis = best_axis; nd.left = l; nd.right = r;
        nd.bound = pool[l].bound;
        aabb_grow(nd.bound, pool[r].bound);
        return id;
    }
};

}  // namespace

std::vector<Bvh2QNode> quantize_bvh2(const std::vector<Bvh2Node>& nodes, const HostAabb& bounds,
                                     const float* extra)
{
    double M = 0.0;
    for (int c = 0; c < 3; c++) {
        M = std::max(M, (double)std::fabs(bounds.mn[c]));
        M = std::max(M, (double)std::fabs(bounds.mx[c]));
        if (extra) M = std::max(M, (double)std::fabs(extra[c]));
    }
    // 16 ulps of the largest magnitude a ray origin or a plane takes
    const double min_step = 16.0 * (M > 0.0 ? std::ldexp(1.0, std::ilogb(M) - 23) : std::ldexp(1.0, -126));
    std::vector<Bvh2QNode> out(nodes.size());
    for (size_t i = 0; i < nodes.size(); i++) {
        const Bvh2Node& n = nodes[i];
        const float* ax[3] = { n.bx, n.by, n.bz };
        Bvh2QNode& o = out[i];
        uint32_t exps = (uint32_t)(n.axis & 0xff) << 24;
        for (int k = 0; k < 3; k++) {
            const double lo = std::min(ax[k][0], ax[k][2]), hi = std::max(ax[k][1], ax[k][3]);
            // 65,520 steps cover the box, its two-step margins and the
            // origin's rounding; a power of two, so q * step is exact.
            const double need = std::max(min_step, (hi - lo) / 65520.0);
            int E = std::ilogb(need);
            if (std::ldexp(1.0, E) < need) E++;
            E = std::min(std::max(E, -126), 127);
            const double step = std::ldexp(1.0, E);
            const double od = lo - 2.0 * step;
            float of = (float)od;
            if ((double)of > od) of = std::nextafter(of, -std::numeric_limits<float>::infinity());
            o.origin[k] = of;
            for (int c = 0; c < 2; c++) {
                const double clo = ax[k][2 * c], chi = ax[k][2 * c + 1];
                const double qlo = std::max(0.0, std::floor((clo - (double)of) / step) - 2.0);
                const double qhi = std::min(65535.0, std::ceil((chi - (double)of) / step) + 2.0);
                o.q[2 * k + c] = (uint32_t)qlo | ((uint32_t)qhi << 16);
            }
            exps |= (uint32_t)(E + 127) << (8 * k);
        }
        o.exps = exps;
        o.left = n.left;
        o.right = n.right;
    }
    return out;
}

void build_render_tree(BuiltScene& s, int threads)
{
    auto t0 = std::chrono::steady_clock::now();
    const int64_t ntris = s.num_tris;
    if (ntris <= 0) return;
    std::vector<HostAabb> tb((size_t)ntris);
    std::vector<float> cen(3 * (size_t)ntris);
    for (int64_t t = 0; t < ntris; t++) {
        const float* p1 = &s.positions[3 * (size_t)s.tri_vidx[3 * t]];
        const float* p2 = &s.positions[3 * (size_t)s.tri_vidx[3 * t + 1]];
        const float* p3 = &s.positions[3 * (size_t)s.tri_vidx[3 * t + 2]];
        HostAabb b;
        for (int c = 0; c < 3; c++) { b.mn[c] = min_sse(p1[c], p2[c]); b.mx[c] = max_sse(p1[c], p2[c]); }
        aabb_grow_p(b, p3);
        tb[(size_t)t] = b;
        for (int c = 0; c < 3; c++) cen[3 * (size_t)t + c] = (b.mn[c] + b.mx[c]) * 0.5f;
    }
    RenderBuilder B(tb, cen);
    B.order.resize((size_t)ntris);
    for (int64_t t = 0; t < ntris; t++) B.order[(size_t)t] = static_cast<int32_t>(t);
    if (threads <= 0) threads = static_cast<int>(std::max(1u, std::thread::hardware_concurrency()));
    while ((1 << B.spawn_depth) < threads) B.spawn_depth++;
    B.spawn_depth += 1;
    B.pool.resize(2 * (size_t)ntris);
    const int32_t root = B.build(0, static_cast<int32_t>(ntris), 0);
    B.pool.resize((size_t)B.pool_next.load());
    // Records in the render tree's leaf order: the same TriAccel constants.
    std::vector<TriRecord> by_id((size_t)ntris);
    for (int64_t i = 0; i < ntris; i++) by_id[s.tris[(size_t)i].tri_id] = s.tris[(size_t)i];
    s.rtris.resize((size_t)ntris);
    for (int64_t i = 0; i < ntris; i++) {
        s.rtris[(size_t)i] = by_id[(size_t)B.order[(size_t)i]];
        s.rtris[(size_t)i].k_flags &= ~TRI_LAST_IN_LEAF;
    }
    for (auto& n : B.pool)
        if (n.leaf) s.rtris[(size_t)(n.end - 1)].k_flags |= TRI_LAST_IN_LEAF;
    s.rbvh2.clear();
    s.rbvh2.reserve((size_t)std::max<int64_t>(1, ntris));
    s.rbvh2_root = flatten_bvh2(B.pool, root, s.rbvh2);
    s.rbvh4.clear();
    s.rbvh4_root = flatten_bvh4(B.pool, root, s.rbvh4);
    const HostAabb& rb = B.pool[root].bound;
    for (int c = 0; c < 3; c++) { s.rroot_box[c] = rb.mn[c]; s.rroot_box[3 + c] = rb.mx[c]; }
    s.rnum_nodes = (int64_t)B.pool.size();
    s.rnum_leaves = B.leaves.load();
    s.rmax_depth = B.depth.load();
    s.has_render_tree = true;
    s.rbuild_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

std::string build_scene(const std::vector<PrimitiveInput>& prims, int threads, bool want_bvh, BuiltScene& s)
{
    auto t0 = std::chrono::steady_clock::now();
    static const float identity[16] = { 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1 };

    // ---- world-space geometry and TriAccel records (primitive-major order)
    int64_t ntris = 0, nverts = 0;
    for (auto& p : prims) {
        if (p.num_faces < 0 || p.num_vertices < 0) return "negative primitive size";
        if (p.num_faces > 0 && (!p.positions || !p.faces)) return "primitive without positions or faces";
        ntris += p.num_faces;
        nverts += p.num_vertices;
    }
    if (ntris >= (int64_t(1) << 31) - 1) return "too many triangles";
    s.num_tris = ntris;
    s.positions.resize(3 * (size_t)nverts);
    s.normals.resize(3 * (size_t)nverts);
    s.texcoords.assign(2 * (size_t)nverts, 0.0f);
    s.tri_vidx.resize(3 * (size_t)ntris);
    s.tri_prim.resize((size_t)ntris);
    s.has_uv.resize(prims.size());
    std::vector<TriRecord> ta((size_t)ntris);
    s.bounds = aabb_empty();

    int64_t vbase = 0, tbase = 0;
    for (size_t pi = 0; pi < prims.size(); pi++) {
        const PrimitiveInput& p = prims[pi];
        const float* m = p.transform ? p.transform : identity;
        s.has_uv[pi] = p.texcoords != nullptr;
        // Normal transform: transpose(inverse(M)) upper 3x3 (primitive.h:42-44).
        double inv[9];
        {
            const double a = m[0], b = m[4], c = m[8], d = m[1], e = m[5], f = m[9], g = m[2], h = m[6], i = m[10];
            const double det = a * (e * i - f * h) - b * (d * i - f * g) + c * (d * h - e * g);
            const double id = det != 0.0 ? 1.0 / det : 0.0;
            // inverse (row-major r,c) then transposed => normal matrix N[r][c] = inv[c][r]
            const double I[3][3] = {
                { (e * i - f * h) * id, (c * h - b * i) * id, (b * f - c * e) * id },
                { (f * g - d * i) * id, (a * i - c * g) * id, (c * d - a * f) * id },
                { (d * h - e * g) * id, (b * g - a * h) * id, (a * e - b * d) * id } };
            for (int r = 0; r < 3; r++)
                for (int c2 = 0; c2 < 3; c2++) inv[3 * r + c2] = I[c2][r];
        }
        for (int v = 0; v < p.num_vertices; v++) {
            float w[3];
            xform_point(m, p.positions + 3 * (size_t)v, w);
            std::memcpy(&s.positions[3 * (size_t)(vbase + v)], w, sizeof(w));
            float nn[3] = { 0, 0, 0 };
            if (p.normals) {
                const float* n0 = p.normals + 3 * (size_t)v;
                for (int r = 0; r < 3; r++)
                    nn[r] = static_cast<float>(inv[3 * r] * n0[0] + inv[3 * r + 1] * n0[1] + inv[3 * r + 2] * n0[2]);
            }
            std::memcpy(&s.normals[3 * (size_t)(vbase + v)], nn, sizeof(nn));
            if (p.texcoords) {
                s.texcoords[2 * (size_t)(vbase + v)] = p.texcoords[2 * (size_t)v];
                s.texcoords[2 * (size_t)(vbase + v) + 1] = p.texcoords[2 * (size_t)v + 1];
            }
        }
        for (int f = 0; f < p.num_faces; f++) {
            const int64_t t = tbase + f;
            uint32_t vi[3];
            for (int c = 0; c < 3; c++) {
                vi[c] = p.faces[3 * (size_t)f + c];
                if ((int64_t)vi[c] >= p.num_vertices) return "face index out of range";
                s.tri_vidx[3 * (size_t)t + c] = static_cast<uint32_t>(vbase + vi[c]);
            }
            s.tri_prim[(size_t)t] = static_cast<int32_t>(pi);
            const float* A = &s.positions[3 * (size_t)(vbase + vi[0])];
            const float* B = &s.positions[3 * (size_t)(vbase + vi[1])];
            const float* C = &s.positions[3 * (size_t)(vbase + vi[2])];
            load_triaccel(ta[(size_t)t], A, B, C);
            ta[(size_t)t].tri_id = static_cast<uint32_t>(t);
            ta[(size_t)t].prim = static_cast<uint32_t>(pi);
            // Geometric normal stands in for missing vertex normals.
            if (!p.normals) {
                float e1[3], e2[3], g[3];
                for (int c = 0; c < 3; c++) { e1[c] = B[c] - A[c]; e2[c] = C[c] - A[c]; }
                g[0] = e1[1] * e2[2] - e1[2] * e2[1];
                g[1] = e1[2] * e2[0] - e1[0] * e2[2];
                g[2] = e1[0] * e2[1] - e1[1] * e2[0];
                for (int c = 0; c < 3; c++)
                    for (int k = 0; k < 3; k++) s.normals[3 * (size_t)(vbase + vi[c]) + k] = g[k];
            }
        }
        vbase += p.num_vertices;
        tbase += p.num_faces;
    }

    // ---- bounds, centroids, BVH
    Builder B(s);
    B.tri_bounds.resize((size_t)ntris);
    B.centroids.resize(3 * (size_t)ntris);
    s.tri_order.resize((size_t)ntris);
    for (int64_t t = 0; t < ntris; t++) {
        const float* p1 = &s.positions[3 * (size_t)s.tri_vidx[3 * t]];
        const float* p2 = &s.positions[3 * (size_t)s.tri_vidx[3 * t + 1]];
        const float* p3 = &s.positions[3 * (size_t)s.tri_vidx[3 * t + 2]];
        HostAabb tb;
        for (int c = 0; c < 3; c++) { tb.mn[c] = min_sse(p1[c], p2[c]); tb.mx[c] = max_sse(p1[c], p2[c]); }
        aabb_grow_p(tb, p3);
        aabb_grow(s.bounds, tb);
        B.tri_bounds[(size_t)t] = tb;
        for (int c = 0; c < 3; c++) B.centroids[3 * (size_t)t + c] = (tb.mn[c] + tb.mx[c]) * 0.5f;
        s.tri_order[(size_t)t] = static_cast<int32_t>(t);
    }

    if (threads <= 0) threads = static_cast<int>(std::max(1u, std::thread::hardware_concurrency()));
    while ((1 << B.spawn_depth) < threads) B.spawn_depth++;
    B.spawn_depth += 1;

    if (want_bvh && ntris > 0) {
        B.pool.resize(2 * (size_t)ntris);
        const int32_t root = B.build(0, static_cast<int32_t>(ntris), 0);
        B.pool.resize((size_t)B.pool_next.load());
        s.nodes.swap(B.pool);
        s.root = root;
        s.num_leaves = B.leaves.load();
        s.max_depth = B.depth.load();
    }

    // ---- device layouts
    s.tris.resize((size_t)ntris);
    for (int64_t i = 0; i < ntris; i++) s.tris[(size_t)i] = ta[(size_t)s.tri_order[(size_t)i]];
    if (want_bvh && ntris > 0) {
        for (auto& n : s.nodes)
            if (n.leaf) s.tris[(size_t)(n.end - 1)].k_flags |= TRI_LAST_IN_LEAF;
        s.bvh2.reserve((size_t)std::max<int64_t>(1, ntris));
        s.bvh2_root = flatten_bvh2(s.nodes, s.root, s.bvh2);
        s.bvh4.reserve((size_t)std::max<int64_t>(1, ntris / 2));
        s.bvh4_root = flatten_bvh4(s.nodes, s.root, s.bvh4);
        const HostAabb& rb = s.nodes[s.root].bound;
        for (int c = 0; c < 3; c++) { s.root_box[c] = rb.mn[c]; s.root_box[3 + c] = rb.mx[c]; }
        s.max_stack = s.max_depth + 2;
    } else if (ntris > 0) {
        s.tris[(size_t)(ntris - 1)].k_flags |= TRI_LAST_IN_LEAF;
    }
    s.build_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return std::string();
}

}  // namespace lmgpu
