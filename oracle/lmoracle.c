/*
 * ORACLE — test infrastructure, not product code (see lmoracle.h).
 *
 * Restates, in plain C99 single precision, the reference's
 *   - TriAccel::Load / TriAccel::Intersect   include/lightmetrica/triaccel.h:57-160
 *   - BVHScene::Build / recursive Build      src/liblightmetrica/scene.bvh.cpp:202-388
 *   - CompareToBucket                        src/liblightmetrica/scene.bvh.cpp:83-116
 *   - BVHTraversalData                       src/liblightmetrica/scene.bvh.cpp:118-149
 *   - BVHScene::Intersect(node) / (AABB)     src/liblightmetrica/scene.bvh.cpp:405-473
 *   - NaiveScene::IntersectTriangles         src/liblightmetrica/scene.naive.cpp:98-121
 *   - AABB                                   include/lightmetrica/aabb.inl:24-93
 * Every float operation is written in the reference's evaluation order and
 * must be compiled without contraction (-ffp-contract=off): the float SSE
 * build of the reference rounds each operation separately.
 */
#include "lmoracle.h"
#include <float.h>
#include <stdlib.h>
#include <string.h>

/* _mm_min_ps / _mm_max_ps semantics (math.vector.inl:1023-1033): the second
 * operand is returned unless the first compares strictly smaller/larger. */
static inline float fmin_sse(float a, float b) { return a < b ? a : b; }
static inline float fmax_sse(float a, float b) { return a > b ? a : b; }

typedef struct { float mn[3], mx[3]; } aabb;

static inline aabb aabb_empty(void)
{   /* aabb.inl:24-29: min = Inf() = FLT_MAX, max = -FLT_MAX */
    aabb b;
    for (int i = 0; i < 3; i++) { b.mn[i] = FLT_MAX; b.mx[i] = -FLT_MAX; }
    return b;
}
static inline aabb aabb_union(aabb a, const aabb* b)
{   /* aabb.inl:79-85 */
    aabb r;
    for (int i = 0; i < 3; i++) { r.mn[i] = fmin_sse(a.mn[i], b->mn[i]); r.mx[i] = fmax_sse(a.mx[i], b->mx[i]); }
    return r;
}
static inline aabb aabb_union_p(aabb a, const float p[3])
{   /* aabb.inl:87-93 */
    aabb r;
    for (int i = 0; i < 3; i++) { r.mn[i] = fmin_sse(a.mn[i], p[i]); r.mx[i] = fmax_sse(a.mx[i], p[i]); }
    return r;
}
static inline float aabb_area(const aabb* b)
{   /* aabb.inl:61-65 */
    float dx = b->mx[0] - b->mn[0], dy = b->mx[1] - b->mn[1], dz = b->mx[2] - b->mn[2];
    float s = dx * dy;
    s = s + dy * dz;
    s = s + dz * dx;
    return 2.0f * s;
}
static inline int aabb_longest(const aabb* b)
{   /* aabb.inl:73-77 */
    float dx = b->mx[0] - b->mn[0], dy = b->mx[1] - b->mn[1], dz = b->mx[2] - b->mn[2];
    return (dx > dy && dx > dz) ? 0 : (dy > dz ? 1 : 2);
}

/* ------------------------------------------------------------ TriAccel ---- */

int orc_triaccel_load(orc_triaccel* ta, const float A[3], const float B[3], const float C[3])
{
    static const int wald_modulo[4] = { 1, 2, 0, 1 };
    float b[3], c[3], N[3];
    for (int i = 0; i < 3; i++) { b[i] = C[i] - A[i]; c[i] = B[i] - A[i]; }
    /* Cross(c, b), math.vector.inl:994-1004 */
    N[0] = c[1] * b[2] - c[2] * b[1];
    N[1] = c[2] * b[0] - c[0] * b[2];
    N[2] = c[0] * b[1] - c[1] * b[0];
    uint32_t k = 0;
    for (int j = 0; j < 3; j++)
        if (__builtin_fabsf(N[j]) > __builtin_fabsf(N[k])) k = (uint32_t)j;
    int u = wald_modulo[k], v = wald_modulo[k + 1];
    float n_k = N[k];
    float denom = b[u] * c[v] - b[v] * c[u];
    ta->k = k;
    if (denom == 0.0f) { ta->k = 3; return 1; }
    ta->n_u = N[u] / n_k;
    ta->n_v = N[v] / n_k;
    /* Dot(A, N) via _mm_dp_ps(.., 0x71): (x*x' + y*y') + (z*z' + 0) */
    float dot = A[0] * N[0] + A[1] * N[1];
    dot = dot + A[2] * N[2];
    ta->n_d = dot / n_k;
    ta->b_nu = b[u] / denom;
    ta->b_nv = -b[v] / denom;
    ta->a_u = A[u];
    ta->a_v = A[v];
    ta->c_nu = c[v] / denom;
    ta->c_nv = -c[u] / denom;
    return 0;
}

int orc_triaccel_intersect(const orc_triaccel* ta, const float o[3], const float d[3],
                           float mint, float maxt, float* uo, float* vo, float* to)
{
    float o_u, o_v, o_k, d_u, d_v, d_k;
    switch (ta->k) {
    case 0: o_u = o[1]; o_v = o[2]; o_k = o[0]; d_u = d[1]; d_v = d[2]; d_k = d[0]; break;
    case 1: o_u = o[2]; o_v = o[0]; o_k = o[1]; d_u = d[2]; d_v = d[0]; d_k = d[1]; break;
    case 2: o_u = o[0]; o_v = o[1]; o_k = o[2]; d_u = d[0]; d_v = d[1]; d_k = d[2]; break;
    default: return 0;
    }
    float num = ta->n_d - o_u * ta->n_u;
    num = num - o_v * ta->n_v;
    num = num - o_k;
    float den = d_u * ta->n_u + d_v * ta->n_v;
    den = den + d_k;
    float t = num / den;
    *to = t;
    if (t < mint || t > maxt) return 0;
    float hu = o_u + t * d_u;
    hu = hu - ta->a_u;
    float hv = o_v + t * d_v;
    hv = hv - ta->a_v;
    float u = hv * ta->b_nu + hu * ta->b_nv;
    float v = hu * ta->c_nu + hv * ta->c_nv;
    *uo = u;
    *vo = v;
    return u >= 0.0f && v >= 0.0f && u + v <= 1.0f;
}

/* ------------------------------------------------------------------ BVH --- */

typedef struct {
    aabb bound;
    int leaf;
    int begin, end;     /* leaf: [begin, end) into tri_order */
    int axis;           /* internal */
    int left, right;    /* internal: node indices */
} node_t;

struct orc_scene {
    int kind;
    int ntris;
    orc_triaccel* ta;
    aabb* tri_bounds;
    float* centroids;   /* 3 per triangle */
    int32_t* tri_order; /* bvhTriIndices */
    node_t* nodes;
    int64_t nnodes, cap;
    int64_t nleaves;
    int32_t max_depth;
    int root;
};

static int new_node(orc_scene* s)
{
    if (s->nnodes == s->cap) {
        s->cap = s->cap ? s->cap * 2 : 1024;
        s->nodes = (node_t*)realloc(s->nodes, (size_t)s->cap * sizeof(node_t));
    }
    memset(&s->nodes[s->nnodes], 0, sizeof(node_t));
    return (int)s->nnodes++;
}

/* Bucket of triangle i along axis, scene.bvh.cpp:99-104 and :322-326. */
static inline int bucket_of(const orc_scene* s, int tri, int axis, const aabb* cb)
{
    float c = s->centroids[3 * tri + axis];
    float num = c - cb->mn[axis];
    float den = cb->mx[axis] - cb->mn[axis];
    float x = 12.0f * (num / den);
    int b = (int)x;
    return b < 11 ? b : 11;
}

/* Hoare-style two-pointer partition (the bidirectional-iterator algorithm of
 * std::partition): elements satisfying pred move to the front. Returns mid. */
static int partition_bucket(orc_scene* s, int first, int last, int axis, int min_idx, const aabb* cb)
{
    int32_t* a = s->tri_order;
    for (;;) {
        for (;;) {
            if (first == last) return first;
            if (bucket_of(s, a[first], axis, cb) <= min_idx) ++first; else break;
        }
        --last;
        for (;;) {
            if (first == last) return first;
            if (!(bucket_of(s, a[last], axis, cb) <= min_idx)) --last; else break;
        }
        int32_t tmp = a[first]; a[first] = a[last]; a[last] = tmp;
        ++first;
    }
}

static int build_rec(orc_scene* s, int begin, int end, int depth)
{
    if (depth > s->max_depth) s->max_depth = depth;
    aabb bound = aabb_empty();
    for (int i = begin; i < end; i++) bound = aabb_union(bound, &s->tri_bounds[s->tri_order[i]]);
    int n = end - begin;
    int id;
    if (n == 1) {
        id = new_node(s);
        s->nodes[id].leaf = 1; s->nodes[id].begin = begin; s->nodes[id].end = end; s->nodes[id].bound = bound;
        s->nleaves++;
        return id;
    }
    aabb cb = aabb_empty();
    for (int i = begin; i < end; i++) cb = aabb_union_p(cb, &s->centroids[3 * s->tri_order[i]]);
    int axis = aabb_longest(&cb);
    if (cb.mn[axis] == cb.mx[axis]) {
        id = new_node(s);
        s->nodes[id].leaf = 1; s->nodes[id].begin = begin; s->nodes[id].end = end; s->nodes[id].bound = bound;
        s->nleaves++;
        return id;
    }
    aabb bb[12];
    int bc[12];
    for (int i = 0; i < 12; i++) { bb[i] = aabb_empty(); bc[i] = 0; }
    for (int i = begin; i < end; i++) {
        int t = s->tri_order[i];
        int b = bucket_of(s, t, axis, &cb);
        bc[b]++;
        bb[b] = aabb_union(bb[b], &s->tri_bounds[t]);
    }
    float costs[11];
    float area = aabb_area(&bound);
    for (int i = 0; i < 11; i++) {
        aabb b1 = aabb_empty(), b2 = aabb_empty();
        int c1 = 0, c2 = 0;
        for (int j = 0; j <= i; j++) { b1 = aabb_union(b1, &bb[j]); c1 += bc[j]; }
        for (int j = i + 1; j < 12; j++) { b2 = aabb_union(b2, &bb[j]); c2 += bc[j]; }
        float num = (float)c1 * aabb_area(&b1) + (float)c2 * aabb_area(&b2);
        costs[i] = 0.125f + num / area;
    }
    int min_idx = 0;
    double min_cost = costs[0];
    for (int i = 1; i < 11; i++)
        if (min_cost > costs[i]) { min_cost = costs[i]; min_idx = i; }
    if (min_cost < (float)n || n > 255) {
        int mid = partition_bucket(s, begin, end, axis, min_idx, &cb);
        int l = build_rec(s, begin, mid, depth + 1);
        int r = build_rec(s, mid, end, depth + 1);
        id = new_node(s);
        s->nodes[id].leaf = 0; s->nodes[id].axis = axis; s->nodes[id].left = l; s->nodes[id].right = r;
        s->nodes[id].bound = aabb_union(s->nodes[l].bound, &s->nodes[r].bound);
        return id;
    }
    id = new_node(s);
    s->nodes[id].leaf = 1; s->nodes[id].begin = begin; s->nodes[id].end = end; s->nodes[id].bound = bound;
    s->nleaves++;
    return id;
}

orc_scene* orc_scene_create(int kind, const float* positions, int num_vertices,
                            const uint32_t* faces, int num_tris)
{
    (void)num_vertices;
    orc_scene* s = (orc_scene*)calloc(1, sizeof(orc_scene));
    s->kind = kind;
    s->ntris = num_tris;
    s->ta = (orc_triaccel*)calloc((size_t)num_tris + 1, sizeof(orc_triaccel));
    s->tri_bounds = (aabb*)calloc((size_t)num_tris + 1, sizeof(aabb));
    s->centroids = (float*)calloc(3 * (size_t)num_tris + 3, sizeof(float));
    s->tri_order = (int32_t*)calloc((size_t)num_tris + 1, sizeof(int32_t));
    for (int j = 0; j < num_tris; j++) {
        const float* p1 = positions + 3 * (size_t)faces[3 * (size_t)j];
        const float* p2 = positions + 3 * (size_t)faces[3 * (size_t)j + 1];
        const float* p3 = positions + 3 * (size_t)faces[3 * (size_t)j + 2];
        /* identity Mat4f * Vec4f (math.matrix.inl:692-702) maps -0 to +0 */
        float q1[3], q2[3], q3[3];
        for (int c = 0; c < 3; c++) { q1[c] = p1[c] + 0.0f; q2[c] = p2[c] + 0.0f; q3[c] = p3[c] + 0.0f; }
        orc_triaccel_load(&s->ta[j], q1, q2, q3);
        s->ta[j].shape_index = (uint32_t)j;
        s->ta[j].prim_index = 0;
        s->tri_order[j] = j;
        aabb tb;
        for (int c = 0; c < 3; c++) { tb.mn[c] = fmin_sse(q1[c], q2[c]); tb.mx[c] = fmax_sse(q1[c], q2[c]); }
        tb = aabb_union_p(tb, q3);
        s->tri_bounds[j] = tb;
        for (int c = 0; c < 3; c++) s->centroids[3 * j + c] = (tb.mn[c] + tb.mx[c]) * 0.5f;
    }
    if (kind == ORC_SCENE_BVH && num_tris > 0) s->root = build_rec(s, 0, num_tris, 0);
    else s->root = -1;
    return s;
}

void orc_scene_destroy(orc_scene* s)
{
    if (!s) return;
    free(s->ta); free(s->tri_bounds); free(s->centroids); free(s->tri_order); free(s->nodes);
    free(s);
}

void orc_scene_stats(const orc_scene* s, int64_t* nodes, int64_t* leaves, int32_t* max_depth)
{
    if (nodes) *nodes = s->nnodes;
    if (leaves) *leaves = s->nleaves;
    if (max_depth) *max_depth = s->max_depth;
}

const int32_t* orc_scene_tri_order(const orc_scene* s) { return s->tri_order; }

typedef struct {
    float o[3], d[3];
    float mint, maxt;
    int neg[3];
    float inv_min[3], inv_max[3];
    int hit_tri;
    float hu, hv;
    int32_t node_tests, tri_tests;
} trav_t;

static int slab(const aabb* b, trav_t* r)
{   /* scene.bvh.cpp:450-473 */
    r->node_tests++;
    const float* lo0 = r->neg[0] ? b->mx : b->mn;
    const float* hi0 = r->neg[0] ? b->mn : b->mx;
    const float* lo1 = r->neg[1] ? b->mx : b->mn;
    const float* hi1 = r->neg[1] ? b->mn : b->mx;
    const float* lo2 = r->neg[2] ? b->mx : b->mn;
    const float* hi2 = r->neg[2] ? b->mn : b->mx;
    float tmin = (lo0[0] - r->o[0]) * r->inv_min[0];
    float tmax = (hi0[0] - r->o[0]) * r->inv_max[0];
    float tymin = (lo1[1] - r->o[1]) * r->inv_min[1];
    float tymax = (hi1[1] - r->o[1]) * r->inv_max[1];
    if ((tmin > tymax) || (tymin > tmax)) return 0;
    if (tymin > tmin) tmin = tymin;
    if (tymax < tmax) tmax = tymax;
    float tzmin = (lo2[2] - r->o[2]) * r->inv_min[2];
    float tzmax = (hi2[2] - r->o[2]) * r->inv_max[2];
    if ((tmin > tzmax) || (tzmin > tmax)) return 0;
    if (tzmin > tmin) tmin = tzmin;
    if (tzmax < tmax) tmax = tzmax;
    return (tmin < r->maxt) && (tmax > r->mint);
}

static int trav_rec(const orc_scene* s, int ni, trav_t* r)
{   /* scene.bvh.cpp:405-448 */
    const node_t* nd = &s->nodes[ni];
    int hit = 0;
    if (!slab(&nd->bound, r)) return 0;
    if (nd->leaf) {
        for (int i = nd->begin; i < nd->end; i++) {
            int tri = s->tri_order[i];
            float u, v, t;
            r->tri_tests++;
            if (orc_triaccel_intersect(&s->ta[tri], r->o, r->d, r->mint, r->maxt, &u, &v, &t)) {
                r->maxt = t; r->hit_tri = tri; r->hu = u; r->hv = v; hit = 1;
            }
        }
    } else if (r->neg[nd->axis]) {
        hit |= trav_rec(s, nd->right, r);
        hit |= trav_rec(s, nd->left, r);
    } else {
        hit |= trav_rec(s, nd->left, r);
        hit |= trav_rec(s, nd->right, r);
    }
    return hit;
}

int64_t orc_intersect(const orc_scene* s, int64_t n, const float* rays, int32_t* tri_id,
                      float* t, float* u, float* v, int32_t* node_tests, int32_t* tri_tests)
{
    int64_t hits = 0;
    for (int64_t i = 0; i < n; i++) {
        const float* ry = rays + 8 * i;
        trav_t r;
        memset(&r, 0, sizeof(r));
        for (int c = 0; c < 3; c++) {
            r.o[c] = ry[c];
            r.d[c] = ry[3 + c];
            /* scene.bvh.cpp:124-137 */
            r.inv_min[c] = (r.d[c] == 0.0f) ? 0.0f : 1.0f / r.d[c];
            r.inv_max[c] = (r.d[c] == 0.0f) ? FLT_MAX : 1.0f / r.d[c];
            r.neg[c] = r.d[c] < 0.0f;
        }
        r.mint = ry[6];
        r.maxt = ry[7];
        r.hit_tri = -1;
        int hit = 0;
        if (s->kind == ORC_SCENE_BVH) {
            if (s->root >= 0) hit = trav_rec(s, s->root, &r);
        } else {
            for (int k = 0; k < s->ntris; k++) {
                float uu, vv, tt;
                r.tri_tests++;
                if (orc_triaccel_intersect(&s->ta[k], r.o, r.d, r.mint, r.maxt, &uu, &vv, &tt)) {
                    r.maxt = tt; r.hit_tri = k; r.hu = uu; r.hv = vv; hit = 1;
                }
            }
        }
        if (tri_id) tri_id[i] = hit ? r.hit_tri : -1;
        if (t) t[i] = hit ? r.maxt : 0.0f;
        if (u) u[i] = hit ? r.hu : 0.0f;
        if (v) v[i] = hit ? r.hv : 0.0f;
        if (node_tests) node_tests[i] = r.node_tests;
        if (tri_tests) tri_tests[i] = r.tri_tests;
        hits += hit;
    }
    return hits;
}
