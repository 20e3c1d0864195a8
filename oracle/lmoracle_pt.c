/*
 * ORACLE — test infrastructure, not product code (see lmoracle.h).
 *
 * Double-precision restatement of the reference's unidirectional path
 * tracers, one sample at a time:
 *   pt         src/liblightmetrica/pathtrace.cpp:165-266
 *   pt.direct  src/liblightmetrica/pathtrace.direct.cpp:170-338
 *   pt.mis     src/liblightmetrica/pathtrace.mis.cpp:167-369
 * with the reference's camera (perspectivecamera.cpp:97-353), BSDFs
 * (diffuse.cpp:133-220, mirror.cpp:84-107, diffusemirror.cpp:84-270,
 * bsdf.h:57-83), lights (light.area.cpp:109-252, light.env.const.cpp:90-214,
 * emittershape.sphere.cpp:117-171), geometry term and visibility
 * (renderutils.cpp:29-70) and film accumulate/rescale (hdrfilm.cpp:151-171,
 * sched.mt.cpp:250-256). Ray casting uses a median-split BVH in double (the
 * accelerator does not change images). Random numbers follow the same
 * counter-based scheme as the GPU renderer (seed, sample, dimension), so
 * results are reproducible; parity with the reference's Mersenne-twister
 * stream is statistical.
 *
 * Also provides the FP64 reference gradient of an image loss with respect
 * to per-triangle diffuse albedo and light emission (orc_render_grad), by
 * differentiating each sample's contributions along its replayed path.
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define PI 3.14159265358979323846
#define INV_PI 0.31830988618379067154
#define EPS 1e-7             /* Math::Constants::Eps() (double build) */
#define EPS_LARGE 1e-5       /* Math::Constants::EpsLarge() (double build) */
#define MAX_VERTS 64              /* initial capacity of a path's vertex records */
#define MAX_PATH_VERTICES 4096    /* the device's bound on replayed surface vertices */

typedef struct { double x, y, z; } v3;
static inline v3 mk(double x, double y, double z) { v3 r = { x, y, z }; return r; }
static inline v3 add(v3 a, v3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 sub(v3 a, v3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 mul(v3 a, double s) { return mk(a.x * s, a.y * s, a.z * s); }
static inline v3 mulv(v3 a, v3 b) { return mk(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline double dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline v3 cross(v3 a, v3 b) { return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
static inline v3 normalize(v3 a) { return mul(a, 1.0 / sqrt(dot(a, a))); }
static inline int is_zero(v3 a) { return a.x == 0.0 && a.y == 0.0 && a.z == 0.0; }
static inline double lum(v3 v) { return 0.212671 * v.x + 0.715160 * v.y + 0.072169 * v.z; }
static inline double comp(v3 v, int c) { return c == 0 ? v.x : (c == 1 ? v.y : v.z); }

/* ------------------------------------------------------------- RNG ------ */
static inline uint64_t mix64(uint64_t x)
{
    x ^= x >> 30; x *= 0xBF58476D1CE4E5B9ull;
    x ^= x >> 27; x *= 0x94D049BB133111EBull;
    x ^= x >> 31;
    return x;
}
static inline uint64_t sample_key(uint64_t seed, uint64_t s)
{
    return mix64(mix64(seed + 0x9E3779B97F4A7C15ull) ^ (s * 0xD1B54A32D192ED03ull));
}
static inline double rnd(uint64_t key, uint32_t dim)
{
    uint64_t x = mix64(key ^ ((uint64_t)(dim + 1) * 0x9E3779B97F4A7C15ull));
    return (double)(uint32_t)(x >> 40) * (1.0 / 16777216.0);
}
#define DIM_V(k) (8u * (uint32_t)(k))
enum { D_LIGHT = 0, D_RR = 2, D_BSDF = 3, D_COMP = 5 };

/* ----------------------------------------------------------- scene ----- */
typedef struct {
    int num_tris;
    const float* pos;        /* 9 per triangle, world space */
    const float* nrm;        /* 9 per triangle */
    const int* tri_mat;      /* material per triangle, -1 = black */
    const int* tri_light;    /* area light per triangle, -1 = none */
    int num_mats;
    const int* mat_type;     /* 0 diffuse, 1 mirror, 2 diffuse-mirror */
    const float* mat_R;      /* 3 per material */
    const float* tri_albedo; /* optional 3 per triangle: overrides R of diffuse BSDFs */
    int num_lights;
    const float* light_Le;   /* 3 per area light */
    int has_env;
    float env_Le[3];
    float eye[3], center[3], up[3];
    float fovy;
    int width, height;
    int technique;           /* 0 pt, 1 pt.direct, 2 pt.mis */
    int rr_depth, max_pv;
    int sampling;            /* 0 stratified, 1 uniform */
    uint64_t seed;
    int64_t sample_begin, sample_end;
} orc_pt_desc;

typedef struct { double mn[3], mx[3]; int left, right, begin, end; } bnode;

typedef struct {
    const orc_pt_desc* d;
    v3* p;          /* 3 per triangle */
    v3* n;
    int* order;
    bnode* nodes;
    int nnodes;
    /* lights */
    double* cdf;    /* per area light: prefix areas (normalised), packed */
    int* cdf_begin; int* cdf_count; int* ltris; double* larea;
    v3 env_c; double env_r, env_inv_area;
    /* camera */
    double view[16], iview[16], proj[16], iproj[16];
    v3 cam_p; double inv_A;
} pt_scene;

/* qsort comparator context (one per thread: several scenes may build at once). */
typedef struct { const pt_scene* s; int axis; } sort_ctx;
static __thread sort_ctx g_sort;

static double tri_centroid(const pt_scene* s, int t, int a)
{
    return (comp(s->p[3 * t], a) + comp(s->p[3 * t + 1], a) + comp(s->p[3 * t + 2], a)) / 3.0;
}

static int cmp_tri(const void* a, const void* b)
{
    double ca = tri_centroid(g_sort.s, *(const int*)a, g_sort.axis);
    double cb = tri_centroid(g_sort.s, *(const int*)b, g_sort.axis);
    return ca < cb ? -1 : (ca > cb ? 1 : 0);
}

static int build(pt_scene* s, int b, int e)
{
    int id = s->nnodes++;
    bnode* nd = &s->nodes[id];
    for (int c = 0; c < 3; c++) { nd->mn[c] = DBL_MAX; nd->mx[c] = -DBL_MAX; }
    for (int i = b; i < e; i++)
        for (int k = 0; k < 3; k++) {
            v3 q = s->p[3 * s->order[i] + k];
            for (int c = 0; c < 3; c++) {
                double v = comp(q, c);
                if (v < nd->mn[c]) nd->mn[c] = v;
                if (v > nd->mx[c]) nd->mx[c] = v;
            }
        }
    nd->begin = b; nd->end = e; nd->left = nd->right = -1;
    if (e - b <= 4) return id;
    int axis = 0;
    double ext = -1;
    for (int c = 0; c < 3; c++) if (nd->mx[c] - nd->mn[c] > ext) { ext = nd->mx[c] - nd->mn[c]; axis = c; }
    g_sort.s = s;
    g_sort.axis = axis;
    qsort(s->order + b, (size_t)(e - b), sizeof(int), cmp_tri);
    int m = (b + e) / 2;
    int l = build(s, b, m);
    int r = build(s, m, e);
    s->nodes[id].left = l; s->nodes[id].right = r;
    return id;
}

/* Moller-Trumbore in double (the image does not depend on the test used). */
static int hit_tri(const pt_scene* s, int t, v3 o, v3 d, double tmin, double tmax, double* tt, double* b0, double* b1)
{
    v3 p0 = s->p[3 * t], e1 = sub(s->p[3 * t + 1], p0), e2 = sub(s->p[3 * t + 2], p0);
    v3 pv = cross(d, e2);
    double det = dot(e1, pv);
    if (det == 0.0) return 0;
    double inv = 1.0 / det;
    v3 tv = sub(o, p0);
    double u = dot(tv, pv) * inv;
    if (u < 0.0 || u > 1.0) return 0;
    v3 qv = cross(tv, e1);
    double v = dot(d, qv) * inv;
    if (v < 0.0 || u + v > 1.0) return 0;
    double t_ = dot(e2, qv) * inv;
    if (t_ < tmin || t_ > tmax) return 0;
    *tt = t_; *b0 = u; *b1 = v;
    return 1;
}

static int box_hit(const bnode* n, v3 o, v3 inv, double tmin, double tmax)
{
    for (int c = 0; c < 3; c++) {
        double oc = comp(o, c), ic = comp(inv, c);
        double t0 = (n->mn[c] - oc) * ic, t1 = (n->mx[c] - oc) * ic;
        if (t0 > t1) { double x = t0; t0 = t1; t1 = x; }
        if (t0 > tmin) tmin = t0;
        if (t1 < tmax) tmax = t1;
        if (tmin > tmax) return 0;
    }
    return 1;
}

/* Closest (or any) triangle hit: returns triangle or -1. */
static int cast(const pt_scene* s, v3 o, v3 d, double tmin, double tmax, double* t, double* b0, double* b1, int any)
{
    v3 inv = mk(1.0 / d.x, 1.0 / d.y, 1.0 / d.z);
    int stack[128], sp = 0, best = -1;
    if (s->nnodes == 0) return -1;
    stack[sp++] = 0;
    while (sp) {
        const bnode* n = &s->nodes[stack[--sp]];
        if (!box_hit(n, o, inv, tmin, tmax)) continue;
        if (n->left < 0) {
            for (int i = n->begin; i < n->end; i++) {
                double tt, u, v;
                int tri = s->order[i];
                if (hit_tri(s, tri, o, d, tmin, tmax, &tt, &u, &v)) {
                    tmax = tt; best = tri; *t = tt; *b0 = u; *b1 = v;
                    if (any) return best;
                }
            }
        } else {
            stack[sp++] = n->left;
            stack[sp++] = n->right;
        }
    }
    return best;
}

/* -------------------------------------------------------- geometry ----- */
typedef struct { v3 p, gn, sn, ss, st; int deg; } geom;

static void tangent(geom* g)
{   /* OrthonormalBasis, math.linalgebra.inl:26-33 */
    v3 a = g->sn;
    g->st = fabs(a.x) > fabs(a.y) ? normalize(mk(a.z, 0, -a.x)) : normalize(mk(0, a.z, -a.y));
    g->ss = normalize(cross(g->st, a));
}
static inline v3 to_local(const geom* g, v3 w) { return mk(dot(g->ss, w), dot(g->st, w), dot(g->sn, w)); }
static inline v3 to_world(const geom* g, v3 l) { return add(add(mul(g->ss, l.x), mul(g->st, l.y)), mul(g->sn, l.z)); }

static int env_hit(const pt_scene* s, v3 ro, v3 rd, double mint, double maxt, double* t)
{   /* emittershape.sphere.cpp:117-152 */
    v3 o = sub(ro, s->env_c);
    double a = dot(rd, rd), b = 2.0 * dot(o, rd), c = dot(o, o) - s->env_r * s->env_r;
    double det = b * b - 4.0 * a * c;
    if (det < 0.0) return 0;
    double e = sqrt(det), den = 2.0 * a;
    double t0 = (-b - e) / den, t1 = (-b + e) / den;
    if (t0 > maxt || t1 < mint) return 0;
    *t = t0;
    if (*t < mint) { *t = t1; if (*t > maxt) return 0; }
    return 1;
}

/* ---------------------------------------------------------- camera ----- */
static void m4v(const double* m, double x, double y, double z, double w, double* o)
{
    for (int r = 0; r < 4; r++) o[r] = m[r] * x + m[4 + r] * y + m[8 + r] * z + m[12 + r] * w;
}
static int inv4(const double* m, double* inv)
{
    double a[4][8];
    for (int r = 0; r < 4; r++)
        for (int c = 0; c < 4; c++) { a[r][c] = m[4 * c + r]; a[r][4 + c] = r == c; }
    for (int c = 0; c < 4; c++) {
        int piv = c;
        for (int r = c + 1; r < 4; r++) if (fabs(a[r][c]) > fabs(a[piv][c])) piv = r;
        if (a[piv][c] == 0.0) return 0;
        for (int k = 0; k < 8; k++) { double t = a[c][k]; a[c][k] = a[piv][k]; a[piv][k] = t; }
        double dd = a[c][c];
        for (int k = 0; k < 8; k++) a[c][k] /= dd;
        for (int r = 0; r < 4; r++) if (r != c) { double f = a[r][c]; for (int k = 0; k < 8; k++) a[r][k] -= f * a[c][k]; }
    }
    for (int r = 0; r < 4; r++) for (int c = 0; c < 4; c++) inv[4 * c + r] = a[r][4 + c];
    return 1;
}
static double importance(const pt_scene* s, double cs)
{   /* perspectivecamera.cpp:325-353 */
    if (cs <= 0.0) return 0.0;
    if (fabs(cs - 1.0) < EPS_LARGE) cs = 1.0;
    double ic = 1.0 / cs;
    return s->inv_A * ic * ic * ic;
}
static v3 cam_dir(const pt_scene* s, double rx, double ry, double* pdf)
{   /* perspectivecamera.cpp:216-240 */
    double q[4], w[4];
    m4v(s->iproj, rx * 2 - 1, ry * 2 - 1, 0, 1, q);
    v3 dc = normalize(mk(q[0] / q[3], q[1] / q[3], q[2] / q[3]));
    *pdf = importance(s, -dc.z);
    m4v(s->iview, dc.x, dc.y, dc.z, 0, w);
    return normalize(mk(w[0], w[1], w[2]));
}
static int cam_project(const pt_scene* s, v3 p, v3 d, double* rx, double* ry, double* We)
{   /* RayToRasterPosition / EvaluateDirection, perspectivecamera.cpp:276-323 */
    v3 q = add(p, d);
    double c4[4], n4[4];
    m4v(s->view, q.x, q.y, q.z, 1, c4);
    m4v(s->proj, c4[0], c4[1], c4[2], c4[3], n4);
    *rx = (n4[0] / n4[3] + 1) / 2;
    *ry = (n4[1] / n4[3] + 1) / 2;
    if (*rx < 0 || *rx > 1 || *ry < 0 || *ry > 1) { *We = 0; return 0; }
    *We = importance(s, -normalize(mk(c4[0], c4[1], c4[2])).z);
    return 1;
}
static int pixel_of(const pt_scene* s, double rx, double ry)
{   /* hdrfilm.cpp:151-171 */
    if (rx < 0 || rx > 1 || ry < 0 || ry > 1) return -1;
    int W = s->d->width, H = s->d->height;
    int x = (int)(rx * W), y = (int)(ry * H);
    if (x < 0) x = 0;
    if (x > W - 1) x = W - 1;
    if (y < 0) y = 0;
    if (y > H - 1) y = H - 1;
    return y * W + x;
}

/* ----------------------------------------------------------- lights ---- */
typedef struct { v3 p, n, Le; double pdf; int light; } lpoint;

static int sample_light(const pt_scene* s, double u0, double u1, lpoint* lp)
{   /* scene.cpp:79-86 + light.area.cpp:146-179 / light.env.const.cpp:194-203 */
    const orc_pt_desc* d = s->d;
    int nl = d->num_lights + (d->has_env ? 1 : 0);
    if (nl == 0) return 0;
    int li = (int)(u0 * nl);
    if (li > nl - 1) li = nl - 1;
    u0 = u0 * nl - li;
    double sel = 1.0 / nl;
    if (li >= d->num_lights) {
        double z = 1 - 2 * u0, r = sqrt(fmax(0.0, 1 - z * z)), ph = 2 * PI * u1;
        v3 dd = mk(r * cos(ph), r * sin(ph), z);
        lp->p = add(s->env_c, mul(dd, s->env_r));
        lp->n = mul(dd, -1);
        lp->pdf = s->env_inv_area * sel;
        lp->Le = mk(d->env_Le[0], d->env_Le[1], d->env_Le[2]);
        lp->light = li;
        return 1;
    }
    const double* cdf = s->cdf + s->cdf_begin[li];
    int n = s->cdf_count[li];
    int lo = 0, hi = n + 1;
    while (lo < hi) { int m = (lo + hi) / 2; if (cdf[m] > u1) hi = m; else lo = m + 1; }
    int idx = lo - 1;
    if (idx < 0) idx = 0;
    if (idx > n - 1) idx = n - 1;
    double v = (u1 - cdf[idx]) / (cdf[idx + 1] - cdf[idx]);
    int t = s->ltris[s->cdf_begin[li] - li + idx];
    v3 p1 = s->p[3 * t], p2 = s->p[3 * t + 1], p3 = s->p[3 * t + 2];
    double sq = sqrt(fmax(0.0, u0)), b0 = 1 - sq, b1 = v * sq;
    lp->p = add(add(mul(p1, 1 - b0 - b1), mul(p2, b0)), mul(p3, b1));
    lp->n = normalize(cross(sub(p2, p1), sub(p3, p1)));
    lp->pdf = sel / s->larea[li];
    lp->Le = mk(d->light_Le[3 * li], d->light_Le[3 * li + 1], d->light_Le[3 * li + 2]);
    lp->light = li;
    return 1;
}

static double gterm(v3 p1, v3 n1, int deg1, v3 p2, v3 n2, int deg2)
{   /* renderutils.cpp:29-56 */
    v3 d = sub(p2, p1);
    double l2 = dot(d, d), l = sqrt(l2);
    d = mul(d, 1.0 / l);
    double num = 1;
    if (!deg1) num *= fabs(dot(n1, d));
    if (!deg2) num *= fabs(dot(n2, mul(d, -1)));
    if (fabs(l) < EPS) return 0;
    return num / l2;
}

static int visible(const pt_scene* s, v3 a, v3 b)
{   /* renderutils.cpp:58-70: triangles and the environment's emitter shape */
    v3 d = sub(b, a);
    double len = sqrt(dot(d, d));
    d = mul(d, 1.0 / len);
    double t, u, v;
    double maxt = len * (1 - EPS);
    if (cast(s, a, d, EPS, maxt, &t, &u, &v, 1) >= 0) return 0;
    if (s->d->has_env && env_hit(s, a, d, EPS, maxt, &t)) return 0;
    return 1;
}

/* ----------------------------------------------------------- BSDFs ----- */
typedef struct { int type; v3 R; } mat_t;   /* type 3 = black */

static mat_t tri_material(const pt_scene* s, int tri)
{
    const orc_pt_desc* d = s->d;
    mat_t m;
    int mi = d->tri_mat[tri];
    if (mi < 0) { m.type = 3; m.R = mk(0, 0, 0); return m; }
    m.type = d->mat_type[mi];
    m.R = mk(d->mat_R[3 * mi], d->mat_R[3 * mi + 1], d->mat_R[3 * mi + 2]);
    if (d->tri_albedo && m.type == 0)
        m.R = mk(d->tri_albedo[3 * tri], d->tri_albedo[3 * tri + 1], d->tri_albedo[3 * tri + 2]);
    return m;
}

static void concentric(double u0, double u1, double* x, double* y)
{   /* math.stats.inl:25-56 */
    double v1 = 2 * u0 - 1, v2 = 2 * u1 - 1, r, th;
    if (v1 == 0 && v2 == 0) { *x = *y = 0; return; }
    if (v1 > -v2) { if (v1 > v2) { r = v1; th = (PI / 4) * v2 / v1; } else { r = v2; th = (PI / 4) * (2 - v1 / v2); } }
    else { if (v1 < v2) { r = -v1; th = (PI / 4) * (4 + v2 / v1); } else { r = -v2; th = (PI / 4) * (6 - v1 / v2); } }
    *x = r * cos(th);
    *y = r * sin(th);
}

static double sfactor(const geom* g, v3 wi, v3 wo, double wiz, double woz)
{   /* bsdf.h:57-83, EL */
    return (dot(wi, g->gn) * wiz <= 0 || dot(wo, g->gn) * woz <= 0) ? 0.0 : 1.0;
}

/* SampleAndEstimateDirection: returns weight (0 = stop), wo, pdf, specular. */
static v3 bsdf_sample(const mat_t* m, const geom* g, v3 wi, double u0, double u1, double uc, v3* wo, double* pdf, int* spec)
{
    v3 z = mk(0, 0, 0);
    v3 lwi = to_local(g, wi);
    *spec = 0;
    *pdf = 0;
    if (lwi.z <= 0 || m->type == 3) return z;
    int diffuse = m->type == 0 || (m->type == 2 && uc < 0.5);
    v3 lwo;
    double k = m->type == 2 ? 0.5 : 1.0;
    if (diffuse) {
        double x, y;
        concentric(u0, u1, &x, &y);
        lwo = mk(x, y, sqrt(fmax(0.0, 1 - x * x - y * y)));
        *pdf = INV_PI * k;
    } else {
        lwo = mk(-lwi.x, -lwi.y, lwi.z);
        *pdf = k / lwo.z;
        *spec = 1;
    }
    *wo = to_world(g, lwo);
    return mul(m->R, sfactor(g, wi, *wo, lwi.z, lwo.z));
}

static v3 bsdf_eval(const mat_t* m, const geom* g, v3 wi, v3 wo, double* pdf)
{   /* EvaluateDirection / EvaluateDirectionPDF, NonDelta query */
    *pdf = 0;
    if (m->type == 1 || m->type == 3) return mk(0, 0, 0);
    v3 lwi = to_local(g, wi), lwo = to_local(g, wo);
    if (lwi.z <= 0 || lwo.z <= 0) return mk(0, 0, 0);
    double k = m->type == 2 ? 0.5 : 1.0;
    *pdf = INV_PI * k;
    return mul(m->R, INV_PI * sfactor(g, wi, wo, lwi.z, lwo.z) * k);
}

/* ------------------------------------------------------------ setup ---- */
static int setup(pt_scene* s, const orc_pt_desc* d)
{
    memset(s, 0, sizeof(*s));
    s->d = d;
    int T = d->num_tris;
    s->p = (v3*)malloc(sizeof(v3) * 3 * (size_t)(T + 1));
    s->n = (v3*)malloc(sizeof(v3) * 3 * (size_t)(T + 1));
    s->order = (int*)malloc(sizeof(int) * (size_t)(T + 1));
    s->nodes = (bnode*)malloc(sizeof(bnode) * 2 * (size_t)(T + 1));
    double mn[3] = { DBL_MAX, DBL_MAX, DBL_MAX }, mx[3] = { -DBL_MAX, -DBL_MAX, -DBL_MAX };
    for (int t = 0; t < T; t++) {
        s->order[t] = t;
        for (int k = 0; k < 3; k++) {
            const float* q = d->pos + 9 * (size_t)t + 3 * k;
            const float* nn = d->nrm + 9 * (size_t)t + 3 * k;
            s->p[3 * t + k] = mk(q[0], q[1], q[2]);
            s->n[3 * t + k] = mk(nn[0], nn[1], nn[2]);
            for (int c = 0; c < 3; c++) { if (q[c] < mn[c]) mn[c] = q[c]; if (q[c] > mx[c]) mx[c] = q[c]; }
        }
    }
    if (T > 0) build(s, 0, T);
    /* area light CDFs in triangle order (light.area.cpp:109-144) */
    int L = d->num_lights;
    s->cdf_begin = (int*)calloc((size_t)L + 1, sizeof(int));
    s->cdf_count = (int*)calloc((size_t)L + 1, sizeof(int));
    s->larea = (double*)calloc((size_t)L + 1, sizeof(double));
    s->cdf = (double*)malloc(sizeof(double) * ((size_t)T + (size_t)L + 1));
    s->ltris = (int*)malloc(sizeof(int) * ((size_t)T + 1));
    int pos = 0, tpos = 0;
    for (int li = 0; li < L; li++) {
        s->cdf_begin[li] = pos;
        int start = pos;
        s->cdf[pos++] = 0;
        for (int t = 0; t < T; t++) {
            if (d->tri_light[t] != li) continue;
            v3 c = cross(sub(s->p[3 * t + 1], s->p[3 * t]), sub(s->p[3 * t + 2], s->p[3 * t]));
            s->cdf[pos] = s->cdf[pos - 1] + 0.5 * sqrt(dot(c, c));
            pos++;
            s->ltris[tpos++] = t;
        }
        s->cdf_count[li] = pos - start - 1;
        s->larea[li] = s->cdf[pos - 1];
        for (int k = start; k < pos; k++) s->cdf[k] /= s->larea[li];
    }
    /* camera (math.transform.inl:88-113, perspectivecamera.cpp:97-168) */
    v3 eye = mk(d->eye[0], d->eye[1], d->eye[2]), ctr = mk(d->center[0], d->center[1], d->center[2]);
    v3 f = normalize(sub(ctr, eye)), u = normalize(mk(d->up[0], d->up[1], d->up[2]));
    v3 sv = normalize(cross(f, u));
    u = cross(sv, f);
    double view[16] = { sv.x, u.x, -f.x, 0, sv.y, u.y, -f.y, 0, sv.z, u.z, -f.z, 0,
                        -dot(sv, eye), -dot(u, eye), dot(f, eye), 1 };
    double aspect = (double)d->width / d->height, tt = tan(d->fovy * PI / 180.0 / 2.0);
    double proj[16] = { 1 / (aspect * tt), 0, 0, 0, 0, 1 / tt, 0, 0, 0, 0, -(1000.0 + 1.0) / (1000.0 - 1.0), -1,
                        0, 0, -(2 * 1000.0 * 1.0) / (1000.0 - 1.0), 0 };
    memcpy(s->view, view, sizeof(view));
    memcpy(s->proj, proj, sizeof(proj));
    if (!inv4(view, s->iview) || !inv4(proj, s->iproj)) return 0;
    s->cam_p = mk(s->iview[12], s->iview[13], s->iview[14]);
    double q1[4], q2[4];
    m4v(s->iproj, -1, -1, 0, 1, q1);
    m4v(s->iproj, 1, 1, 0, 1, q2);
    double c1x = q1[0] / q1[3], c1y = q1[1] / q1[3], c1z = q1[2] / q1[3];
    double c2x = q2[0] / q2[3], c2y = q2[1] / q2[3], c2z = q2[2] / q2[3];
    c1x /= c1z; c1y /= c1z; c2x /= c2z; c2y /= c2z;
    s->inv_A = 1.0 / ((c2x - c1x) * (c2y - c1y));
    /* environment bounding sphere over triangles + camera (light.env.const.cpp:90-97) */
    if (d->has_env) {
        double cp[3] = { s->cam_p.x, s->cam_p.y, s->cam_p.z };
        for (int c = 0; c < 3; c++) { if (cp[c] < mn[c]) mn[c] = cp[c]; if (cp[c] > mx[c]) mx[c] = cp[c]; }
        s->env_c = mk((mx[0] + mn[0]) / 2, (mx[1] + mn[1]) / 2, (mx[2] + mn[2]) / 2);
        v3 dd = sub(s->env_c, mk(mx[0], mx[1], mx[2]));
        s->env_r = sqrt(dot(dd, dd));
        s->env_inv_area = 1.0 / (4 * PI * s->env_r * s->env_r);
    }
    return 1;
}

static void teardown(pt_scene* s)
{
    free(s->p); free(s->n); free(s->order); free(s->nodes);
    free(s->cdf); free(s->cdf_begin); free(s->cdf_count); free(s->ltris); free(s->larea);
}

/* ------------------------------------------------------- one sample ---- */
/* A contribution event: radiance `c` splatted at `pixel`; `depth` = number of
 * surface vertices (from the camera) whose BSDF factors it contains. */
typedef struct { int pixel; v3 c; int depth; int light; v3 Le; } event_t;

typedef struct {
    event_t* ev;           /* grows as needed */
    int nev, cap_ev;
    int* vtri;             /* triangle of surface vertex 1..: index i-1 */
    int nv, cap_v;
    int overflow;          /* the path reached MAX_PATH_VERTICES */
} path_t;

static path_t* path_new(void)
{
    path_t* P = (path_t*)calloc(1, sizeof(path_t));
    P->cap_ev = 2 * MAX_VERTS + 2;
    P->cap_v = MAX_VERTS;
    P->ev = (event_t*)malloc(sizeof(event_t) * P->cap_ev);
    P->vtri = (int*)malloc(sizeof(int) * P->cap_v);
    return P;
}

static void path_free(path_t* P)
{
    free(P->ev);
    free(P->vtri);
    free(P);
}

static void add_event(path_t* P, int pixel, v3 c, int depth, int light, v3 Le)
{
    if (pixel < 0 || is_zero(c)) return;
    if (P->nev == P->cap_ev) {
        P->cap_ev *= 2;
        P->ev = (event_t*)realloc(P->ev, sizeof(event_t) * P->cap_ev);
    }
    event_t* e = &P->ev[P->nev++];
    e->pixel = pixel; e->c = c; e->depth = depth; e->light = light; e->Le = Le;
}

static void add_vertex(path_t* P, int tri)
{
    if (P->nv == P->cap_v) {
        P->cap_v *= 2;
        P->vtri = (int*)realloc(P->vtri, sizeof(int) * P->cap_v);
    }
    P->vtri[P->nv++] = tri;
}

static void run_sample(const pt_scene* s, uint64_t sample, path_t* P)
{
    const orc_pt_desc* d = s->d;
    const int tech = d->technique;
    const int nl = d->num_lights + (d->has_env ? 1 : 0);
    uint64_t key = sample_key(d->seed, sample);
    P->nev = 0;
    P->nv = 0;
    P->overflow = 0;
    double rx, ry;
    double u0 = rnd(key, 0), u1 = rnd(key, 1);
    int64_t pixels = (int64_t)d->width * d->height;
    if (d->sampling == 0) {
        int64_t pix = (int64_t)(sample % (uint64_t)pixels);
        rx = ((double)(pix % d->width) + u0) / d->width;
        ry = ((double)(pix / d->width) + u1) / d->height;
    } else { rx = u0; ry = u1; }
    int path_pixel = pixel_of(s, rx, ry);
    double pdf_cam;
    v3 dir = cam_dir(s, rx, ry, &pdf_cam);
    v3 thr = mk(1, 1, 1);
    if (d->max_pv != -1 && d->max_pv <= 1) return;
    /* previous vertex (for MIS) */
    v3 prev_p = s->cam_p, prev_n = mk(0, 0, 1);
    int prev_deg = 1, prev_spec = 0;
    double prev_pdf = pdf_cam;
    double tmin = tech == 0 ? 0.0 : EPS;
    if (tech != 0) {
        /* camera vertex: NEE, RR (pathtrace.direct.cpp:188-280) */
        lpoint lp;
        if (sample_light(s, rnd(key, DIM_V(1) + D_LIGHT), rnd(key, DIM_V(1) + D_LIGHT + 1), &lp)) {
            v3 ppL = normalize(sub(lp.p, s->cam_p));
            double lrx, lry, We;
            if (visible(s, s->cam_p, lp.p) && cam_project(s, s->cam_p, ppL, &lrx, &lry, &We) && We > 0) {
                double G = gterm(s->cam_p, mk(0, 0, 1), 1, lp.p, lp.n, 0);
                v3 Le = dot(lp.n, mul(ppL, -1)) > 0 ? lp.Le : mk(0, 0, 0);
                if (G != 0) {
                    double w = 1;
                    if (tech == 2) { double pdl = lp.pdf / G; w = pdl / (pdl + We); }
                    add_event(P, pixel_of(s, lrx, lry), mul(Le, w * We * G / lp.pdf), 0, lp.light, lp.Le);
                }
            }
        }
        if (d->rr_depth != -1 && 1 >= d->rr_depth) {
            double p = fmin(0.5, lum(thr));
            if (rnd(key, DIM_V(1) + D_RR) > p) return;
            thr = mul(thr, 1.0 / p);
        }
    }
    v3 ro = s->cam_p, rd = dir;
    for (int k = 1;; k++) {
        if (d->max_pv != -1 && k >= d->max_pv) return;
        double t, b0, b1;
        int tri = cast(s, ro, rd, tmin, DBL_MAX, &t, &b0, &b1, 0);
        geom g;
        v3 wi = mul(rd, -1);
        v3 Le = mk(0, 0, 0);
        double lpdf = 0;
        int light = -1, surface = 0;
        mat_t m;
        m.type = 3;
        m.R = mk(0, 0, 0);
        if (tri < 0) {
            if (!(d->has_env && env_hit(s, ro, rd, tmin, DBL_MAX, &t))) return;
            g.p = add(ro, mul(rd, t));
            g.gn = g.sn = normalize(sub(s->env_c, g.p));
            g.deg = 0;
            tangent(&g);
            if (dot(g.sn, wi) > 0) Le = mk(d->env_Le[0], d->env_Le[1], d->env_Le[2]);
            lpdf = s->env_inv_area;
            light = d->num_lights;
        } else {
            /* StoreIntersectionFromBarycentricCoords, scene.cpp:101-149 */
            g.p = add(ro, mul(rd, t));
            v3 p1 = s->p[3 * tri], p2 = s->p[3 * tri + 1], p3 = s->p[3 * tri + 2];
            g.gn = normalize(cross(sub(p2, p1), sub(p3, p1)));
            g.sn = normalize(add(add(mul(s->n[3 * tri], 1 - b0 - b1), mul(s->n[3 * tri + 1], b0)), mul(s->n[3 * tri + 2], b1)));
            g.deg = 0;
            tangent(&g);
            int li = d->tri_light[tri];
            if (li >= 0) {
                if (dot(g.sn, wi) > 0) Le = mk(d->light_Le[3 * li], d->light_Le[3 * li + 1], d->light_Le[3 * li + 2]);
                lpdf = 1.0 / s->larea[li];
                light = li;
            }
            m = tri_material(s, tri);
            surface = 1;
            /* The device replays at most MAX_PATH_VERTICES surface vertices
             * (paths that long occur only in closed scenes without Russian
             * roulette, where the reference's loop does not end). */
            if (P->nv == MAX_PATH_VERTICES) { P->overflow = 1; return; }
            add_vertex(P, tri);
        }
        int depth_here = P->nv - (surface ? 1 : 0);   /* BSDF factors in thr */
        if (!is_zero(Le)) {
            v3 c = mulv(thr, Le);
            if (tech == 0 || prev_spec) add_event(P, path_pixel, c, depth_here, light, Le);
            else if (tech == 2) {
                double G = gterm(prev_p, prev_n, prev_deg, g.p, g.sn, 0);
                double pdl = G == 0 ? 0 : lpdf / (nl * G);
                add_event(P, path_pixel, mul(c, prev_pdf / (prev_pdf + pdl)), depth_here, light, Le);
            }
        }
        if (!surface) return;
        int v = k + 1;
        if (tech != 0 && d->max_pv != -1 && v >= d->max_pv) return;
        if (tech != 0 && m.type != 1) {
            lpoint lp;
            if (sample_light(s, rnd(key, DIM_V(v) + D_LIGHT), rnd(key, DIM_V(v) + D_LIGHT + 1), &lp)) {
                v3 ppL = normalize(sub(lp.p, g.p));
                double pb;
                v3 fs = bsdf_eval(&m, &g, wi, ppL, &pb);
                double G = gterm(g.p, g.sn, 0, lp.p, lp.n, 0);
                v3 Lel = dot(lp.n, mul(ppL, -1)) > 0 ? lp.Le : mk(0, 0, 0);
                if (G != 0 && !is_zero(fs) && !is_zero(Lel) && visible(s, g.p, lp.p)) {
                    double w = 1;
                    if (tech == 2) { double pdl = lp.pdf / G; w = pdl / (pdl + pb); }
                    add_event(P, path_pixel, mul(mulv(mulv(thr, fs), Lel), w * G / lp.pdf), P->nv, lp.light, lp.Le);
                }
            }
        }
        int kv = tech == 0 ? k : v;
        if (tech != 0 && d->rr_depth != -1 && kv >= d->rr_depth) {
            double p = fmin(0.5, lum(thr));
            if (rnd(key, DIM_V(kv) + D_RR) > p) return;
            thr = mul(thr, 1.0 / p);
        }
        v3 wo;
        double pdf;
        int spec;
        v3 wgt = bsdf_sample(&m, &g, wi, rnd(key, DIM_V(kv) + D_BSDF), rnd(key, DIM_V(kv) + D_BSDF + 1),
                             rnd(key, DIM_V(kv) + D_COMP), &wo, &pdf, &spec);
        if (is_zero(wgt)) return;
        thr = mulv(thr, wgt);
        if (tech == 0 && d->rr_depth != -1 && k >= d->rr_depth) {
            double p = fmin(0.5, lum(thr));
            if (rnd(key, DIM_V(k) + D_RR) > p) return;
            thr = mul(thr, 1.0 / p);
        }
        if (tech == 0 && d->max_pv != -1 && k + 1 >= d->max_pv) return;
        prev_p = g.p; prev_n = g.sn; prev_deg = 0; prev_spec = spec; prev_pdf = pdf;
        ro = g.p; rd = wo; tmin = EPS;
    }
}

/* Renders samples [sample_begin, sample_end) into film (W*H*3 doubles,
 * accumulated, not rescaled). Returns the number of samples. */
int64_t orc_render(const orc_pt_desc* d, double* film)
{
    pt_scene s;
    if (!setup(&s, d)) { teardown(&s); return -1; }
    path_t* P = path_new();
    for (int64_t smp = d->sample_begin; smp < d->sample_end; smp++) {
        run_sample(&s, (uint64_t)smp, P);
        for (int e = 0; e < P->nev; e++) {
            film[3 * P->ev[e].pixel] += P->ev[e].c.x;
            film[3 * P->ev[e].pixel + 1] += P->ev[e].c.y;
            film[3 * P->ev[e].pixel + 2] += P->ev[e].c.z;
        }
    }
    path_free(P);
    teardown(&s);
    return d->sample_end - d->sample_begin;
}

/* FP64 reference gradient of a loss L(image): given dL/dI (W*H*3, already
 * including the film rescale factor), adds dL/d(albedo) (3 per triangle;
 * diffuse BSDFs only) and dL/d(Le) (3 per area light) over samples
 * [sample_begin, sample_end). Each contribution is a product of the albedos
 * of the surface vertices on its prefix (linear in each) and of its light's
 * Le (linear). MIS weights and sampling densities do not depend on these
 * parameters. Russian-roulette probabilities p = min(0.5, lum(thr)) are held
 * at their sampled values: the expected image does not depend on p, so this
 * is an unbiased estimate of the gradient of the expected image (the terms
 * d(1/p) of the fixed-seed estimator cancel in expectation against its
 * jumps where a roulette decision flips). With Russian roulette disabled it
 * is the exact derivative of the fixed-seed estimator. */
int64_t orc_render_grad(const orc_pt_desc* d, const double* dL_dI, double* d_albedo, double* d_Le)
{
    pt_scene s;
    if (!setup(&s, d)) { teardown(&s); return -1; }
    path_t* P = path_new();
    for (int64_t smp = d->sample_begin; smp < d->sample_end; smp++) {
        run_sample(&s, (uint64_t)smp, P);
        for (int e = 0; e < P->nev; e++) {
            const event_t* ev = &P->ev[e];
            double w[3];
            for (int c = 0; c < 3; c++) w[c] = dL_dI[3 * ev->pixel + c] * comp(ev->c, c);
            for (int i = 0; i < ev->depth && i < P->nv; i++) {
                int tri = P->vtri[i];
                mat_t m = tri_material(&s, tri);
                if (m.type != 0) continue;
                for (int c = 0; c < 3; c++) {
                    double R = comp(m.R, c);
                    if (R != 0) d_albedo[3 * tri + c] += w[c] / R;
                }
            }
            if (ev->light >= 0 && ev->light < d->num_lights)
                for (int c = 0; c < 3; c++) {
                    double le = comp(ev->Le, c);
                    if (le != 0) d_Le[3 * ev->light + c] += w[c] / le;
                }
        }
    }
    path_free(P);
    teardown(&s);
    return d->sample_end - d->sample_begin;
}

/* ------------------------------------------------ component evaluation -- */
/* The camera, sampling and BSDF functions above for caller-given inputs:
 * tests check them against the reference's component tests
 * (test.math.stats.cpp:32-84, test.perspectivecamera.cpp:84-194,
 * test.generalizedbsdf.cpp:129-268) and compare the device's versions with
 * them. */

/* UniformConcentricDiskSample: u (n x 2) -> points (n x 2). */
void orc_eval_disk(const double* u, int n, double* out)
{
    for (int i = 0; i < n; i++) concentric(u[2 * i], u[2 * i + 1], &out[2 * i], &out[2 * i + 1]);
}

/* CosineSampleHemisphere (math.stats.inl:64-69): u (n x 2) -> directions (n x 3). */
void orc_eval_cosine(const double* u, int n, double* out)
{
    for (int i = 0; i < n; i++) {
        double x, y;
        concentric(u[2 * i], u[2 * i + 1], &x, &y);
        out[3 * i] = x;
        out[3 * i + 1] = y;
        out[3 * i + 2] = sqrt(fmax(0.0, 1 - x * x - y * y));
    }
}

/* The camera of d (eye, center, up, fovy, width, height; no geometry is
 * needed): raster positions (n x 2) -> ray origin and direction (n x 6) and
 * the importance pdf (n). Returns 0 for a degenerate camera. */
int orc_camera_rays(const orc_pt_desc* d, const double* raster, int n, double* rays, double* pdf)
{
    pt_scene s;
    const int ok = setup(&s, d);
    for (int i = 0; ok && i < n; i++) {
        v3 w = cam_dir(&s, raster[2 * i], raster[2 * i + 1], &pdf[i]);
        rays[6 * i] = s.cam_p.x; rays[6 * i + 1] = s.cam_p.y; rays[6 * i + 2] = s.cam_p.z;
        rays[6 * i + 3] = w.x; rays[6 * i + 4] = w.y; rays[6 * i + 5] = w.z;
    }
    teardown(&s);
    return ok;
}

/* The lights of d: (u0, u1) (n x 2) -> the point sample_light draws
 * (position, normal, area pdf times the selection probability; n x 7) and
 * the light index (n; num_lights for the environment, -1 without lights).
 * Returns 0 if the scene cannot be set up. */
int orc_light_sample(const orc_pt_desc* d, const double* u, int n, double* out, int* light)
{
    pt_scene s;
    const int ok = setup(&s, d);
    for (int i = 0; ok && i < n; i++) {
        lpoint lp;
        double* o = out + 7 * i;
        if (sample_light(&s, u[2 * i], u[2 * i + 1], &lp)) {
            o[0] = lp.p.x; o[1] = lp.p.y; o[2] = lp.p.z;
            o[3] = lp.n.x; o[4] = lp.n.y; o[5] = lp.n.z;
            o[6] = lp.pdf;
            light[i] = lp.light;
        } else {
            for (int c = 0; c < 7; c++) o[c] = 0.0;
            light[i] = -1;
        }
    }
    teardown(&s);
    return ok;
}

/* RayToRasterPosition: rays (n x 6) -> raster (n x 2) and valid (n; 0 when
 * the direction leaves the film). Returns 0 for a degenerate camera. */
int orc_camera_raster(const orc_pt_desc* d, const double* rays, int n, double* raster, int* valid)
{
    pt_scene s;
    const int ok = setup(&s, d);
    for (int i = 0; ok && i < n; i++) {
        double We;
        const double* r = rays + 6 * i;
        valid[i] = cam_project(&s, mk(r[0], r[1], r[2]), mk(r[3], r[4], r[5]), &raster[2 * i], &raster[2 * i + 1], &We);
    }
    teardown(&s);
    return ok;
}

static geom frame_of(const double* gnsn)
{
    geom g;
    memset(&g, 0, sizeof(g));
    g.gn = mk(gnsn[0], gnsn[1], gnsn[2]);
    g.sn = mk(gnsn[3], gnsn[4], gnsn[5]);
    tangent(&g);
    return g;
}

/* BSDF type (0 diffuse, 1 mirror, 2 diffuse-mirror) with reflectance R (3)
 * at frames given by geometric and shading normals (n x 6; tangents from the
 * shading normal, SurfaceGeometry::ComputeTangentSpace): SampleAndEstimate-
 * Direction (EL) for wi (n x 3) and u (n x 3: sample, component) -> wo,
 * weight (n x 3 each), pdf (n, projected solid angle) and specular (n). */
void orc_bsdf_sample(int type, const double* R, const double* frames, const double* wi, const double* u, int n,
                     double* wo, double* weight, double* pdf, int* spec)
{
    mat_t m;
    m.type = type;
    m.R = mk(R[0], R[1], R[2]);
    for (int i = 0; i < n; i++) {
        geom g = frame_of(frames + 6 * i);
        v3 o = mk(0, 0, 1);
        v3 w = bsdf_sample(&m, &g, mk(wi[3 * i], wi[3 * i + 1], wi[3 * i + 2]), u[3 * i], u[3 * i + 1], u[3 * i + 2],
                           &o, &pdf[i], &spec[i]);
        wo[3 * i] = o.x; wo[3 * i + 1] = o.y; wo[3 * i + 2] = o.z;
        weight[3 * i] = w.x; weight[3 * i + 1] = w.y; weight[3 * i + 2] = w.z;
    }
}

/* EvaluateDirection and EvaluateDirectionPDF for a NonDelta query (EL):
 * wi, wo (n x 3) -> f (n x 3) and pdf (n). */
void orc_bsdf_eval(int type, const double* R, const double* frames, const double* wi, const double* wo, int n,
                   double* f, double* pdf)
{
    mat_t m;
    m.type = type;
    m.R = mk(R[0], R[1], R[2]);
    for (int i = 0; i < n; i++) {
        geom g = frame_of(frames + 6 * i);
        v3 v = bsdf_eval(&m, &g, mk(wi[3 * i], wi[3 * i + 1], wi[3 * i + 2]), mk(wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]),
                         &pdf[i]);
        f[3 * i] = v.x; f[3 * i + 1] = v.y; f[3 * i + 2] = v.z;
    }
}
