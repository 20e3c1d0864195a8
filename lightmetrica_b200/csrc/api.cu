// C ABI: scene creation/upload and intersection queries.
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/lmgpu.h"
#include "builder.h"
#include "internal.h"
#include "trace.cuh"
#include "trace4.cuh"
#include "trace_kernels.cuh"
#include <condition_variable>
#include <functional>
#include <mutex>
#include <thread>
#include <unordered_map>

namespace lmgpu {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }

int fail(int code, const std::string& msg)
{
    g_last_error = msg;
    return code;
}

int cuda_fail(cudaError_t e, const char* what)
{
    g_last_error = std::string(what) + ": " + cudaGetErrorString(e);
    return LMGPU_ERR_CUDA;
}

int64_t check_limit_from_env(const char* name)
{
    const char* v = std::getenv(name);
    if (!v || !*v) return INT64_MAX;
    char* end = nullptr;
    const long long x = std::strtoll(v, &end, 10);
    return (end && *end == 0 && x >= 0) ? (int64_t)x : INT64_MAX;
}

int status_error(int32_t st)
{
    if (st & STATUS_BOUNDS) return fail(LMGPU_ERR_BOUNDS, "bounds check: index out of range");
    if (st & STATUS_STACK_OVERFLOW) return fail(LMGPU_ERR_STACK_OVERFLOW, "traversal stack bound exceeded");
    if (st & STATUS_QUEUE_OVERFLOW) return fail(LMGPU_ERR_QUEUE_OVERFLOW, "wavefront queue bound exceeded");
    if (st & STATUS_TIMEOUT) return fail(LMGPU_ERR_TIMEOUT, "bounded device wait gave up");
    return fail(LMGPU_ERR_CUDA, "unknown device status");
}

int consume_status(LmgpuScene* s, cudaStream_t stream)
{
    int32_t st = 0;
    LMGPU_CUDA_TRY(cudaMemcpyAsync(&st, s->d_status, sizeof(st), cudaMemcpyDeviceToHost, stream));
    LMGPU_CUDA_TRY(cudaStreamSynchronize(stream));
    if (st == 0) return LMGPU_OK;
    LMGPU_CUDA_TRY(cudaMemsetAsync(s->d_status, 0, sizeof(int32_t), stream));
    return status_error(st);
}

int resident_blocks_of(const void* kernel)
{
    static std::mutex mu;
    static std::unordered_map<const void*, int> cache;
    std::lock_guard<std::mutex> lock(mu);
    auto it = cache.find(kernel);
    if (it != cache.end()) return it->second;
    int per_sm = 0, sms = 0, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 128, 0);
    const int b = std::max(1, per_sm) * std::max(1, sms);
    cache[kernel] = b;
    return b;
}

namespace {

template <class T>
int upload(LmgpuScene* s, const std::vector<T>& v, const T** out)
{
    *out = nullptr;
    if (v.empty()) return LMGPU_OK;
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, v.size() * sizeof(T));
    if (e != cudaSuccess) return e == cudaErrorMemoryAllocation ? fail(LMGPU_ERR_OOM, "device allocation failed") : cuda_fail(e, "cudaMalloc");
    s->allocations.push_back(p);
    LMGPU_CUDA_TRY(cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
    *out = static_cast<const T*>(p);
    return LMGPU_OK;
}

#if LMGPU_BOUNDS_CHECK
// ---- tree references, checked on the device (bounds-checked build)
// A walk follows only the references stored in the nodes, from the root: if
// every internal reference is below the node limit and every leaf's run of
// TriRecords ends (TRI_LAST_IN_LEAF) inside the triangle array, no walk
// leaves the arrays. Leaves hold at most 255 triangles; a longer run fails.
__device__ bool leaf_in_range(int32_t ref, const TriRecord* tris, int64_t ntris)
{
    const int64_t first = ~(int64_t)ref;
    const int64_t end = first + 256 < ntris ? first + 256 : ntris;
    for (int64_t k = first; k < end; k++)
        if (tris[k].k_flags & TRI_LAST_IN_LEAF) return true;
    return false;
}
__device__ bool ref_in_range(int32_t ref, int64_t limit, const TriRecord* tris, int64_t ntris)
{
    return ref >= 0 ? ref < limit : leaf_in_range(ref, tris, ntris);
}
// One thread per node; node n (n < num, the array's size) is read only.
__global__ void k_check_bvh2(const Bvh2Node* nodes, int64_t num, int64_t limit, int32_t root,
                             const TriRecord* tris, int64_t ntris, int32_t* status)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0 && !ref_in_range(root, limit, tris, ntris)) atomicOr(status, STATUS_BOUNDS);
    if (i >= num) return;
    if (!ref_in_range(nodes[i].left, limit, tris, ntris) || !ref_in_range(nodes[i].right, limit, tris, ntris))
        atomicOr(status, STATUS_BOUNDS);
}
__global__ void k_check_bvh4(const Bvh4Node* nodes, int64_t num, int64_t limit, int32_t root,
                             const TriRecord* tris, int64_t ntris, int32_t* status)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0 && !ref_in_range(root, limit, tris, ntris)) atomicOr(status, STATUS_BOUNDS);
    if (i >= num) return;
    for (int c = 0; c < 4; c++) {
        const int32_t r = nodes[i].child[c];
        if (r != BVH4_EMPTY && !ref_in_range(r, limit, tris, ntris)) atomicOr(status, STATUS_BOUNDS);
    }
}

// Checks the uploaded trees of `d` (node counts n2 / n4, triangle count
// ntris) into the scene's status word and consumes it.
int check_trees(LmgpuScene* s, const DeviceScene& d, int64_t n2, int64_t n4, int64_t ntris)
{
    if (ntris <= 0) return LMGPU_OK;
    const int64_t lim = check_limit_from_env("LMGPU_CHECK_NODE_LIMIT");
    if (n2 > 0)
        k_check_bvh2<<<(unsigned)((n2 + 127) / 128), 128>>>(d.bvh2, n2, std::min(n2, lim), d.root_ref, d.tris, ntris,
                                                            s->d_status);
    if (n4 > 0)
        k_check_bvh4<<<(unsigned)((n4 + 127) / 128), 128>>>(d.bvh4, n4, std::min(n4, lim), d.root_ref4, d.tris, ntris,
                                                            s->d_status);
    LMGPU_CUDA_TRY(cudaGetLastError());
    return consume_status(s, nullptr);
}
#endif

// ---- camera matrices (reference math.transform.inl:88-113, perspectivecamera.cpp:97-160)
bool mat_inverse(const double* m, double* inv)
{
    // Gauss-Jordan on a row-major copy.
    double a[4][8];
    for (int r = 0; r < 4; r++)
        for (int c = 0; c < 4; c++) { a[r][c] = m[4 * c + r]; a[r][4 + c] = r == c ? 1.0 : 0.0; }
    for (int c = 0; c < 4; c++) {
        int piv = c;
        for (int r = c + 1; r < 4; r++) if (std::fabs(a[r][c]) > std::fabs(a[piv][c])) piv = r;
        if (a[piv][c] == 0.0) return false;
        if (piv != c) for (int k = 0; k < 8; k++) std::swap(a[c][k], a[piv][k]);
        const double d = a[c][c];
        for (int k = 0; k < 8; k++) a[c][k] /= d;
        for (int r = 0; r < 4; r++) {
            if (r == c) continue;
            const double f = a[r][c];
            for (int k = 0; k < 8; k++) a[r][k] -= f * a[c][k];
        }
    }
    for (int r = 0; r < 4; r++)
        for (int c = 0; c < 4; c++) inv[4 * c + r] = a[r][4 + c];
    return true;
}

void normalize3(double* v)
{
    const double l = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    for (int i = 0; i < 3; i++) v[i] /= l;
}

bool setup_camera(const LmgpuSceneDesc& d, CameraGpu& cam)
{
    std::memset(&cam, 0, sizeof(cam));
    if (!d.has_camera) return true;
    if (d.film_width <= 0 || d.film_height <= 0 || !(d.camera_fovy_degrees > 0.0f)) return false;
    if ((int64_t)d.film_width * d.film_height >= (int64_t(1) << 31)) return false;   // pixel indices are 32-bit
    double eye[3], ctr[3], up[3];
    for (int i = 0; i < 3; i++) { eye[i] = d.camera_eye[i]; ctr[i] = d.camera_center[i]; up[i] = d.camera_up[i]; }
    // LookAt: f = normalize(center - eye), s = normalize(f x up), u = s x f
    double f[3] = { ctr[0] - eye[0], ctr[1] - eye[1], ctr[2] - eye[2] };
    normalize3(f);
    double u[3] = { up[0], up[1], up[2] };
    normalize3(u);
    double s[3] = { f[1] * u[2] - f[2] * u[1], f[2] * u[0] - f[0] * u[2], f[0] * u[1] - f[1] * u[0] };
    normalize3(s);
    u[0] = s[1] * f[2] - s[2] * f[1]; u[1] = s[2] * f[0] - s[0] * f[2]; u[2] = s[0] * f[1] - s[1] * f[0];
    const double view[16] = { s[0], u[0], -f[0], 0, s[1], u[1], -f[1], 0, s[2], u[2], -f[2], 0,
                              -(s[0] * eye[0] + s[1] * eye[1] + s[2] * eye[2]),
                              -(u[0] * eye[0] + u[1] * eye[1] + u[2] * eye[2]),
                              (f[0] * eye[0] + f[1] * eye[1] + f[2] * eye[2]), 1 };
    const double aspect = double(d.film_width) / double(d.film_height);
    const double rad = double(d.camera_fovy_degrees) * 3.14159265358979323846 / 180.0;
    const double t = std::tan(rad / 2.0);
    const double zn = 1.0, zf = 1000.0;
    const double proj[16] = { 1.0 / (aspect * t), 0, 0, 0, 0, 1.0 / t, 0, 0,
                              0, 0, -(zf + zn) / (zf - zn), -1, 0, 0, -(2.0 * zf * zn) / (zf - zn), 0 };
    double iview[16], iproj[16];
    if (!mat_inverse(view, iview) || !mat_inverse(proj, iproj)) return false;
    for (int i = 0; i < 16; i++) {
        cam.view[i] = float(view[i]); cam.inv_view[i] = float(iview[i]);
        cam.proj[i] = float(proj[i]); cam.inv_proj[i] = float(iproj[i]);
    }
    for (int i = 0; i < 3; i++) cam.position[i] = float(iview[12 + i]);
    // Sensor area at distance 1 (perspectivecamera.cpp:145-156).
    auto unproj = [&](double x, double y, double* o) {
        double v[4] = { x, y, 0, 1 }, w[4];
        for (int r = 0; r < 4; r++) w[r] = iproj[r] * v[0] + iproj[4 + r] * v[1] + iproj[8 + r] * v[2] + iproj[12 + r] * v[3];
        for (int k = 0; k < 3; k++) o[k] = w[k] / w[3];
        for (int k = 0; k < 3; k++) o[k] = o[k] / o[2];
    };
    double p1[3], p2[3];
    unproj(-1, -1, p1);
    unproj(1, 1, p2);
    const double A = (p2[0] - p1[0]) * (p2[1] - p1[1]);
    cam.inv_A = float(1.0 / A);
    cam.width = d.film_width;
    cam.height = d.film_height;
    cam.valid = 1;
    return true;
}

int create_impl(const LmgpuSceneDesc* desc, LmgpuScene** out)
{
    if (!desc || !out) return fail(LMGPU_ERR_INVALID, "null argument");
    *out = nullptr;
    if (desc->num_primitives < 0 || (desc->num_primitives > 0 && !desc->primitives))
        return fail(LMGPU_ERR_INVALID, "bad primitive list");
    if (desc->max_stack_entries < 0) return fail(LMGPU_ERR_INVALID, "negative traversal stack bound");
    if (desc->render_tree != LMGPU_RENDER_TREE_SAH && desc->render_tree != LMGPU_RENDER_TREE_REFERENCE)
        return fail(LMGPU_ERR_INVALID, "unknown render tree");
    if (desc->layout < LMGPU_LAYOUT_BVH2 || desc->layout > LMGPU_LAYOUT_NAIVE)
        return fail(LMGPU_ERR_INVALID, "unknown layout");
    for (int i = 0; i < desc->num_primitives; i++) {
        const auto& p = desc->primitives[i];
        if (p.material >= desc->num_materials || p.area_light >= desc->num_area_lights)
            return fail(LMGPU_ERR_INVALID, "primitive references a missing material or light");
        if (p.positions && p.num_vertices > 0)
            for (int64_t k = 0; k < 3 * (int64_t)p.num_vertices; k++)
                if (!std::isfinite(p.positions[k])) return fail(LMGPU_ERR_INVALID, "non-finite vertex position");
    }
    for (int i = 0; i < desc->num_materials; i++)
        if (desc->materials[i].type < LMGPU_BSDF_DIFFUSE || desc->materials[i].type > LMGPU_BSDF_BLACK)
            return fail(LMGPU_ERR_INVALID, "unknown BSDF type");

    std::vector<PrimitiveInput> prims(desc->num_primitives);
    for (int i = 0; i < desc->num_primitives; i++) {
        const auto& p = desc->primitives[i];
        prims[i] = PrimitiveInput{ p.positions, p.normals, p.texcoords, p.faces, p.num_vertices, p.num_faces, p.transform };
    }
    BuiltScene b;
    std::string err;
    try {
        err = build_scene(prims, desc->build_threads, desc->layout != LMGPU_LAYOUT_NAIVE, b);
    } catch (const std::bad_alloc&) {
        return fail(LMGPU_ERR_OOM, "host allocation failed during the BVH build");
    }
    if (!err.empty()) return fail(LMGPU_ERR_INVALID, err);
    const bool render_tree = desc->layout != LMGPU_LAYOUT_NAIVE && desc->render_tree == LMGPU_RENDER_TREE_SAH &&
                             b.num_tris > 0;
    if (render_tree) {
        try {
            build_render_tree(b, desc->build_threads);
        } catch (const std::bad_alloc&) {
            return fail(LMGPU_ERR_OOM, "host allocation failed during the render tree build");
        }
    }

    CameraGpu cam;
    if (!setup_camera(*desc, cam)) return fail(LMGPU_ERR_INVALID, "invalid camera");

    LmgpuScene* s = new (std::nothrow) LmgpuScene;
    if (!s) return fail(LMGPU_ERR_OOM, "host allocation failed");
    LMGPU_CUDA_TRY(cudaGetDevice(&s->device));
    DeviceScene& d = s->dev;
    std::memset(&d, 0, sizeof(d));
    d.layout = desc->layout;
    d.num_tris = b.num_tris;
    d.root_ref = b.bvh2_root;
    d.root_ref4 = b.bvh4_root;
    d.stack_cap = 2 * b.max_depth + 4;
    if (desc->max_stack_entries > 0 && desc->max_stack_entries < d.stack_cap) d.stack_cap = desc->max_stack_entries;
    std::memcpy(d.root_box, b.root_box, sizeof(d.root_box));
    d.cam = cam;

    int rc = LMGPU_OK;
    auto up = [&](auto& vec, auto** dst) { if (rc == LMGPU_OK) rc = upload(s, vec, dst); };
    up(b.tris, &d.tris);
    up(b.bvh2, &d.bvh2);
    up(b.bvh4, &d.bvh4);
    std::vector<TriRecord> by_id;
    if (desc->layout == LMGPU_LAYOUT_NAIVE) {
        by_id.resize(b.tris.size());
        for (auto& t : b.tris) by_id[t.tri_id] = t;
        up(by_id, &d.tris_by_id);
    }
    up(b.positions, &d.vpos);
    up(b.normals, &d.vnrm);
    up(b.texcoords, &d.vuv);
    up(b.tri_vidx, &d.tri_vidx);
    up(b.tri_prim, &d.tri_prim);

    std::vector<int32_t> pm(desc->num_primitives), pl(desc->num_primitives);
    for (int i = 0; i < desc->num_primitives; i++) {
        pm[i] = desc->primitives[i].material;
        pl[i] = desc->primitives[i].area_light;
    }
    up(pm, &d.prim_material);
    up(pl, &d.prim_light);
    std::vector<float4> mats(std::max(1, desc->num_materials));
    for (int i = 0; i < desc->num_materials; i++) {
        const auto& m = desc->materials[i];
        float type_bits;
        std::memcpy(&type_bits, &m.type, sizeof(float));
        mats[i] = make_float4(m.reflectance[0], m.reflectance[1], m.reflectance[2], type_bits);
    }
    up(mats, &d.materials);
    d.num_materials = desc->num_materials;

    // Area lights: triangle-area CDF per light in primitive order
    // (light.area.cpp:109-144).
    std::vector<AreaLightGpu> lights(desc->num_area_lights);
    std::vector<float> cdf;
    std::vector<int32_t> ltris, guide;
    for (int li = 0; li < desc->num_area_lights; li++) {
        AreaLightGpu& L = lights[li];
        std::memset(&L, 0, sizeof(L));
        for (int c = 0; c < 3; c++) L.Le[c] = desc->area_lights[li].luminance[c];
        L.cdf_begin = static_cast<int32_t>(cdf.size());
        std::vector<double> acc{ 0.0 };
        for (int64_t t = 0; t < b.num_tris; t++) {
            if (desc->primitives[b.tri_prim[t]].area_light != li) continue;
            const float* p1 = &b.positions[3 * (size_t)b.tri_vidx[3 * t]];
            const float* p2 = &b.positions[3 * (size_t)b.tri_vidx[3 * t + 1]];
            const float* p3 = &b.positions[3 * (size_t)b.tri_vidx[3 * t + 2]];
            double e1[3], e2[3];
            for (int c = 0; c < 3; c++) { e1[c] = double(p2[c]) - p1[c]; e2[c] = double(p3[c]) - p1[c]; }
            const double cx = e1[1] * e2[2] - e1[2] * e2[1], cy = e1[2] * e2[0] - e1[0] * e2[2], cz = e1[0] * e2[1] - e1[1] * e2[0];
            acc.push_back(acc.back() + 0.5 * std::sqrt(cx * cx + cy * cy + cz * cz));
            ltris.push_back(static_cast<int32_t>(t));
        }
        const double area = acc.back();
        if (!(area > 0.0)) return fail(LMGPU_ERR_INVALID, "area light without area");
        for (double v : acc) cdf.push_back(float(v / area));
        L.num_tris = static_cast<int32_t>(acc.size() - 1);
        // Guide of the CDF search: the same float comparison the device makes.
        L.guide_begin = static_cast<int32_t>(guide.size());
        const float* lc = cdf.data() + L.cdf_begin;
        const int32_t n1 = L.num_tris + 1;
        for (int j = 0; j <= LIGHT_GUIDE_BINS; j++) {
            const float x = float(j) / float(LIGHT_GUIDE_BINS);
            guide.push_back(static_cast<int32_t>(std::upper_bound(lc, lc + n1, x) - lc));
        }
        guide.push_back(n1);
        L.area = float(area);
        L.inv_area = float(1.0 / area);
    }
    up(lights, &d.area_lights);
    up(cdf, &d.light_cdf);
    std::vector<float4> lrecs;
    lrecs.reserve(3 * ltris.size());
    for (int li = 0; li < desc->num_area_lights; li++) {
        const AreaLightGpu& L = lights[li];
        for (int32_t k = 0; k < L.num_tris; k++) {
            const int64_t t = ltris[(size_t)(L.cdf_begin - li + k)];
            const float* p[3];
            for (int c = 0; c < 3; c++) p[c] = &b.positions[3 * (size_t)b.tri_vidx[3 * t + c]];
            const float c0 = cdf[(size_t)(L.cdf_begin + k)], c1 = cdf[(size_t)(L.cdf_begin + k + 1)];
            lrecs.push_back(make_float4(p[0][0], p[0][1], p[0][2], p[1][0]));
            lrecs.push_back(make_float4(p[1][1], p[1][2], p[2][0], p[2][1]));
            lrecs.push_back(make_float4(p[2][2], c0, c1, 0.0f));
        }
    }
    up(lrecs, &d.light_recs);
    up(guide, &d.light_guide);
    d.num_area_lights = desc->num_area_lights;
    d.has_env = desc->has_env_light ? 1 : 0;
    d.num_lights = d.num_area_lights + d.has_env;
    if (d.has_env) {
        // Bounding sphere of triangles + camera (light.env.const.cpp:90-97, scene.cpp:58-65).
        float mn[3], mx[3];
        for (int c = 0; c < 3; c++) { mn[c] = b.bounds.mn[c]; mx[c] = b.bounds.mx[c]; }
        if (cam.valid)
            for (int c = 0; c < 3; c++) { mn[c] = std::min(mn[c], cam.position[c]); mx[c] = std::max(mx[c], cam.position[c]); }
        double r2 = 0;
        for (int c = 0; c < 3; c++) {
            d.env_center[c] = float((double(mx[c]) + mn[c]) / 2.0);
            const double dd = double(d.env_center[c]) - mx[c];
            r2 += dd * dd;
            d.env_Le[c] = desc->env_luminance[c];
        }
        d.env_radius = float(std::sqrt(r2));
        d.env_inv_area = float(1.0 / (4.0 * 3.14159265358979323846 * r2));
    }
    // Render view: the same scene with the render tree's accelerator.
    s->rdev = d;
    if (render_tree) {
        DeviceScene& r = s->rdev;
        up(b.rtris, &r.tris);
        up(b.rbvh2, &r.bvh2);
        up(b.rbvh4, &r.bvh4);
        r.root_ref = b.rbvh2_root;
        r.root_ref4 = b.rbvh4_root;
        std::memcpy(r.root_box, b.rroot_box, sizeof(r.root_box));
        r.stack_cap = 2 * b.rmax_depth + 4;
        if (desc->max_stack_entries > 0 && desc->max_stack_entries < r.stack_cap) r.stack_cap = desc->max_stack_entries;
    }
    // The quantised copy of the binary tree renders traverse (batch layout
    // LMGPU_LAYOUT_BVH2Q); rays start in the scene's bounds or at the camera.
    if (desc->layout != LMGPU_LAYOUT_NAIVE && b.num_tris > 0) {
        const std::vector<Bvh2QNode> qn = quantize_bvh2(render_tree ? b.rbvh2 : b.bvh2, b.bounds,
                                                        cam.valid ? cam.position : nullptr);
        up(qn, &s->rdev.bvh2q);
    }
    if (rc != LMGPU_OK) { lmgpu_scene_destroy(s); return rc; }

    // Scratch: status word and the persistent kernels' work counter.
    void* st = nullptr;
    const size_t scratch = 256 + LmgpuScene::WORK_SLOTS * sizeof(unsigned long long);
    cudaError_t e = cudaMalloc(&st, scratch);
    if (e != cudaSuccess) { lmgpu_scene_destroy(s); return cuda_fail(e, "cudaMalloc(status)"); }
    s->allocations.push_back(st);
    s->d_status = static_cast<int32_t*>(st);
    s->d_work = reinterpret_cast<unsigned long long*>(static_cast<char*>(st) + 256);
    LMGPU_CUDA_TRY(cudaMemset(st, 0, scratch));
#if LMGPU_BOUNDS_CHECK
    if (desc->layout != LMGPU_LAYOUT_NAIVE) {
        rc = check_trees(s, s->dev, (int64_t)b.bvh2.size(), (int64_t)b.bvh4.size(), (int64_t)b.tris.size());
        if (rc == LMGPU_OK && render_tree)
            rc = check_trees(s, s->rdev, (int64_t)b.rbvh2.size(), (int64_t)b.rbvh4.size(), (int64_t)b.rtris.size());
        if (rc != LMGPU_OK) { lmgpu_scene_destroy(s); return rc; }
    }
#endif

    LmgpuSceneInfo& info = s->info;
    info.num_triangles = b.num_tris;
    info.num_nodes = static_cast<int64_t>(b.nodes.size());
    info.num_leaves = b.num_leaves;
    info.max_depth = b.max_depth;
    info.layout = desc->layout;
    info.build_seconds = b.build_seconds;
    // Everything uploaded for traversal: both layouts of each tree (a batch
    // may pick either), the quantised copy of the render view's binary tree,
    // and the triangle records.
    int64_t bytes = 0;
    bytes += (int64_t)b.tris.size() * sizeof(TriRecord);
    bytes += (int64_t)b.bvh4.size() * sizeof(Bvh4Node) + (int64_t)b.bvh2.size() * sizeof(Bvh2Node);
    if (render_tree) {
        bytes += (int64_t)b.rtris.size() * sizeof(TriRecord);
        bytes += (int64_t)b.rbvh4.size() * sizeof(Bvh4Node) + (int64_t)b.rbvh2.size() * sizeof(Bvh2Node);
    }
    if (s->rdev.bvh2q) bytes += (int64_t)(render_tree ? b.rbvh2 : b.bvh2).size() * sizeof(Bvh2QNode);
    info.device_bytes = bytes;
    for (int c = 0; c < 3; c++) { info.bounds_min[c] = b.bounds.mn[c]; info.bounds_max[c] = b.bounds.mx[c]; }
    info.render_tree = render_tree ? LMGPU_RENDER_TREE_SAH : LMGPU_RENDER_TREE_REFERENCE;
    info.render_max_depth = render_tree ? b.rmax_depth : b.max_depth;
    info.render_num_nodes = render_tree ? b.rnum_nodes : static_cast<int64_t>(b.nodes.size());
    info.render_num_leaves = render_tree ? b.rnum_leaves : b.num_leaves;
    info.render_build_seconds = render_tree ? b.rbuild_seconds : 0.0;
    *out = s;
    return LMGPU_OK;
}

// ------------------------------------------------------------- kernels ----

// Ray source: SoA arrays (device API) or AoS records of 8 floats
// (o.xyz, d.xyz, minT, maxT; the host-buffer API), read with two 16 B loads.
struct RaySrc {
    LmgpuRaysSoA soa;
    const float4* aos;   // non-null selects AoS
};

__device__ __forceinline__ RayIn load_ray(const RaySrc& R, int64_t i)
{
    RayIn in;
    // Rays are read once: streaming loads keep them from evicting the BVH in L2.
    if (R.aos) {
        const float4 a = __ldcs(R.aos + 2 * i), b = __ldcs(R.aos + 2 * i + 1);
        in.o[0] = a.x; in.o[1] = a.y; in.o[2] = a.z;
        in.d[0] = a.w; in.d[1] = b.x; in.d[2] = b.y;
        in.tmin = b.z; in.tmax = b.w;
        return in;
    }
    in.o[0] = __ldcs(R.soa.ox + i); in.o[1] = __ldcs(R.soa.oy + i); in.o[2] = __ldcs(R.soa.oz + i);
    in.d[0] = __ldcs(R.soa.dx + i); in.d[1] = __ldcs(R.soa.dy + i); in.d[2] = __ldcs(R.soa.dz + i);
    in.tmin = __ldcs(R.soa.tmin + i); in.tmax = __ldcs(R.soa.tmax + i);
    return in;
}

__device__ __forceinline__ void store_hit(const LmgpuHitsSoA& hits, int64_t i, const Hit& h)
{
    const bool hit = h.tri >= 0;
    if (hits.tri_id) __stcs(hits.tri_id + i, h.tri);
    if (hits.t) __stcs(hits.t + i, hit ? h.t : 0.0f);
    if (hits.u) __stcs(hits.u + i, hit ? h.u : 0.0f);
    if (hits.v) __stcs(hits.v + i, hit ? h.v : 0.0f);
}

// I/O policy of the intersection API: SoA or AoS rays in, hit arrays out.
struct ApiHitIO {
    static constexpr int MIN_BLOCKS = LMGPU_TRACE_API_MIN_BLOCKS;
    RaySrc rays;
    int64_t n;
    LmgpuHitsSoA hits;
    __device__ int64_t count() const { return n; }
    __device__ RayIn load(int64_t i) const { return load_ray(rays, i); }
    __device__ void store(int64_t i, const Hit& h, const TraversalRay&) const { store_hit(hits, i, h); }
};

// I/O policy of the visibility API: occluded flag per ray.
struct ApiAnyIO {
    RaySrc rays;
    int64_t n;
    uint8_t* occluded;
    __device__ int64_t count() const { return n; }
    __device__ RayIn load(int64_t i) const { return load_ray(rays, i); }
    __device__ void store(int64_t i, const Hit& h, const TraversalRay&) const { occluded[i] = h.tri >= 0 ? 1 : 0; }
};

int launch_intersect(LmgpuScene* sc, const RaySrc& rays, int64_t n, const LmgpuHitsSoA& hits,
                     cudaStream_t stream, unsigned long long* counters)
{
    if (n == 0) return LMGPU_OK;
    if (!counters) return launch_trace<false>(sc, ApiHitIO{ rays, n, hits }, n, stream);
    // The counting instantiation of the same persistent kernel the path
    // tracer's measurement renders use.
    return launch_trace<false, ApiHitIO, true>(sc, ApiHitIO{ rays, n, hits }, n, stream, counters);
}

// Exposed for the measurement path (traversal counters).
}  // namespace

// Batches at least this large stage pageable caller buffers.
constexpr int64_t STAGE_MIN_RAYS = int64_t(1) << 16;

// True if p is page-locked host memory (copies from or to it can overlap
// kernels); pageable memory goes through the staged path below.
bool page_locked(const void* p)
{
    if (!p) return true;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

// A few host threads for the staged path's copies, started on first use and
// kept for the process's lifetime. run(n, fn) calls fn(0) .. fn(n - 1), on
// the pool and the calling thread, and returns when all have returned.
class CopyPool {
public:
    static CopyPool& get()
    {
        static CopyPool* pool = new CopyPool();     // never destroyed: no joins at exit
        return *pool;
    }
    int size() const { return static_cast<int>(workers.size()) + 1; }
    void run(int n, const std::function<void(int)>& fn)
    {
        std::lock_guard<std::mutex> serial(run_mu);
        {
            std::lock_guard<std::mutex> lock(mu);
            job = &fn;
            next = 1;
            count = n;
            pending = n - 1;
            ++generation;
        }
        cv.notify_all();
        if (n > 0) fn(0);
        for (;;) {                                  // help with the rest
            int i;
            {
                std::lock_guard<std::mutex> lock(mu);
                if (next >= count) break;
                i = next++;
            }
            fn(i);
            std::lock_guard<std::mutex> lock(mu);
            if (--pending == 0) done_cv.notify_all();
        }
        std::unique_lock<std::mutex> lock(mu);
        done_cv.wait(lock, [&] { return pending <= 0; });
        job = nullptr;
    }

private:
    CopyPool()
    {
        const unsigned hw = std::max(2u, std::thread::hardware_concurrency());
        const int n = static_cast<int>(std::min(8u, hw / 2)) - 1;
        for (int t = 0; t < n; t++) workers.emplace_back([this] { loop(); });
    }
    void loop()
    {
        uint64_t seen = 0;
        for (;;) {
            int i;
            const std::function<void(int)>* f;
            {
                std::unique_lock<std::mutex> lock(mu);
                cv.wait(lock, [&] { return generation != seen && next < count; });
                i = next++;
                f = job;
                if (next >= count) seen = generation;
            }
            (*f)(i);
            std::lock_guard<std::mutex> lock(mu);
            if (--pending == 0) done_cv.notify_all();
        }
    }
    std::vector<std::thread> workers;
    std::mutex mu, run_mu;
    std::condition_variable cv, done_cv;
    const std::function<void(int)>* job = nullptr;
    int next = 0, count = 0, pending = 0;
    uint64_t generation = 0;
};

// memcpy split over the copy pool (small copies stay on the calling thread).
void parallel_copy(void* dst, const void* src, size_t bytes)
{
    CopyPool& pool = CopyPool::get();
    const int parts = bytes < (size_t(1) << 21) ? 1 : pool.size();
    const size_t part = (bytes / parts + 63) / 64 * 64;
    pool.run(parts, [&](int i) {
        const size_t b = size_t(i) * part;
        if (b >= bytes) return;
        std::memcpy(static_cast<char*>(dst) + b, static_cast<const char*>(src) + b, std::min(part, bytes - b));
    });
}

int ensure_host_pipeline(LmgpuScene* sc)
{
    HostPipeline& hp = sc->pipe;
    if (hp.ready) return LMGPU_OK;
    hp.chunk = int64_t(1) << 20;   // 1M rays: 32 MB in, 16 MB out per stage
    for (int k = 0; k < HostPipeline::SLOTS; k++) {
        LMGPU_CUDA_TRY(cudaStreamCreateWithFlags(&hp.stream[k], cudaStreamNonBlocking));
        void* p = nullptr;
        LMGPU_CUDA_TRY(cudaMalloc(&p, (size_t)hp.chunk * 12 * sizeof(float)));
        sc->allocations.push_back(p);
        hp.rays[k] = static_cast<float*>(p);
        hp.hits[k] = hp.rays[k] + 8 * hp.chunk;
    }
    hp.ready = true;
    return LMGPU_OK;
}

// lmgpu_intersect_host for pageable caller buffers: copies to or from
// pageable memory cannot overlap anything and go through the driver's own
// staging (measured 7-10x slower than page-locked buffers on 2^24 rays), and
// registering the caller's pages costs more than the call. Instead the
// chunks pass through the pipeline's pinned buffers: while chunk c's
// upload, traversal and download run, the host copies chunk c's rays in
// and chunk c - SLOTS's hits out, split over a pool of host threads.
int intersect_host_staged(LmgpuScene* scene, const float* rays_aos, int64_t n, void* const* outs, bool stage_in,
                          bool stage_out)
{
    HostPipeline& hp = scene->pipe;
    const int64_t chunk = hp.chunk;
    for (int k = 0; k < HostPipeline::SLOTS; k++) {
        if (!hp.stage_rays[k]) LMGPU_CUDA_TRY(cudaMallocHost(&hp.stage_rays[k], (size_t)chunk * 8 * sizeof(float)));
        if (!hp.stage_hits[k]) LMGPU_CUDA_TRY(cudaMallocHost(&hp.stage_hits[k], (size_t)chunk * 4 * sizeof(float)));
        if (!hp.done[k]) LMGPU_CUDA_TRY(cudaEventCreateWithFlags(&hp.done[k], cudaEventDisableTiming));
    }
    const int64_t nchunks = (n + chunk - 1) / chunk;
    // Hands chunk c's hits (in slot c % SLOTS) to the caller's arrays.
    auto drain = [&](int64_t c) -> int {
        const int k = static_cast<int>(c % HostPipeline::SLOTS);
        const int64_t b = c * chunk, m = std::min(chunk, n - b);
        LMGPU_CUDA_TRY(cudaEventSynchronize(hp.done[k]));
        if (stage_out)
            for (int a = 0; a < 4; a++)
                if (outs[a])
                    parallel_copy(static_cast<char*>(outs[a]) + 4 * b, hp.stage_hits[k] + a * chunk, (size_t)m * 4);
        return LMGPU_OK;
    };
    int rc = LMGPU_OK;
    int64_t drained = 0;
    for (int64_t c = 0; c < nchunks && rc == LMGPU_OK; c++) {
        const int k = static_cast<int>(c % HostPipeline::SLOTS);
        if (c >= HostPipeline::SLOTS) {                 // the slot's previous chunk must be out
            rc = drain(c - HostPipeline::SLOTS);
            drained = c - HostPipeline::SLOTS + 1;
            if (rc != LMGPU_OK) break;
        }
        cudaStream_t st = hp.stream[k];
        const int64_t b = c * chunk, m = std::min(chunk, n - b);
        const float* src = rays_aos + 8 * b;
        if (stage_in) {
            parallel_copy(hp.stage_rays[k], src, (size_t)m * 8 * sizeof(float));
            src = hp.stage_rays[k];
        }
        cudaError_t e = cudaMemcpyAsync(hp.rays[k], src, (size_t)m * 8 * sizeof(float), cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) { rc = cuda_fail(e, "cudaMemcpyAsync(rays)"); break; }
        RaySrc rs;
        std::memset(&rs, 0, sizeof(rs));
        rs.aos = reinterpret_cast<const float4*>(hp.rays[k]);
        float* dh = hp.hits[k];
        LmgpuHitsSoA H{ reinterpret_cast<int32_t*>(dh), dh + chunk, dh + 2 * chunk, dh + 3 * chunk };
        rc = launch_intersect(scene, rs, m, H, st, nullptr);
        if (rc != LMGPU_OK) break;
        for (int a = 0; a < 4 && rc == LMGPU_OK; a++) {
            if (!outs[a]) continue;
            void* dst = stage_out ? static_cast<void*>(hp.stage_hits[k] + a * chunk) : static_cast<char*>(outs[a]) + 4 * b;
            e = cudaMemcpyAsync(dst, dh + a * chunk, (size_t)m * 4, cudaMemcpyDeviceToHost, st);
            if (e != cudaSuccess) rc = cuda_fail(e, "cudaMemcpyAsync(hits)");
        }
        if (rc == LMGPU_OK) {
            e = cudaEventRecord(hp.done[k], st);
            if (e != cudaSuccess) rc = cuda_fail(e, "cudaEventRecord");
        }
    }
    for (int64_t c = drained; c < nchunks && rc == LMGPU_OK; c++) rc = drain(c);
    for (int k = 0; k < HostPipeline::SLOTS; k++) {
        cudaError_t e = cudaStreamSynchronize(hp.stream[k]);
        if (e != cudaSuccess && rc == LMGPU_OK) rc = cuda_fail(e, "cudaStreamSynchronize");
    }
    if (rc == LMGPU_OK) rc = consume_status(scene, hp.stream[0]);
    return rc;
}

RaySrc soa_src(const LmgpuRaysSoA& r)
{
    RaySrc s;
    s.soa = r;
    s.aos = nullptr;
    return s;
}

}  // namespace lmgpu

using namespace lmgpu;

extern "C" {

int lmgpu_abi_version(void) { return LMGPU_ABI_VERSION; }

const char* lmgpu_last_error(void) { return g_last_error.c_str(); }

int lmgpu_scene_create(const LmgpuSceneDesc* desc, LmgpuScene** out_scene)
{
    try {
        return create_impl(desc, out_scene);
    } catch (const std::bad_alloc&) {
        return fail(LMGPU_ERR_OOM, "host allocation failed");
    } catch (...) {
        return fail(LMGPU_ERR_INVALID, "unexpected exception during scene creation");
    }
}

int lmgpu_scene_destroy(LmgpuScene* scene)
{
    if (!scene) return LMGPU_OK;
    if (scene->pipe.ready)
        for (int k = 0; k < HostPipeline::SLOTS; k++) {
            cudaStreamDestroy(scene->pipe.stream[k]);
            if (scene->pipe.stage_rays[k]) cudaFreeHost(scene->pipe.stage_rays[k]);
            if (scene->pipe.stage_hits[k]) cudaFreeHost(scene->pipe.stage_hits[k]);
            if (scene->pipe.done[k]) cudaEventDestroy(scene->pipe.done[k]);
        }
    for (void* p : scene->allocations) cudaFree(p);
    delete scene;
    return LMGPU_OK;
}

int lmgpu_scene_info(const LmgpuScene* scene, LmgpuSceneInfo* info)
{
    if (!scene || !info) return fail(LMGPU_ERR_INVALID, "null argument");
    *info = scene->info;
    return LMGPU_OK;
}

int lmgpu_intersect(LmgpuScene* scene, const LmgpuRaysSoA* rays, int64_t n, LmgpuHitsSoA* hits, void* stream)
{
    if (!scene || !rays || !hits || n < 0) return fail(LMGPU_ERR_INVALID, "null argument or negative count");
    if (const int rc = check_scene_device(scene)) return rc;
    if (n > 0 && (!rays->ox || !rays->oy || !rays->oz || !rays->dx || !rays->dy || !rays->dz || !rays->tmin || !rays->tmax))
        return fail(LMGPU_ERR_INVALID, "null ray array");
    return launch_intersect(scene, soa_src(*rays), n, *hits, static_cast<cudaStream_t>(stream), nullptr);
}

int lmgpu_occluded(LmgpuScene* scene, const LmgpuRaysSoA* rays, int64_t n, uint8_t* occluded, void* stream)
{
    if (!scene || !rays || !occluded || n < 0) return fail(LMGPU_ERR_INVALID, "null argument or negative count");
    if (const int rc = check_scene_device(scene)) return rc;
    if (n == 0) return LMGPU_OK;
    return launch_trace<true>(scene, ApiAnyIO{ soa_src(*rays), n, occluded }, n, static_cast<cudaStream_t>(stream));
}

int lmgpu_intersect_host(LmgpuScene* scene, const float* rays_aos, int64_t n, int32_t* tri_id, float* t, float* u, float* v)
{
    if (!scene || (n > 0 && !rays_aos) || n < 0) return fail(LMGPU_ERR_INVALID, "null argument or negative count");
    if (const int rc = check_scene_device(scene)) return rc;
    if (n == 0) return LMGPU_OK;
    // Chunked pipeline over HostPipeline::SLOTS streams: uploads, traversals
    // and downloads of neighbouring chunks overlap (full-duplex PCIe).
    // Staging buffers are cached in the scene.
    int rc = ensure_host_pipeline(scene);
    if (rc != LMGPU_OK) return rc;
    HostPipeline& hp = scene->pipe;
    const int64_t chunk = hp.chunk;
    const int64_t nchunks = (n + chunk - 1) / chunk;
    void* outs[4] = { tri_id, t, u, v };
    // Small batches (a renderer's single rays) copy directly: staging pays
    // off only when the copies are long enough to overlap.
    if (n >= STAGE_MIN_RAYS) {
        const bool stage_in = !page_locked(rays_aos);
        bool stage_out = false;
        for (void* o : outs) stage_out = stage_out || !page_locked(o);
        if (stage_in || stage_out) return intersect_host_staged(scene, rays_aos, n, outs, stage_in, stage_out);
    }
    for (int64_t c = 0; c < nchunks && rc == LMGPU_OK; c++) {
        const int k = static_cast<int>(c % HostPipeline::SLOTS);
        cudaStream_t st = hp.stream[k];
        const int64_t b = c * chunk, m = std::min(chunk, n - b);
        float* dr = hp.rays[k];
        float* dh = hp.hits[k];
        cudaError_t e = cudaMemcpyAsync(dr, rays_aos + 8 * b, (size_t)m * 8 * sizeof(float), cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) { rc = cuda_fail(e, "cudaMemcpyAsync(rays)"); break; }
        RaySrc src;
        std::memset(&src, 0, sizeof(src));
        src.aos = reinterpret_cast<const float4*>(dr);
        LmgpuHitsSoA H{ reinterpret_cast<int32_t*>(dh), dh + chunk, dh + 2 * chunk, dh + 3 * chunk };
        rc = launch_intersect(scene, src, m, H, st, nullptr);
        if (rc != LMGPU_OK) break;
        for (int a = 0; a < 4 && rc == LMGPU_OK; a++) {
            if (!outs[a]) continue;
            e = cudaMemcpyAsync(static_cast<char*>(outs[a]) + 4 * b, dh + a * chunk, (size_t)m * 4, cudaMemcpyDeviceToHost, st);
            if (e != cudaSuccess) rc = cuda_fail(e, "cudaMemcpyAsync(hits)");
        }
    }
    for (int k = 0; k < HostPipeline::SLOTS; k++) {
        cudaError_t e = cudaStreamSynchronize(hp.stream[k]);
        if (e != cudaSuccess && rc == LMGPU_OK) rc = cuda_fail(e, "cudaStreamSynchronize");
    }
    if (rc == LMGPU_OK) rc = consume_status(scene, hp.stream[0]);
    return rc;
}

// Traversal counters (binary slab tests, TriAccel tests) summed over a batch;
// counters must point to 2 device unsigned long long values (not cleared).
int lmgpu_intersect_counted(LmgpuScene* scene, const LmgpuRaysSoA* rays, int64_t n, LmgpuHitsSoA* hits,
                            unsigned long long* counters_device, void* stream)
{
    if (!scene || !rays || !hits || !counters_device || n < 0) return fail(LMGPU_ERR_INVALID, "null argument");
    if (const int rc = check_scene_device(scene)) return rc;
    return launch_intersect(scene, soa_src(*rays), n, *hits, static_cast<cudaStream_t>(stream), counters_device);
}

// Host-only build (no device work): info and, optionally, the leaf triangle
// order (the reference's bvhTriIndices, scene.bvh.cpp:193).
int lmgpu_scene_build_host(const LmgpuSceneDesc* desc, LmgpuSceneInfo* info, int32_t* tri_order, int64_t capacity)
{
    if (!desc || !info) return fail(LMGPU_ERR_INVALID, "null argument");
    std::vector<PrimitiveInput> prims(desc->num_primitives);
    for (int i = 0; i < desc->num_primitives; i++) {
        const auto& p = desc->primitives[i];
        prims[i] = PrimitiveInput{ p.positions, p.normals, p.texcoords, p.faces, p.num_vertices, p.num_faces, p.transform };
    }
    BuiltScene b;
    std::string err;
    try {
        err = build_scene(prims, desc->build_threads, desc->layout != LMGPU_LAYOUT_NAIVE, b);
    } catch (const std::bad_alloc&) {
        return fail(LMGPU_ERR_OOM, "host allocation failed during the BVH build");
    }
    if (!err.empty()) return fail(LMGPU_ERR_INVALID, err);
    std::memset(info, 0, sizeof(*info));
    info->num_triangles = b.num_tris;
    info->num_nodes = static_cast<int64_t>(b.nodes.size());
    info->num_leaves = b.num_leaves;
    info->max_depth = b.max_depth;
    info->layout = desc->layout;
    info->build_seconds = b.build_seconds;
    info->device_bytes = (int64_t)b.tris.size() * sizeof(TriRecord) +
                         (desc->layout == LMGPU_LAYOUT_BVH4 ? (int64_t)b.bvh4.size() * sizeof(Bvh4Node)
                                                            : (int64_t)b.bvh2.size() * sizeof(Bvh2Node));
    for (int c = 0; c < 3; c++) { info->bounds_min[c] = b.bounds.mn[c]; info->bounds_max[c] = b.bounds.mx[c]; }
    // The render tree, as lmgpu_scene_create builds it.
    if (desc->layout != LMGPU_LAYOUT_NAIVE && desc->render_tree == LMGPU_RENDER_TREE_SAH && b.num_tris > 0) {
        try {
            build_render_tree(b, desc->build_threads);
        } catch (const std::bad_alloc&) {
            return fail(LMGPU_ERR_OOM, "host allocation failed during the render tree build");
        }
        info->render_tree = LMGPU_RENDER_TREE_SAH;
        info->render_max_depth = b.rmax_depth;
        info->render_num_nodes = b.rnum_nodes;
        info->render_num_leaves = b.rnum_leaves;
        info->render_build_seconds = b.rbuild_seconds;
    } else {
        info->render_tree = LMGPU_RENDER_TREE_REFERENCE;
        info->render_max_depth = b.max_depth;
        info->render_num_nodes = info->num_nodes;
        info->render_num_leaves = b.num_leaves;
    }
    if (tri_order) {
        if (capacity < b.num_tris) return fail(LMGPU_ERR_INVALID, "tri_order capacity too small");
        std::memcpy(tri_order, b.tri_order.data(), (size_t)b.num_tris * sizeof(int32_t));
    }
    return LMGPU_OK;
}

// Status word of the last asynchronous calls on this scene (synchronises `stream`).
int lmgpu_scene_status(LmgpuScene* scene, void* stream)
{
    if (!scene) return fail(LMGPU_ERR_INVALID, "null scene");
    return consume_status(scene, static_cast<cudaStream_t>(stream));
}

}  // extern "C"
