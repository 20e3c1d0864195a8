// Component evaluation: the path tracer's own device functions (camera,
// sampling, BSDFs; pathtrace.cuh) run on caller-given inputs. The renderers
// inline the same functions, so checking these entry points against the
// reference's component tests (test.math.stats.cpp, test.perspectivecamera.cpp,
// test.generalizedbsdf.cpp) checks the code that renders. Host arrays in and
// out; each call allocates scratch device memory, copies, runs one kernel on
// the legacy default stream and synchronises: utility calls, not a hot path.
#include <cuda_runtime.h>
#include <algorithm>
#include <cstring>

#include "../../include/lmgpu.h"
#include "internal.h"
#include "pathtrace.cuh"

using namespace lmgpu;

namespace {

constexpr int64_t MAX_EVAL = int64_t(1) << 30;

unsigned eval_blocks(int64_t n) { return (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 127) / 128, 148 * 32)); }

__global__ void k_eval_sampling(int fn, const float* __restrict__ u, int64_t n, float* __restrict__ out)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float u0 = u[2 * i], u1 = u[2 * i + 1];
        if (fn == LMGPU_EVAL_CONCENTRIC_DISK) {
            float x, y;
            concentric_disk(u0, u1, x, y);
            out[2 * i] = x;
            out[2 * i + 1] = y;
        } else {
            const V3 d = cosine_hemisphere(u0, u1);
            out[3 * i] = d.x;
            out[3 * i + 1] = d.y;
            out[3 * i + 2] = d.z;
        }
    }
}

__global__ void k_camera_rays(const CameraGpu cam, const float* __restrict__ raster, int64_t n, float* __restrict__ rays,
                              float* __restrict__ pdf)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        float p;
        const V3 d = camera_direction(cam, raster[2 * i], raster[2 * i + 1], p);
        rays[6 * i] = cam.position[0];
        rays[6 * i + 1] = cam.position[1];
        rays[6 * i + 2] = cam.position[2];
        rays[6 * i + 3] = d.x;
        rays[6 * i + 4] = d.y;
        rays[6 * i + 5] = d.z;
        pdf[i] = p;
    }
}

__global__ void k_camera_raster(const CameraGpu cam, const float* __restrict__ rays, int64_t n, float* __restrict__ raster,
                                int32_t* __restrict__ valid)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float* r = rays + 6 * i;
        float rx, ry, imp;
        valid[i] = camera_project(cam, v3(r[0], r[1], r[2]), v3(r[3], r[4], r[5]), rx, ry, imp) ? 1 : 0;
        raster[2 * i] = rx;
        raster[2 * i + 1] = ry;
    }
}

// Scene::SampleLightSelection + the light's SamplePosition (sample_light)
// for given (u0, u1): position, normal, area pdf with the selection
// probability, and the light index per sample (-1 if the scene has no light).
__global__ void k_light_sample(const DeviceScene s, const float* __restrict__ u, int64_t n, float* __restrict__ out,
                               int32_t* __restrict__ light)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        LightPoint lp;
        float* o = out + 7 * i;
        if (sample_light(s, u[2 * i], u[2 * i + 1], lp)) {
            o[0] = lp.p.x; o[1] = lp.p.y; o[2] = lp.p.z;
            o[3] = lp.n.x; o[4] = lp.n.y; o[5] = lp.n.z;
            o[6] = lp.pdf_area;
            light[i] = lp.light;
        } else {
            for (int c = 0; c < 7; c++) o[c] = 0.0f;
            light[i] = -1;
        }
    }
}

__global__ void k_film_pixels(const CameraGpu cam, const float* __restrict__ raster, int64_t n, int32_t* __restrict__ pixel)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        pixel[i] = film_pixel(cam, raster[2 * i], raster[2 * i + 1]);
}

__device__ __forceinline__ Geom frame_of(const float* gnsn)
{
    Geom g;
    g.p = v3(0, 0, 0);
    g.gn = v3(gnsn[0], gnsn[1], gnsn[2]);
    g.sn = v3(gnsn[3], gnsn[4], gnsn[5]);
    g.u = g.v = 0.0f;
    g.degenerated = false;
    tangent_space(g);
    return g;
}

__global__ void k_bsdf_sample(const Material m, const float* __restrict__ frames, const float* __restrict__ wi,
                              const float* __restrict__ u, int64_t n, float* __restrict__ wo, float* __restrict__ weight,
                              float* __restrict__ pdf, int32_t* __restrict__ specular)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const Geom g = frame_of(frames + 6 * i);
        const BsdfSample s = sample_bsdf(m, g, v3(wi[3 * i], wi[3 * i + 1], wi[3 * i + 2]), u[3 * i], u[3 * i + 1], u[3 * i + 2]);
        wo[3 * i] = s.wo.x; wo[3 * i + 1] = s.wo.y; wo[3 * i + 2] = s.wo.z;
        weight[3 * i] = s.weight.x; weight[3 * i + 1] = s.weight.y; weight[3 * i + 2] = s.weight.z;
        pdf[i] = s.pdf;
        specular[i] = s.specular ? 1 : 0;
    }
}

__global__ void k_bsdf_eval(const Material m, const float* __restrict__ frames, const float* __restrict__ wi,
                            const float* __restrict__ wo, int64_t n, float* __restrict__ f, float* __restrict__ pdf)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const Geom g = frame_of(frames + 6 * i);
        float p;
        const V3 v = eval_bsdf(m, g, v3(wi[3 * i], wi[3 * i + 1], wi[3 * i + 2]), v3(wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]), p);
        f[3 * i] = v.x; f[3 * i + 1] = v.y; f[3 * i + 2] = v.z;
        pdf[i] = p;
    }
}

// Device scratch for one call: inputs copied in, outputs copied back, all
// freed on every path out.
struct Scratch {
    void* mem = nullptr;
    size_t used = 0;
    ~Scratch() { cudaFree(mem); }
    int reserve(size_t bytes)
    {
        cudaError_t e = cudaMalloc(&mem, bytes);
        if (e != cudaSuccess) {
            mem = nullptr;
            return e == cudaErrorMemoryAllocation ? fail(LMGPU_ERR_OOM, "device allocation failed") : cuda_fail(e, "cudaMalloc");
        }
        return LMGPU_OK;
    }
    template <class T>
    T* take(size_t count)
    {
        T* p = reinterpret_cast<T*>(static_cast<char*>(mem) + used);
        used += (count * sizeof(T) + 255) / 256 * 256;
        return p;
    }
};

size_t padded(size_t bytes) { return (bytes + 255) / 256 * 256; }

int copy_in(void* dst, const void* src, size_t bytes)
{
    LMGPU_CUDA_TRY(cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice));
    return LMGPU_OK;
}

// Copies the outputs back (each copy waits for the kernel on the legacy
// stream) and waits for that stream alone.
int finish(void* const* dst, void* const* src, const size_t* bytes, int k)
{
    LMGPU_CUDA_TRY(cudaGetLastError());
    for (int i = 0; i < k; i++)
        if (dst[i]) LMGPU_CUDA_TRY(cudaMemcpy(dst[i], src[i], bytes[i], cudaMemcpyDeviceToHost));
    LMGPU_CUDA_TRY(cudaStreamSynchronize(0));
    return LMGPU_OK;
}

int check_count(int64_t n)
{
    if (n < 0 || n > MAX_EVAL) return fail(LMGPU_ERR_INVALID, "count must be in [0, 2^30]");
    return LMGPU_OK;
}

int material_from(int32_t type, const float* R, Material& m)
{
    if (type < LMGPU_BSDF_DIFFUSE || type > LMGPU_BSDF_BLACK) return fail(LMGPU_ERR_INVALID, "unknown BSDF type");
    if (!R) return fail(LMGPU_ERR_INVALID, "null reflectance");
    m.type = type;
    m.R = V3{ R[0], R[1], R[2] };
    return LMGPU_OK;
}

}  // namespace

extern "C" {

int lmgpu_eval_sampling(int32_t fn, const float* u, int64_t n, float* out)
{
    if (fn != LMGPU_EVAL_CONCENTRIC_DISK && fn != LMGPU_EVAL_COSINE_HEMISPHERE)
        return fail(LMGPU_ERR_INVALID, "unknown sampling function");
    int rc = check_count(n);
    if (rc != LMGPU_OK || n == 0) return rc;
    if (!u || !out) return fail(LMGPU_ERR_INVALID, "null argument");
    const int oc = fn == LMGPU_EVAL_CONCENTRIC_DISK ? 2 : 3;
    const size_t bu = (size_t)n * 2 * sizeof(float), bo = (size_t)n * oc * sizeof(float);
    Scratch s;
    if ((rc = s.reserve(padded(bu) + padded(bo))) != LMGPU_OK) return rc;
    float* du = s.take<float>((size_t)n * 2);
    float* dout = s.take<float>((size_t)n * oc);
    if ((rc = copy_in(du, u, bu)) != LMGPU_OK) return rc;
    k_eval_sampling<<<eval_blocks(n), 128>>>(fn, du, n, dout);
    void* dst[1] = { out };
    void* src[1] = { dout };
    return finish(dst, src, &bo, 1);
}

int lmgpu_camera_sample_rays(const LmgpuScene* scene, const float* raster, int64_t n, float* rays, float* pdf)
{
    if (!scene) return fail(LMGPU_ERR_INVALID, "null scene");
    if (!scene->dev.cam.valid) return fail(LMGPU_ERR_INVALID, "scene has no camera");
    int rc = check_count(n);
    if (rc != LMGPU_OK || n == 0) return rc;
    if (!raster || !rays) return fail(LMGPU_ERR_INVALID, "null argument");
    const size_t b_in = (size_t)n * 2 * sizeof(float), b_rays = (size_t)n * 6 * sizeof(float), b_pdf = (size_t)n * sizeof(float);
    Scratch s;
    if ((rc = s.reserve(padded(b_in) + padded(b_rays) + padded(b_pdf))) != LMGPU_OK) return rc;
    float* d_in = s.take<float>((size_t)n * 2);
    float* d_rays = s.take<float>((size_t)n * 6);
    float* d_pdf = s.take<float>((size_t)n);
    if ((rc = copy_in(d_in, raster, b_in)) != LMGPU_OK) return rc;
    k_camera_rays<<<eval_blocks(n), 128>>>(scene->dev.cam, d_in, n, d_rays, d_pdf);
    void* dst[2] = { rays, pdf };
    void* src[2] = { d_rays, d_pdf };
    const size_t bytes[2] = { b_rays, b_pdf };
    return finish(dst, src, bytes, 2);
}

int lmgpu_camera_raster_positions(const LmgpuScene* scene, const float* rays, int64_t n, float* raster, int32_t* valid)
{
    if (!scene) return fail(LMGPU_ERR_INVALID, "null scene");
    if (!scene->dev.cam.valid) return fail(LMGPU_ERR_INVALID, "scene has no camera");
    int rc = check_count(n);
    if (rc != LMGPU_OK || n == 0) return rc;
    if (!rays || !raster) return fail(LMGPU_ERR_INVALID, "null argument");
    const size_t b_rays = (size_t)n * 6 * sizeof(float), b_out = (size_t)n * 2 * sizeof(float), b_valid = (size_t)n * 4;
    Scratch s;
    if ((rc = s.reserve(padded(b_rays) + padded(b_out) + padded(b_valid))) != LMGPU_OK) return rc;
    float* d_rays = s.take<float>((size_t)n * 6);
    float* d_out = s.take<float>((size_t)n * 2);
    int32_t* d_valid = s.take<int32_t>((size_t)n);
    if ((rc = copy_in(d_rays, rays, b_rays)) != LMGPU_OK) return rc;
    k_camera_raster<<<eval_blocks(n), 128>>>(scene->dev.cam, d_rays, n, d_out, d_valid);
    void* dst[2] = { raster, valid };
    void* src[2] = { d_out, d_valid };
    const size_t bytes[2] = { b_out, b_valid };
    return finish(dst, src, bytes, 2);
}

int lmgpu_light_sample(const LmgpuScene* scene, const float* u, int64_t n, float* points, int32_t* light)
{
    if (!scene) return fail(LMGPU_ERR_INVALID, "null scene");
    int rc = check_count(n);
    if (rc != LMGPU_OK || n == 0) return rc;
    if (!u || !points || !light) return fail(LMGPU_ERR_INVALID, "null argument");
    const size_t b_u = (size_t)n * 2 * sizeof(float), b_p = (size_t)n * 7 * sizeof(float), b_l = (size_t)n * 4;
    Scratch s;
    if ((rc = s.reserve(padded(b_u) + padded(b_p) + padded(b_l))) != LMGPU_OK) return rc;
    float* d_u = s.take<float>((size_t)n * 2);
    float* d_p = s.take<float>((size_t)n * 7);
    int32_t* d_l = s.take<int32_t>((size_t)n);
    if ((rc = copy_in(d_u, u, b_u)) != LMGPU_OK) return rc;
    k_light_sample<<<eval_blocks(n), 128>>>(scene->dev, d_u, n, d_p, d_l);
    void* dst[2] = { points, light };
    void* src[2] = { d_p, d_l };
    const size_t bytes[2] = { b_p, b_l };
    return finish(dst, src, bytes, 2);
}

int lmgpu_film_pixels(const LmgpuScene* scene, const float* raster, int64_t n, int32_t* pixel)
{
    if (!scene) return fail(LMGPU_ERR_INVALID, "null scene");
    if (!scene->dev.cam.valid) return fail(LMGPU_ERR_INVALID, "scene has no camera");
    int rc = check_count(n);
    if (rc != LMGPU_OK || n == 0) return rc;
    if (!raster || !pixel) return fail(LMGPU_ERR_INVALID, "null argument");
    const size_t b_in = (size_t)n * 2 * sizeof(float), b_out = (size_t)n * 4;
    Scratch s;
    if ((rc = s.reserve(padded(b_in) + padded(b_out))) != LMGPU_OK) return rc;
    float* d_in = s.take<float>((size_t)n * 2);
    int32_t* d_out = s.take<int32_t>((size_t)n);
    if ((rc = copy_in(d_in, raster, b_in)) != LMGPU_OK) return rc;
    k_film_pixels<<<eval_blocks(n), 128>>>(scene->dev.cam, d_in, n, d_out);
    void* dst[1] = { pixel };
    void* src[1] = { d_out };
    return finish(dst, src, &b_out, 1);
}

int lmgpu_bsdf_sample(int32_t type, const float* reflectance, const float* frames, const float* wi, const float* u,
                      int64_t n, float* wo, float* weight, float* pdf, int32_t* specular)
{
    Material m;
    int rc = material_from(type, reflectance, m);
    if (rc != LMGPU_OK) return rc;
    if ((rc = check_count(n)) != LMGPU_OK || n == 0) return rc;
    if (!frames || !wi || !u || !wo || !weight || !pdf) return fail(LMGPU_ERR_INVALID, "null argument");
    const size_t b6 = (size_t)n * 6 * sizeof(float), b3 = (size_t)n * 3 * sizeof(float), b1 = (size_t)n * 4;
    Scratch s;
    if ((rc = s.reserve(padded(b6) + 4 * padded(b3) + 2 * padded(b1))) != LMGPU_OK) return rc;
    float* d_frames = s.take<float>((size_t)n * 6);
    float* d_wi = s.take<float>((size_t)n * 3);
    float* d_u = s.take<float>((size_t)n * 3);
    float* d_wo = s.take<float>((size_t)n * 3);
    float* d_w = s.take<float>((size_t)n * 3);
    float* d_pdf = s.take<float>((size_t)n);
    int32_t* d_spec = s.take<int32_t>((size_t)n);
    if ((rc = copy_in(d_frames, frames, b6)) != LMGPU_OK || (rc = copy_in(d_wi, wi, b3)) != LMGPU_OK ||
        (rc = copy_in(d_u, u, b3)) != LMGPU_OK)
        return rc;
    k_bsdf_sample<<<eval_blocks(n), 128>>>(m, d_frames, d_wi, d_u, n, d_wo, d_w, d_pdf, d_spec);
    void* dst[4] = { wo, weight, pdf, specular };
    void* src[4] = { d_wo, d_w, d_pdf, d_spec };
    const size_t bytes[4] = { b3, b3, b1, b1 };
    return finish(dst, src, bytes, 4);
}

int lmgpu_bsdf_evaluate(int32_t type, const float* reflectance, const float* frames, const float* wi, const float* wo,
                        int64_t n, float* f, float* pdf)
{
    Material m;
    int rc = material_from(type, reflectance, m);
    if (rc != LMGPU_OK) return rc;
    if ((rc = check_count(n)) != LMGPU_OK || n == 0) return rc;
    if (!frames || !wi || !wo || !f || !pdf) return fail(LMGPU_ERR_INVALID, "null argument");
    const size_t b6 = (size_t)n * 6 * sizeof(float), b3 = (size_t)n * 3 * sizeof(float), b1 = (size_t)n * 4;
    Scratch s;
    if ((rc = s.reserve(padded(b6) + 3 * padded(b3) + padded(b1))) != LMGPU_OK) return rc;
    float* d_frames = s.take<float>((size_t)n * 6);
    float* d_wi = s.take<float>((size_t)n * 3);
    float* d_wo = s.take<float>((size_t)n * 3);
    float* d_f = s.take<float>((size_t)n * 3);
    float* d_pdf = s.take<float>((size_t)n);
    if ((rc = copy_in(d_frames, frames, b6)) != LMGPU_OK || (rc = copy_in(d_wi, wi, b3)) != LMGPU_OK ||
        (rc = copy_in(d_wo, wo, b3)) != LMGPU_OK)
        return rc;
    k_bsdf_eval<<<eval_blocks(n), 128>>>(m, d_frames, d_wi, d_wo, n, d_f, d_pdf);
    void* dst[2] = { f, pdf };
    void* src[2] = { d_f, d_pdf };
    const size_t bytes[2] = { b3, b1 };
    return finish(dst, src, bytes, 2);
}

}  // extern "C"
