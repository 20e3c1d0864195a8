// Camera, lights and BSDFs of the GPU path tracer (device functions).
// Directions are world space; "local" is the shading frame [ss st sn].
// Query conventions follow the reference: transport direction EL (from the
// eye), wi = direction towards the previous vertex, wo = sampled direction.
#pragma once
#include "shading.cuh"

namespace lmgpu {

// ------------------------------------------------------------ sampling -----

// UniformConcentricDiskSample (math.stats.inl:25-56), Shirley-Chiu mapping.
__device__ __forceinline__ void concentric_disk(float u0, float u1, float& x, float& y)
{
    const float v1 = 2.0f * u0 - 1.0f;
    const float v2 = 2.0f * u1 - 1.0f;
    float r, th;
    if (v1 == 0.0f && v2 == 0.0f) { x = y = 0.0f; return; }
    if (v1 > -v2) {
        if (v1 > v2) { r = v1; th = (PI_F / 4.0f) * v2 / v1; }
        else { r = v2; th = (PI_F / 4.0f) * (2.0f - v1 / v2); }
    } else {
        if (v1 < v2) { r = -v1; th = (PI_F / 4.0f) * (4.0f + v2 / v1); }
        else { r = -v2; th = (PI_F / 4.0f) * (6.0f - v1 / v2); }
    }
    float s, c;
    __sincosf(th, &s, &c);
    x = r * c;
    y = r * s;
}

// CosineSampleHemisphere (math.stats.inl:64-69).
__device__ __forceinline__ V3 cosine_hemisphere(float u0, float u1)
{
    float x, y;
    concentric_disk(u0, u1, x, y);
    return v3(x, y, sqrtf(fmaxf(0.0f, 1.0f - x * x - y * y)));
}

// ------------------------------------------------------------- camera -----

__device__ __forceinline__ float4 mat4_mul(const float* m, float x, float y, float z, float w)
{
    return make_float4(m[0] * x + m[4] * y + m[8] * z + m[12] * w,
                       m[1] * x + m[5] * y + m[9] * z + m[13] * w,
                       m[2] * x + m[6] * y + m[10] * z + m[14] * w,
                       m[3] * x + m[7] * y + m[11] * z + m[15] * w);
}

// PerspectiveCamera::EvaluateImportance (perspectivecamera.cpp:325-353).
__device__ __forceinline__ float camera_importance(const CameraGpu& c, float cos_theta)
{
    if (cos_theta <= 0.0f) return 0.0f;
    if (fabsf(cos_theta - 1.0f) < EPS_LARGE_F) cos_theta = 1.0f;
    const float inv = 1.0f / cos_theta;
    return c.inv_A * inv * inv * inv;
}

// Raster position of a stratified sample: pixel = sample mod (W*H), then
// ((x + u0) / W, (y + u1) / H). The render entry points keep the sample
// index below 2^53 and W*H below 2^31, so the quotient is estimated in
// double precision (the operands are exact and the product's relative
// error is below 2^-52: the estimate is off by at most one, then corrected)
// and the row and column come from a 32-bit division; the result equals
// the 64-bit integer remainder's.
__device__ __forceinline__ void stratified_raster(int64_t sample, int64_t pixels, double inv_pixels, int width,
                                                  int height, float u0, float u1, float& rx, float& ry)
{
    const int64_t q = (int64_t)(double(sample) * inv_pixels);
    int64_t pix = sample - q * pixels;
    if (pix < 0) pix += pixels;
    else if (pix >= pixels) pix -= pixels;
    const uint32_t w = (uint32_t)width, y = (uint32_t)pix / w, x = (uint32_t)pix - y * w;
    rx = (float(x) + u0) / float(width);
    ry = (float(y) + u1) / float(height);
}

// SampleAndEstimateDirection (perspectivecamera.cpp:216-240): raster in
// [0,1]^2 -> world direction; pdf = importance (projected solid angle);
// the estimated weight We/pdf is 1.
__device__ __forceinline__ V3 camera_direction(const CameraGpu& c, float rx, float ry, float& pdf)
{
    const float4 q = mat4_mul(c.inv_proj, rx * 2.0f - 1.0f, ry * 2.0f - 1.0f, 0.0f, 1.0f);
    const V3 dc = normalize(v3(q.x / q.w, q.y / q.w, q.z / q.w));
    pdf = camera_importance(c, -dc.z);
    const float4 w = mat4_mul(c.inv_view, dc.x, dc.y, dc.z, 0.0f);
    return normalize(v3(w.x, w.y, w.z));
}

// RayToRasterPosition (perspectivecamera.cpp:304-323) and the importance of
// EvaluateDirection / EvaluateDirectionPDF (:276-302, :355-383), which share
// the projection: returns false if the direction leaves the film.
__device__ __forceinline__ bool camera_project(const CameraGpu& c, V3 p, V3 d, float& rx, float& ry, float& importance)
{
    const V3 q = p + d;
    const float4 cam = mat4_mul(c.view, q.x, q.y, q.z, 1.0f);
    const float4 ndc = mat4_mul(c.proj, cam.x, cam.y, cam.z, cam.w);
    rx = (ndc.x / ndc.w + 1.0f) / 2.0f;
    ry = (ndc.y / ndc.w + 1.0f) / 2.0f;
    if (rx < 0.0f || rx > 1.0f || ry < 0.0f || ry > 1.0f) { importance = 0.0f; return false; }
    importance = camera_importance(c, -normalize(v3(cam.x, cam.y, cam.z)).z);
    return true;
}

// HDRBitmapFilm::AccumulateContribution pixel mapping (hdrfilm.cpp:151-171).
__device__ __forceinline__ int film_pixel(const CameraGpu& c, float rx, float ry)
{
    if (rx < 0.0f || rx > 1.0f || ry < 0.0f || ry > 1.0f) return -1;
    int x = static_cast<int>(rx * float(c.width));
    int y = static_cast<int>(ry * float(c.height));
    x = min(max(x, 0), c.width - 1);
    y = min(max(y, 0), c.height - 1);
    return y * c.width + x;
}

// ------------------------------------------------------------- lights -----

struct LightPoint {
    V3 p, n;            // position and normal (gn = sn)
    float pdf_area;     // area pdf including the selection probability
    V3 Le;
    int light;          // area light index, num_area_lights for the environment
};

// Scene::SampleLightSelection (scene.cpp:79-86, reuses u0) followed by
// AreaLight::SamplePosition (light.area.cpp:146-179) or
// ConstantEnvironmentLight::SamplePosition (light.env.const.cpp:194-203).
__device__ __forceinline__ bool sample_light(const DeviceScene& s, float u0, float u1, LightPoint& lp)
{
    const int nl = s.num_lights;
    if (nl <= 0) return false;
    const int li = min(static_cast<int>(u0 * float(nl)), nl - 1);
    u0 = u0 * float(nl) - float(li);
    const float sel = 1.0f / float(nl);
    if (li >= s.num_area_lights) {
        // uniform point on the bounding sphere, normal pointing inwards
        const float z = 1.0f - 2.0f * u0;
        const float r = sqrtf(fmaxf(0.0f, 1.0f - z * z));
        float sp, cp;
        __sincosf(2.0f * PI_F * u1, &sp, &cp);
        const V3 d = v3(r * cp, r * sp, z);
        lp.p = load3(s.env_center) + d * s.env_radius;
        lp.n = -d;
        lp.pdf_area = s.env_inv_area * sel;
        lp.Le = load3(s.env_Le);
        lp.light = li;
        return true;
    }
    const AreaLightGpu L = s.area_lights[li];
    const float* cdf = s.light_cdf + L.cdf_begin;
    // index = clamp(upper_bound(cdf, u1) - 1, 0, n - 1); the guide narrows
    // the search to the entries between two of its starting points.
    const int32_t* guide = s.light_guide + L.guide_begin;
    const int gj = min(static_cast<int>(u1 * float(LIGHT_GUIDE_BINS)), LIGHT_GUIDE_BINS);
    int lo = guide[gj], hi = guide[gj + 1];   // first element > u1 in [lo, hi), else hi
    if (hi - lo <= LIGHT_SCAN) {
        // The CDF does not decrease: the entries <= u1 are a prefix of the
        // range, counted with independent loads instead of dependent halvings.
        int below = 0;
#pragma unroll
        for (int k = 0; k < LIGHT_SCAN; k++)
            if (lo + k < hi && cdf[lo + k] <= u1) below++;
        lo += below;
    } else {
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (cdf[mid] > u1) hi = mid; else lo = mid + 1;
        }
    }
    const int idx = min(max(lo - 1, 0), L.num_tris - 1);
    const float4* rec = s.light_recs + 3 * (L.cdf_begin - li + idx);
    const float4 q0 = rec[0], q1 = rec[1], q2 = rec[2];
    const float c0 = q2.y, c1 = q2.z;          // cdf[idx], cdf[idx + 1]
    const float v = (u1 - c0) / (c1 - c0);
    const V3 p1 = v3(q0.x, q0.y, q0.z), p2 = v3(q0.w, q1.x, q1.y), p3 = v3(q1.z, q1.w, q2.x);
    // UniformSampleTriangle (math.stats.inl:120-125)
    const float sq = sqrtf(fmaxf(0.0f, u0));
    const float b0 = 1.0f - sq, b1 = v * sq;
    lp.p = p1 * (1.0f - b0 - b1) + p2 * b0 + p3 * b1;
    lp.n = normalize(cross(p2 - p1, p3 - p1));
    lp.pdf_area = L.inv_area * sel;
    lp.Le = load3(L.Le);
    lp.light = li;
    return true;
}

// RenderUtils::GeneralizedGeometryTerm (renderutils.cpp:29-56).
__device__ __forceinline__ float geometry_term(V3 p1, V3 n1, bool deg1, V3 p2, V3 n2, bool deg2)
{
    V3 d = p2 - p1;
    const float l2 = length2(d);
    const float l = sqrtf(l2);
    d = d / l;
    float num = 1.0f;
    if (!deg1) num *= fabsf(dot(n1, d));
    if (!deg2) num *= fabsf(dot(n2, -d));
    if (fabsf(l) < EPS_F) return 0.0f;
    return num / l2;
}

// -------------------------------------------------------------- BSDFs -----

struct Material {
    V3 R;
    int type;          // LMGPU_BSDF_*
};

__device__ __forceinline__ Material material_of(const DeviceScene& s, int prim)
{
    Material m;
    const int mi = s.prim_material[prim];
    if (mi < 0) { m.R = v3(0, 0, 0); m.type = LMGPU_BSDF_BLACK; return m; }
    const float4 q = s.materials[mi];
    m.R = v3(q.x, q.y, q.z);
    m.type = __float_as_int(q.w);
    return m;
}

// BSDF types with a non-delta component take next-event estimation
// (pathtrace.direct.cpp:206, GeneralizedBSDFType::NonDelta).
__device__ __forceinline__ bool has_non_delta(int type) { return type != LMGPU_BSDF_MIRROR; }

// BSDF::ShadingNormalCorrectionFactor (bsdf.h:57-83), EL transport: 0 when
// wi or wo lie on different sides of the geometric and shading normals.
__device__ __forceinline__ float shading_correction(const Geom& g, V3 wi, V3 wo, float wi_z, float wo_z)
{
    const float a = dot(wi, g.gn) * wi_z;
    const float b = dot(wo, g.gn) * wo_z;
    return (a <= 0.0f || b <= 0.0f) ? 0.0f : 1.0f;
}

struct BsdfSample {
    V3 wo;
    V3 weight;         // f * cos / pdf (0 = path ends)
    float pdf;         // projected solid angle
    bool specular;
};

// SampleAndEstimateDirection of diffuse.cpp:133-157, mirror.cpp:84-107,
// diffusemirror.cpp:84-125 (EL).
__device__ __forceinline__ BsdfSample sample_bsdf(const Material& m, const Geom& g, V3 wi, float u0, float u1, float uc)
{
    BsdfSample r;
    r.weight = v3(0, 0, 0);
    r.pdf = 0.0f;
    r.specular = false;
    r.wo = v3(0, 0, 1);
    const V3 lwi = to_local(g, wi);
    if (lwi.z <= 0.0f || m.type == LMGPU_BSDF_BLACK) return r;
    bool diffuse = m.type == LMGPU_BSDF_DIFFUSE || (m.type == LMGPU_BSDF_DIFFUSE_MIRROR && uc < 0.5f);
    V3 lwo;
    if (diffuse) {
        lwo = cosine_hemisphere(u0, u1);
        r.pdf = INV_PI_F * (m.type == LMGPU_BSDF_DIFFUSE_MIRROR ? 0.5f : 1.0f);
    } else {
        lwo = v3(-lwi.x, -lwi.y, lwi.z);
        r.pdf = (m.type == LMGPU_BSDF_DIFFUSE_MIRROR ? 0.5f : 1.0f) / lwo.z;
        r.specular = true;
    }
    r.wo = to_world(g, lwo);
    const float sf = shading_correction(g, wi, r.wo, lwi.z, lwo.z);
    r.weight = m.R * sf;        // diffuse: R sf; mirror: R sf; mix: sf R 0.5 / 0.5
    return r;
}

// EvaluateDirection and EvaluateDirectionPDF for a NonDelta query (EL).
__device__ __forceinline__ V3 eval_bsdf(const Material& m, const Geom& g, V3 wi, V3 wo, float& pdf)
{
    pdf = 0.0f;
    if (m.type == LMGPU_BSDF_MIRROR || m.type == LMGPU_BSDF_BLACK) return v3(0, 0, 0);
    const V3 lwi = to_local(g, wi), lwo = to_local(g, wo);
    if (lwi.z <= 0.0f || lwo.z <= 0.0f) return v3(0, 0, 0);
    const float k = m.type == LMGPU_BSDF_DIFFUSE_MIRROR ? 0.5f : 1.0f;
    pdf = INV_PI_F * k;
    const float sf = shading_correction(g, wi, wo, lwi.z, lwo.z);
    return m.R * (INV_PI_F * sf * k);
}

// Emitted radiance towards wo from a point with shading normal n (area
// light EvaluateDirection * EvaluatePosition = Le on the front side).
__device__ __forceinline__ V3 emitted(V3 Le, V3 n, V3 wo) { return dot(n, wo) > 0.0f ? Le : v3(0, 0, 0); }

}  // namespace lmgpu
