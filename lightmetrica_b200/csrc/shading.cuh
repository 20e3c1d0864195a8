// Device-side surface geometry, BSDFs, lights and camera of the path tracer.
// Each function cites the reference routine whose behaviour it reproduces.
#pragma once
#include <cfloat>
#include <cstdint>
#include "scene.cuh"

namespace lmgpu {

struct V3 { float x, y, z; };
__device__ __forceinline__ V3 v3(float x, float y, float z) { return V3{ x, y, z }; }
__device__ __forceinline__ V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ V3 operator-(V3 a) { return v3(-a.x, -a.y, -a.z); }
__device__ __forceinline__ V3 operator*(V3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ V3 operator*(float s, V3 a) { return v3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ V3 operator*(V3 a, V3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ V3 operator/(V3 a, float s) { return v3(a.x / s, a.y / s, a.z / s); }
__device__ __forceinline__ float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V3 cross(V3 a, V3 b)
{
    return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float length2(V3 a) { return dot(a, a); }
__device__ __forceinline__ V3 normalize(V3 a) { return a * rsqrtf(dot(a, a)); }
__device__ __forceinline__ bool is_zero(V3 a) { return a.x == 0.0f && a.y == 0.0f && a.z == 0.0f; }
__device__ __forceinline__ float luminance(V3 v)
{   // math.vector.inl:500-506
    return 0.212671f * v.x + 0.715160f * v.y + 0.072169f * v.z;
}
__device__ __forceinline__ V3 load3(const float* p) { return v3(p[0], p[1], p[2]); }

constexpr float PI_F = 3.14159265358979323846f;
constexpr float INV_PI_F = 0.318309886183790671538f;
constexpr float EPS_F = 1e-4f;          // Math::Constants::Eps() (float)
constexpr float EPS_LARGE_F = 1e-3f;    // Math::Constants::EpsLarge() (float)

// SurfaceGeometry (surfacegeometry.h:36-64) with the shading frame as
// tangent vectors: shadingToWorld = [ss st sn], worldToShading its transpose.
struct Geom {
    V3 p, gn, sn, ss, st;
    float u, v;          // texture coordinates
    bool degenerated;
};

// OrthonormalBasis (math.linalgebra.inl:26-33): st from sn, ss = st x sn.
__device__ __forceinline__ void tangent_space(Geom& g)
{
    const V3 a = g.sn;
    g.st = fabsf(a.x) > fabsf(a.y) ? normalize(v3(a.z, 0.0f, -a.x)) : normalize(v3(0.0f, a.z, -a.y));
    g.ss = normalize(cross(g.st, a));
}
__device__ __forceinline__ V3 to_local(const Geom& g, V3 w) { return v3(dot(g.ss, w), dot(g.st, w), dot(g.sn, w)); }
__device__ __forceinline__ V3 to_world(const Geom& g, V3 l) { return g.ss * l.x + g.st * l.y + g.sn * l.z; }

// Scene::StoreIntersectionFromBarycentricCoords (scene.cpp:101-149).
__device__ __forceinline__ void surface_from_hit(const DeviceScene& s, int32_t tri, float b0, float b1,
                                                 V3 o, V3 d, float t, Geom& g)
{
    const uint32_t i1 = __ldg(s.tri_vidx + 3 * (int64_t)tri);
    const uint32_t i2 = __ldg(s.tri_vidx + 3 * (int64_t)tri + 1);
    const uint32_t i3 = __ldg(s.tri_vidx + 3 * (int64_t)tri + 2);
    g.p = o + d * t;
    const V3 p1 = load3(s.vpos + 3 * (int64_t)i1), p2 = load3(s.vpos + 3 * (int64_t)i2), p3 = load3(s.vpos + 3 * (int64_t)i3);
    g.gn = normalize(cross(p2 - p1, p3 - p1));
    const V3 n1 = load3(s.vnrm + 3 * (int64_t)i1), n2 = load3(s.vnrm + 3 * (int64_t)i2), n3 = load3(s.vnrm + 3 * (int64_t)i3);
    const float w0 = 1.0f - b0 - b1;
    g.sn = normalize(n1 * w0 + n2 * b0 + n3 * b1);
    const float* uv = s.vuv;
    g.u = uv[2 * i1] * w0 + uv[2 * i2] * b0 + uv[2 * i3] * b1;
    g.v = uv[2 * i1 + 1] * w0 + uv[2 * i2 + 1] * b0 + uv[2 * i3 + 1] * b1;
    g.degenerated = false;
    tangent_space(g);
}

// SphereEmitterShape::Intersect (emittershape.sphere.cpp:117-152): the
// environment's bounding sphere, tested only when no triangle was hit.
__device__ __forceinline__ bool env_sphere_intersect(const DeviceScene& s, V3 ro, V3 rd, float mint, float maxt, float& t)
{
    const V3 o = ro - load3(s.env_center);
    const float a = length2(rd);
    const float b = 2.0f * dot(o, rd);
    const float c = length2(o) - s.env_radius * s.env_radius;
    const float det = b * b - 4.0f * a * c;
    if (det < 0.0f) return false;
    const float e = sqrtf(det);
    const float denom = 2.0f * a;
    const float t0 = (-b - e) / denom;
    const float t1 = (-b + e) / denom;
    if (t0 > maxt || t1 < mint) return false;
    t = t0;
    if (t < mint) {
        t = t1;
        if (t > maxt) return false;
    }
    return true;
}

// SphereEmitterShape::StoreIntersection (emittershape.sphere.cpp:154-171).
__device__ __forceinline__ void env_surface(const DeviceScene& s, V3 o, V3 d, float t, Geom& g)
{
    g.p = o + d * t;
    g.gn = g.sn = normalize(load3(s.env_center) - g.p);
    g.u = g.v = 0.0f;
    g.degenerated = false;
    tangent_space(g);
}

}  // namespace lmgpu
