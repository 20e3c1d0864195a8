// Device view of a built scene (all pointers are device memory), shared by
// the intersection and path-tracing kernels.
#pragma once
#include <cstdint>
#include "layout.h"

// 1 in the bounds-checked build (liblmgpu_check.so): the scene build checks
// every tree reference on the device, and every wavefront queue append is
// checked against the queue's capacity; a failed check sets a status word
// (LMGPU_ERR_BOUNDS / LMGPU_ERR_QUEUE_OVERFLOW), skips the access and never
// traps. The traversal stack bound is checked in every build.
#ifndef LMGPU_BOUNDS_CHECK
#define LMGPU_BOUNDS_CHECK 0
#endif

namespace lmgpu {

struct AreaLightGpu {
    float Le[3];
    float area, inv_area;
    int32_t cdf_begin;     // into DeviceScene::light_cdf; light_recs from cdf_begin - (light index)
    int32_t num_tris;
    int32_t guide_begin;   // into DeviceScene::light_guide (LIGHT_GUIDE_BINS + 2 entries)
};

// Guide of a light's CDF search: guide[j] = the first CDF index whose value
// exceeds j / LIGHT_GUIDE_BINS (j = 0 .. LIGHT_GUIDE_BINS), guide[BINS + 1] =
// num_tris + 1. The index sought for u lies in [guide[j], guide[j + 1]] for
// j = floor(u * BINS), so the search runs over a few entries and finds the
// same index as a search over the whole CDF.
constexpr int LIGHT_GUIDE_BINS = 256;
// Guide ranges of at most this many CDF entries are scanned, longer ones
// halved (sample_light).
constexpr int LIGHT_SCAN = 8;

// Pinhole camera (reference perspectivecamera.cpp:97-353). Matrices are
// column-major 4x4 like Math::Mat4.
struct CameraGpu {
    float view[16];
    float inv_view[16];
    float proj[16];
    float inv_proj[16];
    float position[3];
    float inv_A;           // 1 / sensor area at distance 1
    int32_t width, height;
    int32_t valid;
    int32_t pad;
};

struct DeviceScene {
    // ---- accelerator
    int32_t layout;
    int32_t root_ref;      // BVH2 root reference
    int32_t root_ref4;     // BVH4 root reference
    int32_t stack_cap;
    float root_box[6];     // lo.xyz, hi.xyz
    const Bvh2Node* bvh2;
    const Bvh4Node* bvh4;
    const Bvh2QNode* bvh2q;       // render view: the quantised copy of bvh2 (LMGPU_LAYOUT_BVH2Q)
    const TriRecord* tris;        // leaf order
    const TriRecord* tris_by_id;  // TriAccel order (naive layout)
    int64_t num_tris;

    // ---- geometry, TriAccel numbering
    const float* vpos;            // 3 per world vertex
    const float* vnrm;
    const float* vuv;
    const uint32_t* tri_vidx;     // 3 per triangle
    const int32_t* tri_prim;
    const int32_t* prim_material; // per primitive
    const int32_t* prim_light;    // per primitive: area light index or -1
    const float4* materials;      // (R.xyz, type bits)
    int32_t num_materials;

    // ---- lights: area lights [0, num_area_lights), then the environment
    int32_t num_area_lights;
    int32_t num_lights;
    int32_t has_env;
    const AreaLightGpu* area_lights;
    const float* light_cdf;       // per light: num_tris + 1 entries
    // Per light triangle, in CDF order (entry cdf_begin - li + idx for light
    // li): its vertices p1, p2, p3 and the CDF values around it, cdf[idx]
    // and cdf[idx + 1], as 3 float4 (p1.xyz p2.x | p2.yz p3.xy | p3.z c0 c1 -):
    // one 48-byte record instead of the chain triangle id -> vertex indices
    // -> positions after the CDF search.
    const float4* light_recs;
    const int32_t* light_guide;   // per light: LIGHT_GUIDE_BINS + 2 starting points of the CDF search
    float env_Le[3];
    float env_center[3];
    float env_radius;
    float env_inv_area;

    CameraGpu cam;
};

}  // namespace lmgpu
