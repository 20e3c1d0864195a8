// Host-side scene builder: world-space triangles, TriAccel records and the
// binned-SAH BVH of the reference's `bvh` scene, flattened into the device
// layouts of layout.h.
#pragma once
#include <stdint.h>
#include <string>
#include <vector>
#include "layout.h"

namespace lmgpu {

struct HostAabb {
    float mn[3], mx[3];
};

// Binary BVH node as built (reference BVHNode, scene.bvh.cpp:35-73).
struct BuildNode {
    HostAabb bound;
    int32_t left = -1, right = -1;  // node indices (internal)
    int32_t begin = 0, end = 0;     // triangle range in tri_order (leaf)
    int32_t axis = 0;
    bool leaf = false;
};

struct BuiltScene {
    // Geometry in world space, reference TriAccel numbering.
    int64_t num_tris = 0;
    std::vector<float> positions;     // 3 per world vertex
    std::vector<float> normals;       // 3 per world vertex
    std::vector<float> texcoords;     // 2 per world vertex (zeros when absent)
    std::vector<uint32_t> tri_vidx;   // 3 per triangle, into the world vertex arrays
    std::vector<int32_t> tri_prim;    // primitive of each triangle
    std::vector<uint8_t> has_uv;      // per primitive
    HostAabb bounds;                  // GetAABBTriangles()

    // Reference-exact BVH.
    std::vector<BuildNode> nodes;     // arbitrary order
    int32_t root = -1;
    std::vector<int32_t> tri_order;   // bvhTriIndices
    int64_t num_leaves = 0;
    int32_t max_depth = 0;

    // Device layouts.
    std::vector<TriRecord> tris;      // leaf order
    std::vector<Bvh2Node> bvh2;
    int32_t bvh2_root = 0;            // root reference
    float root_box[6] = {0, 0, 0, 0, 0, 0};
    std::vector<Bvh4Node> bvh4;
    int32_t bvh4_root = 0;
    int32_t max_stack = 0;            // traversal stack bound for this tree
    double build_seconds = 0.0;

    // Render tree (build_render_tree): a second tree over the same TriAccel
    // records, for the path tracer only.
    bool has_render_tree = false;
    std::vector<TriRecord> rtris;     // its leaf order
    std::vector<Bvh2Node> rbvh2;
    int32_t rbvh2_root = 0;
    float rroot_box[6] = {0, 0, 0, 0, 0, 0};
    std::vector<Bvh4Node> rbvh4;
    int32_t rbvh4_root = 0;
    int64_t rnum_nodes = 0;
    int64_t rnum_leaves = 0;
    int32_t rmax_depth = 0;
    double rbuild_seconds = 0.0;
};

struct PrimitiveInput {
    const float* positions;
    const float* normals;
    const float* texcoords;
    const uint32_t* faces;
    int32_t num_vertices;
    int32_t num_faces;
    const float* transform;   // 16 floats column-major or nullptr
};

// The quantised copy of a binary tree (same node order and references) for
// rays that start within `bounds` (or at `extra`, a camera position): the
// grid step of an axis is a power of two no finer than 16 float ulps of the
// largest coordinate magnitude, so the decode's rounding stays below the
// two-step margin around every box.
std::vector<Bvh2QNode> quantize_bvh2(const std::vector<Bvh2Node>& nodes, const HostAabb& bounds,
                                     const float* extra);

// Builds everything; returns an empty string on success, else an error.
std::string build_scene(const std::vector<PrimitiveInput>& prims, int threads, bool want_bvh,
                        BuiltScene& out);

// Builds the render tree of a scene that build_scene built: a binned SAH
// tree over all three axes, for rendering only (closest hits may differ
// from the reference tree's at exact ties, never in expectation).
void build_render_tree(BuiltScene& s, int threads);

}  // namespace lmgpu
