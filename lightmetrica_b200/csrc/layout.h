// Device data layout of a built scene, shared by the host builder (g++) and
// the CUDA kernels (nvcc). Plain structs only.
//
// HBM layout of the binary accelerator (LMGPU_LAYOUT_BVH2):
//   Bvh2Node[num_internal]  64 B each, DFS pre-order, both children's boxes
//                           stored in the parent so one node fetch (4 x 16 B)
//                           serves both slab tests of a traversal step.
//   TriRecord[num_tris]     48 B each, the reference TriAccel constants
//                           (triaccel.h:31-47) permuted into leaf order
//                           (bvhTriIndices of scene.bvh.cpp:193); leaves are
//                           contiguous runs ended by TRI_LAST_IN_LEAF.
// A child reference >= 0 is an internal node index; < 0 is a leaf whose
// first TriRecord is ~ref.
#pragma once
#include <stdint.h>

namespace lmgpu {

constexpr uint32_t TRI_AXIS_MASK = 3u;          // TriAccel::k (3 = degenerate)
constexpr uint32_t TRI_LAST_IN_LEAF = 1u << 31; // last record of a leaf

struct alignas(16) Bvh2Node {
    // Per axis: left.lo, left.hi, right.lo, right.hi
    float bx[4];
    float by[4];
    float bz[4];
    int32_t left, right;   // child references
    int32_t axis;          // split axis of this node (near-first order)
    int32_t pad;
};
static_assert(sizeof(Bvh2Node) == 64, "Bvh2Node is 64 B");

// 4-wide collapse of the binary tree. Children are the grandchildren of a
// binary node in the reference's DFS order for a ray with all direction
// components positive; the three split axes let the kernel recover the
// reference order for any ray: child slot s = (h << 1) | l where h is the
// top split's side and l the second split's side.
struct alignas(16) Bvh4Node {
    float lox[4], hix[4];
    float loy[4], hiy[4];
    float loz[4], hiz[4];
    int32_t child[4];      // child references (0x7fffffff = empty slot)
    int32_t axis_top;      // split axis between slot pairs {0,1} and {2,3}
    int32_t axis_l;        // split axis inside {0,1} (-1: slot pair is one child)
    int32_t axis_r;        // split axis inside {2,3}
    int32_t pad;
};
static_assert(sizeof(Bvh4Node) == 128, "Bvh4Node is 128 B");
constexpr int32_t BVH4_EMPTY = 0x7fffffff;

// Quantised binary node (LMGPU_LAYOUT_BVH2Q, render trees only): the same
// tree as Bvh2Node with each child box on a per-node grid. Axis k's planes
// sit at origin[k] + q * 2^(e_k - 127) for 16-bit q, where e_k is byte k of
// `exps`. quantize_bvh2 (builder.cpp) chooses grid and q so that every
// quantised box contains its child's float box with a margin of two grid
// steps. 48 B: three 16-byte loads per visit instead of four.
struct alignas(16) Bvh2QNode {
    float origin[3];
    uint32_t exps;         // e_x | e_y << 8 | e_z << 16 | split axis << 24
    uint32_t q[6];         // axis k: q[2k] left child, q[2k + 1] right child, each lo | hi << 16
    int32_t left, right;   // child references as in Bvh2Node
};
static_assert(sizeof(Bvh2QNode) == 48, "Bvh2QNode is 48 B");

struct alignas(16) TriRecord {
    uint32_t k_flags;      // TriAccel::k | TRI_LAST_IN_LEAF
    float n_u, n_v, n_d;
    float a_u, a_v, b_nu, b_nv;
    float c_nu, c_nv;
    uint32_t tri_id;       // reference TriAccel index (primitive-major)
    uint32_t prim;         // primitive index
};
static_assert(sizeof(TriRecord) == 48, "TriRecord is 48 B");

}  // namespace lmgpu
