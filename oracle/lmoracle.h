/*
 * ORACLE — test infrastructure, not product code.
 *
 * Plain-C restatement of lightmetrica's scene-accelerator hot path, used only
 * as the checker by tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline. The product path (lightmetrica_b200) never links or calls it.
 *
 * Parity is pinned: tests/test_oracle_golden.py checks this restatement
 * against golden vectors produced by the reference's own sources compiled
 * unmodified (oracle/build_ref.sh -> oracle/_ref, tests/golden/gen_golden.py).
 */
#ifndef LMORACLE_H
#define LMORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Reference include/lightmetrica/triaccel.h:31-55 (float build). */
typedef struct {
    uint32_t k;
    float n_u, n_v, n_d;
    float a_u, a_v, b_nu, b_nv;
    float c_nu, c_nv;
    uint32_t shape_index, prim_index;
} orc_triaccel;

int orc_triaccel_load(orc_triaccel* ta, const float A[3], const float B[3], const float C[3]);
int orc_triaccel_intersect(const orc_triaccel* ta, const float o[3], const float d[3],
                           float mint, float maxt, float* u, float* v, float* t);

/* Scene kinds mirror the reference component names. */
enum { ORC_SCENE_BVH = 0, ORC_SCENE_NAIVE = 1 };

typedef struct orc_scene orc_scene;

/* World-space triangles (positions: 3 floats per vertex; faces: 3 indices per
 * triangle). Triangle i gets TriAccel index i, as scene.bvh.cpp:210-247 does
 * for one primitive with identity transform. */
orc_scene* orc_scene_create(int kind, const float* positions, int num_vertices,
                            const uint32_t* faces, int num_tris);
void orc_scene_destroy(orc_scene* s);

/* Closest-hit query for n rays (AoS, 8 floats: o, d, minT, maxT).
 * Outputs: tri_id (-1 on miss), t, u, v; node_tests / tri_tests (optional,
 * per ray) count AABB slab tests and TriAccel tests. Returns hits. */
int64_t orc_intersect(const orc_scene* s, int64_t n, const float* rays, int32_t* tri_id,
                      float* t, float* u, float* v, int32_t* node_tests, int32_t* tri_tests);

/* BVH statistics: number of nodes, leaves, maximum depth. */
void orc_scene_stats(const orc_scene* s, int64_t* nodes, int64_t* leaves, int32_t* max_depth);

/* Leaf triangle order (bvhTriIndices of scene.bvh.cpp:193), for layout tests. */
const int32_t* orc_scene_tri_order(const orc_scene* s);

#ifdef __cplusplus
}
#endif
#endif
