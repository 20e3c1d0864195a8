/*
 * lmgpu.h — C ABI of the lightmetrica B200 path-tracing core.
 *
 * This is the drop-in boundary for lightmetrica's scene-accelerator slot and
 * path-tracer bounce loop. A lightmetrica plugin (plugin.gpu.so) or any other
 * host program builds a scene from world-space primitives, then issues
 * intersection queries or whole renders. Plain C types only: no C++ or torch
 * types cross this boundary, and no exceptions escape it.
 *
 * Conventions
 *   - Every entry point returns an int status: LMGPU_OK (0) or a negative
 *     LMGPU_ERR_* code; lmgpu_last_error() gives a message for the calling
 *     thread.
 *   - Handles are opaque and freed only by their destroy call.
 *   - Caller buffers are borrowed for the duration of the call.
 *   - A handle is used by one host thread at a time; independent handles may
 *     run concurrently on separate CUDA streams.
 *   - `stream` arguments are cudaStream_t passed as void* (NULL = legacy
 *     default stream).
 */
#ifndef LMGPU_H
#define LMGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LMGPU_ABI_VERSION 1

/* ------------------------------------------------------------ status ---- */
enum {
    LMGPU_OK = 0,
    LMGPU_ERR_INVALID = -1,        /* bad argument or scene description */
    LMGPU_ERR_OOM = -2,            /* host or device allocation failed */
    LMGPU_ERR_CUDA = -3,           /* a CUDA call failed */
    LMGPU_ERR_STACK_OVERFLOW = -4, /* traversal stack exceeded (device flag) */
    LMGPU_ERR_QUEUE_OVERFLOW = -5, /* wavefront queue exceeded (device flag) */
    LMGPU_ERR_TIMEOUT = -6,        /* a bounded device wait gave up */
    LMGPU_ERR_UNSUPPORTED = -7,    /* feature not available for this scene */
    LMGPU_ERR_BOUNDS = -8          /* the bounds-checked build (liblmgpu_check.so) found
                                      an index out of range (device flag) */
};

/* ------------------------------------------------------------- scene ---- */

/* Acceleration layouts. BVH2 reproduces the reference `bvh` scene
 * (src/liblightmetrica/scene.bvh.cpp) exactly: same tree, same traversal
 * order, same float arithmetic, hence bit-identical closest hits. */
enum {
    LMGPU_LAYOUT_BVH2 = 0,   /* binary, children-in-parent 64 B nodes */
    LMGPU_LAYOUT_BVH4 = 1,   /* 4-wide collapse of the same tree, 128 B nodes */
    LMGPU_LAYOUT_NAIVE = 2,  /* brute force over all triangles (tiny scenes) */
    LMGPU_LAYOUT_BVH2Q = 3,  /* batch renders only: the binary render tree with 48 B nodes whose child
                                boxes are 16-bit planes on a per-node grid (boxes only grow) */
    LMGPU_LAYOUT_BVH2_QSHADOW = 4   /* batch renders only: float binary nodes for bounce rays,
                                       quantised ones (LMGPU_LAYOUT_BVH2Q) for shadow rays */
};

/* BSDFs (reference diffuse.cpp, mirror.cpp, plugin.diffusemirror). */
enum {
    LMGPU_BSDF_DIFFUSE = 0,
    LMGPU_BSDF_MIRROR = 1,
    LMGPU_BSDF_DIFFUSE_MIRROR = 2,
    LMGPU_BSDF_BLACK = 3
};

typedef struct LmgpuScene LmgpuScene;

/* The tree the path tracer traverses (LmgpuSceneDesc.render_tree). The
 * intersection entry points always use the reference's tree, whose closest
 * hits are bit-exact; renders need only the same expected image, so by
 * default they trace a second tree built for traversal cost: binned SAH over
 * all three axes (32 bins), leaves of up to 8 triangles. */
enum {
    LMGPU_RENDER_TREE_SAH = 0,        /* a separate render tree (default) */
    LMGPU_RENDER_TREE_REFERENCE = 1   /* render with the reference's tree */
};

/* One lightmetrica Primitive (reference include/lightmetrica/primitive.h:39-60)
 * with its TriangleMesh (trianglemesh.h:34-84). Vertices are in object space;
 * `transform` is the primitive's 4x4 matrix, column-major like the
 * reference's Math::Mat4 (NULL = identity) and is applied in the reference's
 * float order. `num_faces` counts triangles (the reference's NumFaces()/3). */
typedef struct {
    const float* positions;     /* 3 * num_vertices */
    const float* normals;       /* 3 * num_vertices, NULL = geometric normal */
    const float* texcoords;     /* 2 * num_vertices, NULL = none */
    const uint32_t* faces;      /* 3 * num_faces */
    int32_t num_vertices;
    int32_t num_faces;
    const float* transform;     /* 16 floats or NULL */
    int32_t material;           /* index into LmgpuSceneDesc.materials, -1 = black */
    int32_t area_light;         /* index into LmgpuSceneDesc.area_lights, -1 = none */
} LmgpuPrimitiveDesc;

typedef struct {
    int32_t type;               /* LMGPU_BSDF_* */
    float reflectance[3];       /* R (diffuse_reflectance / specular_reflectance) */
} LmgpuMaterialDesc;

typedef struct {
    float luminance[3];         /* reference light.area.cpp `luminance` (Le) */
} LmgpuAreaLightDesc;

typedef struct {
    const LmgpuPrimitiveDesc* primitives;
    int32_t num_primitives;
    const LmgpuMaterialDesc* materials;
    int32_t num_materials;
    const LmgpuAreaLightDesc* area_lights;
    int32_t num_area_lights;
    int32_t has_env_light;      /* reference light.env.const.cpp */
    float env_luminance[3];
    /* Pinhole camera (reference perspectivecamera.cpp; view = LookAt). */
    int32_t has_camera;
    float camera_eye[3];
    float camera_center[3];
    float camera_up[3];
    float camera_fovy_degrees;
    int32_t film_width;
    int32_t film_height;
    int32_t layout;             /* LMGPU_LAYOUT_* */
    int32_t build_threads;      /* host threads for the BVH build, 0 = all */
    int32_t max_stack_entries;  /* traversal stack bound per ray, 0 = automatic (2 * tree depth + 4,
                                   enough for every walk); a smaller bound makes the walks that
                                   need more fail with LMGPU_ERR_STACK_OVERFLOW (the status word
                                   the kernels raise). The multi-scene batch always uses the
                                   largest compiled bound. */
    int32_t render_tree;        /* LMGPU_RENDER_TREE_* (BVH layouts; 0 = SAH render tree) */
} LmgpuSceneDesc;

typedef struct {
    int64_t num_triangles;
    int64_t num_nodes;          /* binary BVH nodes (reference count) */
    int64_t num_leaves;
    int32_t max_depth;
    int32_t layout;
    int64_t device_bytes;       /* bytes in HBM of the traversal data: every tree in both layouts,
                                   the quantised render nodes and the triangle records */
    double build_seconds;       /* host BVH build time */
    float bounds_min[3];        /* Scene::GetAABBTriangles */
    float bounds_max[3];
    int32_t render_tree;        /* LMGPU_RENDER_TREE_* the renders traverse */
    int32_t render_max_depth;   /* render tree: depth, nodes, leaves, host build time */
    int64_t render_num_nodes;
    int64_t render_num_leaves;
    double render_build_seconds;
} LmgpuSceneInfo;

/* Replaces Scene::Load + Configure + Build (reference scene.h:47-191,
 * scene.bvh.cpp:202-268): builds the accelerator on the host and uploads it. */
int lmgpu_scene_create(const LmgpuSceneDesc* desc, LmgpuScene** out_scene);
int lmgpu_scene_destroy(LmgpuScene* scene);
int lmgpu_scene_info(const LmgpuScene* scene, LmgpuSceneInfo* info);

/* Host-only build of the same accelerator, without any device work: fills
 * `info` and, when `tri_order` is non-NULL (capacity >= triangles), the leaf
 * triangle order (the reference's bvhTriIndices, scene.bvh.cpp:193). For
 * validating the builder on machines without a GPU. */
int lmgpu_scene_build_host(const LmgpuSceneDesc* desc, LmgpuSceneInfo* info,
                           int32_t* tri_order, int64_t capacity);

/* ------------------------------------------------------ intersection ---- */

/* Ray batch, structure of arrays, DEVICE pointers (reference ray.h:37-45). */
typedef struct {
    const float* ox; const float* oy; const float* oz;
    const float* dx; const float* dy; const float* dz;
    const float* tmin; const float* tmax;
} LmgpuRaysSoA;

/* Closest-hit results, DEVICE pointers: triangle index in the reference's
 * TriAccel numbering (primitive-major, scene.bvh.cpp:210-247) or -1, the hit
 * distance t (the reference writes it to ray.maxT) and barycentrics (u, v). */
typedef struct {
    int32_t* tri_id; float* t; float* u; float* v;
} LmgpuHitsSoA;

/* Replaces BVHScene::IntersectTriangles for a batch (scene.bvh.cpp:390-448;
 * TriAccel::Intersect triaccel.h:100-160). Asynchronous on `stream`. */
int lmgpu_intersect(LmgpuScene* scene, const LmgpuRaysSoA* rays, int64_t n,
                    LmgpuHitsSoA* hits, void* stream);

/* Same query from HOST buffers: rays AoS (8 floats per ray: o.xyz, d.xyz,
 * minT, maxT), outputs to host arrays (any may be NULL). Copies in, traces,
 * copies out, synchronises; 2^20-ray chunks on four streams overlap their
 * uploads, traversals and downloads. Page-locked buffers (cudaMallocHost,
 * cudaHostRegister) are copied directly; pageable ones, in batches of 2^16
 * rays or more, through the scene's pinned staging (192 MB, allocated on
 * first use) filled and drained by a pool of host threads. */
int lmgpu_intersect_host(LmgpuScene* scene, const float* rays_aos, int64_t n,
                         int32_t* tri_id, float* t, float* u, float* v);

/* Any-hit visibility for shadow rays (reference RenderUtils::Visible,
 * renderutils.cpp:58-70): occluded[i] = 1 if any triangle is hit within
 * [tmin, tmax]. DEVICE pointers. */
int lmgpu_occluded(LmgpuScene* scene, const LmgpuRaysSoA* rays, int64_t n,
                   uint8_t* occluded, void* stream);

/* Full hit record for tests of Scene::Intersect (scene.cpp:67-72,
 * StoreIntersectionFromBarycentricCoords scene.cpp:101-149, emitter shapes
 * primitives.cpp:214-238): HOST buffers; geom gets 17 floats per ray
 * (p, gn, sn, ss, st, uv); kind[i] = 0 miss, 1 triangle, 2 environment. */
int lmgpu_intersect_full_host(LmgpuScene* scene, const float* rays_aos, int64_t n,
                              int32_t* tri_id, float* t, float* geom, int32_t* kind);

/* ------------------------------------------------------------ render ---- */

enum {
    LMGPU_RENDER_PT = 0,         /* reference pathtrace.cpp  ("pt") */
    LMGPU_RENDER_PT_DIRECT = 1,  /* reference pathtrace.direct.cpp ("pt.direct") */
    LMGPU_RENDER_PT_MIS = 2      /* reference pathtrace.mis.cpp ("pt.mis") */
};

enum {
    LMGPU_SAMPLING_STRATIFIED = 0, /* num_samples/(W*H) samples per pixel */
    LMGPU_SAMPLING_UNIFORM = 1     /* raster uniform over the film, as the reference */
};

typedef struct {
    int32_t technique;          /* LMGPU_RENDER_* */
    int32_t rr_depth;           /* reference `rr_depth` (default 1, -1 = off) */
    int32_t max_path_vertices;  /* reference `max_path_vertices` (-1 = unbounded) */
    int32_t sampling;           /* LMGPU_SAMPLING_* */
    uint64_t seed;
    int64_t num_samples;        /* reference `num_samples`: total samples */
    int64_t sample_offset;      /* first sample index (for splitting a budget) */
    int32_t film_fp64;          /* accumulate the film in FP64 (oracle runs) */
    int32_t wave_paths;         /* paths in flight per wave, 0 = automatic */
} LmgpuRenderParams;

typedef struct {
    int64_t rays_traced;        /* closest-hit + shadow rays */
    int64_t shadow_rays;
    int64_t paths;
    int32_t waves;
    int32_t max_bounces_run;
    double device_ms;           /* device time of the render (CUDA events) */
} LmgpuRenderStats;

/* Renders `num_samples` samples and writes the rescaled film (W*H*3 floats,
 * row y = 0 first, reference HDRBitmapFilm layout) to a HOST buffer:
 * the whole RenderProcessScheduler::Render (sched.mt.cpp:93-266) in one call.
 * Keeps a device film, its rescaled copy and a pinned host copy per device
 * between calls (about 3 * W*H*3*4 bytes for a float film); calls on one
 * device take turns. The calling thread's current device must be the scene's
 * (true of every call that takes a scene). */
int lmgpu_render(LmgpuScene* scene, const LmgpuRenderParams* params,
                 float* film_host, LmgpuRenderStats* stats);

/* Device variant: accumulates un-rescaled contributions into a DEVICE film
 * (float, or double when film_fp64) on `stream`; the caller rescales by
 * W*H/num_samples. The call returns once the render's device work is done
 * (it reads each bounce's queue sizes back to size the next launch). Waves
 * hold `wave_paths` paths (0 = 2^27, fewer if device memory is short) in a
 * workspace of about 216 bytes per path that is shared by all scenes of the
 * device and kept until exit; calls on one device take turns. */
int lmgpu_render_device(LmgpuScene* scene, const LmgpuRenderParams* params,
                        void* film_device, void* stream, LmgpuRenderStats* stats);

/* Frees what lmgpu_render_device and lmgpu_render keep on the calling
 * thread's current device between calls: the wave workspace (28.7 GB after
 * a 1080p 64-spp frame at the default wave size) and lmgpu_render's film
 * buffers. It waits for renders in progress on the device; the next render
 * allocates again. No counterpart in the reference, whose renderers hold
 * only host memory. */
int lmgpu_render_release(void);

/* Same render as lmgpu_render_device, but the call allocates no memory: no
 * cudaMalloc, cudaFree or allocating library routine. It has no counterpart
 * in the reference. It is for callers that cannot allocate device memory
 * while rendering: a host application's render callback under a memory
 * manager that forbids allocations, a process at its memory budget. The wave
 * workspace (path state and queues) lives in a static 32 MiB device array
 * that every GPU loading the library holds until exit; waves are at most
 * 155,343 paths, and a `wave_paths` above that returns LMGPU_ERR_INVALID
 * (0 = the maximum). The scene, created beforehand, and the DEVICE film
 * (float, or double with film_fp64; accumulated, not rescaled; the caller
 * zeroes it) are the caller's. The first call on each device looks up the
 * array's device address, so make it before any stream capture. All calls
 * share the one array, and the counters in it are cleared at the start of
 * each wave, but calls that overlap on the GPU race: run them one after
 * another. Like lmgpu_render_device, the call reads each bounce's queue
 * sizes back to the host, so it synchronises `stream` after every bounce. */
int lmgpu_render_device_noalloc(LmgpuScene* scene, const LmgpuRenderParams* params,
                                void* film_device, void* stream);

/* ---------------------------------------------------- differentiable ---- */

/* Parameters of the differentiable render, DEVICE pointers (NULL = the
 * scene's own values): per-triangle RGB albedo of diffuse BSDFs (3 floats per
 * triangle, reference TriAccel numbering) and per-area-light RGB emission
 * (3 floats per light). No reference counterpart: lightmetrica has no
 * differentiable renderer; these extend its pt / pt.direct / pt.mis. */
typedef struct {
    const float* albedo;
    const float* emission;
} LmgpuDiffParams;

/* Forward pass: renders `params` with `diff` into a DEVICE image (W*H*3,
 * accumulated with atomics, already rescaled by W*H/num_samples; the caller
 * zeroes it). Same estimator as lmgpu_render. */
int lmgpu_adjoint_forward(LmgpuScene* scene, const LmgpuRenderParams* params,
                          const LmgpuDiffParams* diff, float* image_device,
                          void* stream, LmgpuRenderStats* stats);

/* Adjoint pass: given dL/dimage (DEVICE, W*H*3, w.r.t. the rescaled image),
 * replays every sample's path from its random-number counters and adds
 * dL/d(albedo) (3 per triangle) and dL/d(emission) (3 per light) to the
 * DEVICE gradient buffers (FP32 atomics; the caller zeroes them). */
int lmgpu_adjoint_backward(LmgpuScene* scene, const LmgpuRenderParams* params,
                           const LmgpuDiffParams* diff, const float* dL_dimage_device,
                           float* d_albedo_device, float* d_emission_device,
                           void* stream, LmgpuRenderStats* stats);

/* ------------------------------------------------ multi-scene batch ---- */
/* No counterpart in the reference (its schedulers render one scene at a
 * time, sched.mt.cpp:93-266). A batch renders many independent scenes, each
 * with its own camera, film and render parameters, as one stream of waves:
 * a wave's paths span several scenes and every path carries its scene
 * index, so small scenes share the GPU instead of running one after the
 * other. Each wave (initialisation, every bounce, splat) is captured once
 * into a CUDA graph and replayed per wave with no host synchronisation in
 * between. Every scene renders exactly the samples it would render alone
 * with the same parameters (same random numbers, same paths). */
typedef struct LmgpuBatch LmgpuBatch;

enum {
    LMGPU_BATCH_WAVES = 0,   /* fixed waves: each wave's paths run to the end before the next wave */
    LMGPU_BATCH_STREAM = 1,  /* path regeneration: finished paths' slots take new paths every
                                iteration, so the queues stay full until the samples run out */
    LMGPU_BATCH_OVERLAP = 2  /* fixed waves in two path pools: a wave's tail (its bounces from
                                overlap_bounce on, where few paths are left) runs beside the
                                next wave's first bounces; twice the path-state memory.
                                Renders with unbounded depth run as LMGPU_BATCH_WAVES. */
};

typedef struct LmgpuBatchConfig {
    int32_t layout;               /* LMGPU_LAYOUT_BVH2, _BVH4, _BVH2Q or _BVH2_QSHADOW for every scene */
    int32_t wave_paths;           /* paths in flight: the capacity of the ray and shadow queues
                                     (per pool), in [1024, 2^27] */
    int32_t shade_blocks_per_sm;  /* grid of the shading kernel (blocks of 128 threads per SM) */
    int32_t use_graph;            /* 1: replay a captured CUDA graph (a wave, or two stream
                                     iterations); 0: direct launches */
    int32_t mode;                 /* LMGPU_BATCH_WAVES (default), _STREAM or _OVERLAP */
    int32_t overlap_bounce;       /* LMGPU_BATCH_OVERLAP: first bounce of a wave's tail, in
                                     [1, 64]; 0 = automatic (3) */
} LmgpuBatchConfig;

/* The scenes (built with a BVH layout, on the current device) must outlive
 * the batch; a scene may appear more than once. Default configuration:
 * BVH2, 2^27 paths in flight (about 288 bytes of path state per path, a
 * render allocating for min(2^27, its samples)), 16 shading blocks per SM,
 * graphs on, fixed waves (stream mode keeps every slot busy, but its
 * recycled slots scatter path state in memory: slower on the benchmark
 * scenes); a device short of memory gets fewer paths in flight. */
int lmgpu_batch_create(LmgpuScene* const* scenes, int32_t num_scenes, LmgpuBatch** out);
int lmgpu_batch_destroy(LmgpuBatch* batch);
int lmgpu_batch_get_config(const LmgpuBatch* batch, LmgpuBatchConfig* config);
int lmgpu_batch_set_config(LmgpuBatch* batch, const LmgpuBatchConfig* config);

/* Renders every scene of the batch: params[i] and films_device[i] belong to
 * scene i, with lmgpu_render_device's meaning (un-rescaled DEVICE film, float
 * or double by film_fp64; the caller zeroes it). All params share one
 * technique and one film type; wave_paths is ignored (the batch's
 * configuration sets it). Asynchronous on `stream` unless `stats` is given,
 * in which case the call synchronises, fills the totals of the batch and
 * reports the batch's device status (LMGPU_ERR_STACK_OVERFLOW,
 * LMGPU_ERR_QUEUE_OVERFLOW); without `stats`, a status raised by the call
 * is reported by the next call on the batch that synchronises. */
int lmgpu_batch_render_device(LmgpuBatch* batch, const LmgpuRenderParams* params,
                              void* const* films_device, void* stream, LmgpuRenderStats* stats);

/* Host-film variant: renders every scene like lmgpu_batch_render_device and
 * writes each scene's rescaled film (W*H*3 floats, the reference's
 * Rescale(W*H/num_samples), sched.mt.cpp:250-256) to the HOST buffer
 * films_host[i]: the batch counterpart of lmgpu_render. The batch keeps its
 * device films, their rescaled copies and a pinned host copy between calls
 * (about 3 * 12 bytes per pixel over all scenes for float films). Uses the
 * legacy default stream; synchronises. */
int lmgpu_batch_render(LmgpuBatch* batch, const LmgpuRenderParams* params, float* const* films_host,
                       LmgpuRenderStats* stats);

/* Measurement of one batch render (no counterpart in the reference). The
 * batch renders with direct launches in fixed waves (no graph; its
 * configuration is otherwise kept), records CUDA events on `stream` around
 * every traversal launch and, with count_tests, counts each traversal's
 * binary-node slab tests (four per 4-wide node) and TriAccel tests with a
 * counting copy of the traversal kernel, whose times are then not the
 * render's. Films as lmgpu_batch_render_device; synchronises. */
typedef struct {
    int64_t rays[2];            /* [0] closest-hit (path) rays, [1] shadow rays */
    int64_t launches[2];        /* traversal launches of each kind */
    double trace_ms[2];         /* summed device time of those launches */
    double render_ms;           /* device time of the whole render */
    uint64_t node_tests[2];     /* count_tests only: slab tests per kind */
    uint64_t tri_tests[2];      /* count_tests only: TriAccel tests per kind */
} LmgpuTraceProfile;
int lmgpu_batch_profile(LmgpuBatch* batch, const LmgpuRenderParams* params, void* const* films_device,
                        void* stream, int32_t count_tests, LmgpuTraceProfile* profile);

/* Autotuner: renders the batch with each scene's sample count scaled by
 * `sample_fraction` (0 < f <= 1; raised for a candidate until the trial
 * holds four of its waves, eight in overlap mode, or the whole render) under candidate
 * configurations (mode, BVH layout, paths in flight, shading grid, overlap
 * bounce), coordinate by coordinate, keeps the one with the least device
 * time per sample (a candidate must beat the incumbent, which starts as the
 * batch's configuration, by more than 0.5 %), stores it as the batch's
 * configuration and returns it
 * with that time scaled to `sample_fraction` of the samples, in ms. Films
 * are scratch memory of the tuner; synchronises. */
int lmgpu_batch_autotune(LmgpuBatch* batch, const LmgpuRenderParams* params, double sample_fraction,
                         void* stream, LmgpuBatchConfig* chosen, double* best_ms);

/* ------------------------------------------------ component evaluation ---- */
/* The path tracer's own device functions for caller-given inputs (host
 * arrays in and out; each call allocates scratch device memory and
 * synchronises: utility calls for checks and tools, not a hot path). They
 * answer what the reference's components answer for one query:
 *   lmgpu_eval_sampling          Math::UniformConcentricDiskSample /
 *                                CosineSampleHemisphere (math.stats.inl:25-69)
 *   lmgpu_camera_sample_rays     PerspectiveCamera::SamplePosition +
 *                                SampleDirection (perspectivecamera.cpp:170-240)
 *   lmgpu_camera_raster_positions  PerspectiveCamera::RayToRasterPosition
 *                                (perspectivecamera.cpp:304-323)
 *   lmgpu_film_pixels            the pixel HDRBitmapFilm::AccumulateContribution
 *                                adds a raster position to (hdrfilm.cpp:151-171)
 *   lmgpu_light_sample           Scene::SampleLightSelection (scene.cpp:79-86) and
 *                                the light's SamplePosition (light.area.cpp:146-179,
 *                                light.env.const.cpp:194-203)
 *   lmgpu_bsdf_sample            BSDF::SampleAndEstimateDirection, transport
 *                                EL (diffuse.cpp:133-157, mirror.cpp:84-107,
 *                                diffusemirror.cpp:84-125)
 *   lmgpu_bsdf_evaluate          BSDF::EvaluateDirection / EvaluateDirectionPDF
 *                                for a NonDelta query (diffuse.cpp:192-220)
 * Counts are in [0, 2^30]. */
enum {
    LMGPU_EVAL_CONCENTRIC_DISK = 0,     /* u (n x 2) -> point on the unit disk (n x 2) */
    LMGPU_EVAL_COSINE_HEMISPHERE = 1    /* u (n x 2) -> direction, +z hemisphere (n x 3) */
};
int lmgpu_eval_sampling(int32_t fn, const float* u, int64_t n, float* out);

/* The scene's camera: raster positions in [0,1]^2 (n x 2; y = 0 is the
 * bottom row) -> ray origin and direction (n x 6) and the importance pdf
 * (n, projected solid angle). */
int lmgpu_camera_sample_rays(const LmgpuScene* scene, const float* raster, int64_t n, float* rays, float* pdf);
/* Rays (n x 6: origin, direction) -> raster positions (n x 2) and valid (n;
 * 0 when the direction leaves the film). */
int lmgpu_camera_raster_positions(const LmgpuScene* scene, const float* rays, int64_t n, float* raster,
                                  int32_t* valid);
/* Raster positions (n x 2) -> pixel index y * W + x of the scene camera's
 * film (n; -1 outside [0,1]^2), as the renderers' film splats map them. */
int lmgpu_film_pixels(const LmgpuScene* scene, const float* raster, int64_t n, int32_t* pixel);
/* The scene's lights: (u0, u1) (n x 2) -> a point on the light chosen by u0
 * (n x 7: position, normal, area pdf times the selection probability) and
 * its index (n; num_area_lights for the environment, -1 without lights). */
int lmgpu_light_sample(const LmgpuScene* scene, const float* u, int64_t n, float* points, int32_t* light);

/* BSDF `type` (LMGPU_BSDF_*) with reflectance R (3 floats) at frames given by
 * geometric and shading normals (n x 6: gn, sn; tangents from sn as
 * SurfaceGeometry::ComputeTangentSpace makes them), for wi (n x 3, towards the
 * previous vertex) and u (n x 3: direction sample, component sample):
 * sampled wo (n x 3), weight f cos / pdf (n x 3), pdf (n, projected solid
 * angle) and specular (n, optional). */
int lmgpu_bsdf_sample(int32_t type, const float* reflectance, const float* frames, const float* wi, const float* u,
                      int64_t n, float* wo, float* weight, float* pdf, int32_t* specular);
/* f (n x 3) and pdf (n) of the non-delta part for wi, wo (n x 3 each). */
int lmgpu_bsdf_evaluate(int32_t type, const float* reflectance, const float* frames, const float* wi, const float* wo,
                        int64_t n, float* f, float* pdf);

/* ------------------------------------------------------------- misc ----- */
const char* lmgpu_last_error(void);
int lmgpu_abi_version(void);

/* Reads and clears the scene's device status word after asynchronous calls
 * (synchronises `stream`): traversal-stack or queue overflow and bounded-wait
 * timeouts raised inside kernels come back here as LMGPU_ERR_* codes. */
int lmgpu_scene_status(LmgpuScene* scene, void* stream);

/* Measurement variant of lmgpu_intersect: additionally adds the number of
 * binary-node slab tests and TriAccel tests of the batch to two DEVICE
 * unsigned long long counters (the reference's per-ray work, counted the way
 * scene.bvh.cpp:405-473 performs it). */
int lmgpu_intersect_counted(LmgpuScene* scene, const LmgpuRaysSoA* rays, int64_t n,
                            LmgpuHitsSoA* hits, unsigned long long* counters_device,
                            void* stream);

#ifdef __cplusplus
}
#endif
#endif /* LMGPU_H */
