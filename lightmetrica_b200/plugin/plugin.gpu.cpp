// plugin.gpu.so — lightmetrica's Scene, Renderer and RenderProcessScheduler
// slots on the B200 core.
//
// A lightmetrica plugin in the reference's plugin ABI (plugin.common.h:82-103,
// plugin.common.cpp:97-110; the same kind of library as plugin/plugin.embree):
// build it against lightmetrica's headers with LM_USE_SINGLE_PRECISION together
// with lightmetrica's plugin.common.cpp, link it to liblmgpu.so, and put it
// where ComponentFactory::LoadPlugins finds it (component.cpp:61-120). It
// registers
//   Scene                   "plugin.gpu"     <scene type="plugin.gpu">
//   Renderer                "gpu.pt", "gpu.pt.direct", "gpu.pt.mis"
//                                            <renderer type="gpu.pt.mis">
//   RenderProcessScheduler  "gpu"            <render_scheduler type="gpu">
//
// Scene: Build() hands the primitives' meshes and transforms to
// lmgpu_scene_create, which builds the reference's binary SAH BVH on the host
// and uploads it; IntersectTriangles() answers one ray through
// lmgpu_intersect_host with the reference's closest hit bit for bit (same
// triangle, t and barycentrics) and fills the Intersection with the
// reference's own StoreIntersectionFromBarycentricCoords, exactly as BVHScene
// does (scene.bvh.cpp:390-403). The reference's renderers call
// IntersectTriangles from every OpenMP thread; the calls share the scene's
// staging buffers and take turns on a mutex. Build() also describes the
// scene's BSDFs, lights and camera to the core (see the helpers below), so
// the same device scene renders whole images.
//
// Renderers: the reference's pt / pt.direct / pt.mis (their configuration
// keys: rr_depth, max_path_vertices, sampler/rng_seed) rendered by the core
// over a "plugin.gpu" scene. Under the GPU scheduler a render is one call
// (lmgpu_render). Under any other scheduler (the reference's "mt") each
// render process counts the samples it is given and renders them on the GPU
// when the scheduler takes its film, so per-sample scheduling still works.
//
// Scheduler "gpu": the reference "mt" scheduler's keys and semantics
// (num_samples; the film accumulated, then rescaled by W*H / samples,
// sched.mt.cpp:240-256). A GPU renderer renders in one call; any other
// renderer goes to an internal "mt" scheduler configured with the same node.
//
// Configuration of the scene: <layout>bvh</layout> (default; bit-exact) or
// qbvh (4-wide collapse of the same tree, also bit-exact).
#include <lightmetrica/scene.h>
#include <lightmetrica/primitive.h>
#include <lightmetrica/primitives.h>
#include <lightmetrica/trianglemesh.h>
#include <lightmetrica/confignode.h>
#include <lightmetrica/intersection.h>
#include <lightmetrica/ray.h>
#include <lightmetrica/logger.h>
#include <lightmetrica/plugin.common.h>
#include <lightmetrica/renderer.h>
#include <lightmetrica/renderproc.h>
#include <lightmetrica/sched.h>
#include <lightmetrica/bsdf.h>
#include <lightmetrica/light.h>
#include <lightmetrica/camera.h>
#include <lightmetrica/film.h>
#include <lightmetrica/bitmapfilm.h>
#include <lightmetrica/bitmap.h>
#include <lightmetrica/generalizedbsdf.h>
#include <lightmetrica/surfacegeometry.h>
#include <lightmetrica/transportdirection.h>
#include <lightmetrica/math.functions.h>

#include <chrono>
#include <cmath>
#include <map>
#include <memory>
#include <mutex>
#include <random>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "lmgpu.h"

LM_NAMESPACE_BEGIN

namespace {

// The core's material for a reference BSDF: the type from the component's
// name; R from SampleAndEstimateDirection, whose weight is R times the
// shading-normal correction (1 here) for diffuse.cpp:133-157,
// mirror.cpp:84-107 and diffusemirror.cpp:84-125, queried with wi along the
// normal of a flat frame. The diffuse-mirror mix is queried on both
// components (uComp below and above 1/2) and must have one R.
bool MaterialOf(const BSDF* bsdf, LmgpuMaterialDesc& m, std::string& why)
{
    const std::string type = bsdf->ComponentImplTypeName();
    if (type == "diffuse") m.type = LMGPU_BSDF_DIFFUSE;
    else if (type == "mirror") m.type = LMGPU_BSDF_MIRROR;
    else if (type == "plugin.diffusemirror") m.type = LMGPU_BSDF_DIFFUSE_MIRROR;
    else
    {
        why = "BSDF '" + type + "' has no GPU counterpart";
        return false;
    }
    SurfaceGeometry geom;
    geom.degenerated = false;
    geom.p = Math::Vec3();
    geom.gn = geom.sn = Math::Vec3(Math::Float(0), Math::Float(0), Math::Float(1));
    geom.ComputeTangentSpace();
    auto weight = [&](Math::Float uComp) {
        GeneralizedBSDFSampleQuery q;
        q.type = GeneralizedBSDFType::AllBSDF;
        q.sample = Math::Vec2(Math::Float(0.5));
        q.uComp = uComp;
        q.transportDir = TransportDirection::EL;
        q.wi = geom.sn;
        GeneralizedBSDFSampleResult r;
        return bsdf->SampleAndEstimateDirection(q, geom, r);
    };
    const Math::Vec3 a = weight(Math::Float(0.25));
    if (m.type == LMGPU_BSDF_DIFFUSE_MIRROR)
    {
        const Math::Vec3 b = weight(Math::Float(0.75));
        if (a.x != b.x || a.y != b.y || a.z != b.z)
        {
            why = "diffuse-mirror BSDF with different diffuse and specular reflectances";
            return false;
        }
    }
    m.reflectance[0] = static_cast<float>(a.x);
    m.reflectance[1] = static_cast<float>(a.y);
    m.reflectance[2] = static_cast<float>(a.z);
    return true;
}

// Le of an area or constant environment light: EvaluatePosition is Le * pi
// for both (light.area.cpp:233-236, light.env.const.cpp:206-209).
Math::Vec3 LuminanceOf(const Light* light)
{
    SurfaceGeometry geom;
    geom.degenerated = false;
    geom.p = Math::Vec3();
    geom.gn = geom.sn = Math::Vec3(Math::Float(0), Math::Float(0), Math::Float(1));
    geom.ComputeTangentSpace();
    return light->EvaluatePosition(geom) / Math::Constants::Pi();
}

// Inverse of a column-major 4x4 matrix (Gauss-Jordan with partial pivoting).
bool Invert4(const double* m, double* inv)
{
    double a[4][8];
    for (int r = 0; r < 4; r++)
        for (int c = 0; c < 4; c++) { a[r][c] = m[4 * c + r]; a[r][4 + c] = r == c ? 1.0 : 0.0; }
    for (int c = 0; c < 4; c++)
    {
        int piv = c;
        for (int r = c + 1; r < 4; r++)
            if (std::fabs(a[r][c]) > std::fabs(a[piv][c])) piv = r;
        if (a[piv][c] == 0.0) return false;
        if (piv != c)
            for (int k = 0; k < 8; k++) std::swap(a[c][k], a[piv][k]);
        const double d = a[c][c];
        for (int k = 0; k < 8; k++) a[c][k] /= d;
        for (int r = 0; r < 4; r++)
        {
            if (r == c) continue;
            const double g = a[r][c];
            for (int k = 0; k < 8; k++) a[r][k] -= g * a[c][k];
        }
    }
    for (int r = 0; r < 4; r++)
        for (int c = 0; c < 4; c++) inv[4 * c + r] = a[r][4 + c];
    return true;
}

// The core's LookAt camera for a reference perspective camera, whose
// primitive's transform is its view matrix (perspectivecamera.cpp:174-184):
// eye, forward and up through the matrix's inverse; fovy from
// RayToRasterPosition of a ray 10 degrees above the axis (its raster y is
// (tan 10deg / tan(fovy / 2) + 1) / 2, perspectivecamera.cpp:304-323; the
// position is computed even when the ray leaves the film).
bool CameraOf(const Primitives& prims, LmgpuSceneDesc& d, std::string& why)
{
    const Camera* cam = prims.MainCamera();
    if (!cam)
    {
        why = "no camera";
        return false;
    }
    if (cam->ComponentImplTypeName() != "perspective")
    {
        why = "camera '" + cam->ComponentImplTypeName() + "' has no GPU counterpart";
        return false;
    }
    const Primitive* cp = nullptr;
    for (int i = 0; i < prims.NumPrimitives(); i++)
        if (prims.PrimitiveByIndex(i)->camera == cam) cp = prims.PrimitiveByIndex(i);
    const Film* film = cam->GetFilm();
    if (!cp || !film)
    {
        why = "camera without a primitive or a film";
        return false;
    }
    // The reference's own LookAt normalises with an approximate reciprocal
    // square root, so its axes are unit to about 1e-4: accept 1e-3.
    const Math::Mat4& V = cp->transform;
    double m[16], inv[16];
    for (int c = 0; c < 4; c++)
        for (int r = 0; r < 4; r++) m[4 * c + r] = double(V[c][r]);
    auto row = [&](int r, double* o) { for (int k = 0; k < 3; k++) o[k] = m[4 * k + r]; };
    double s[3], u[3], b[3];
    row(0, s);
    row(1, u);
    row(2, b);
    auto dot = [](const double* a, const double* c) { return a[0] * c[0] + a[1] * c[1] + a[2] * c[2]; };
    const double tol = 1e-3;
    if (std::fabs(dot(s, s) - 1) > tol || std::fabs(dot(u, u) - 1) > tol || std::fabs(dot(b, b) - 1) > tol ||
        std::fabs(dot(s, u)) > tol || std::fabs(dot(s, b)) > tol || std::fabs(dot(u, b)) > tol ||
        m[3] != 0 || m[7] != 0 || m[11] != 0 || m[15] != 1 || !Invert4(m, inv))
    {
        why = "camera transform is not a rigid LookAt (rows";
        for (int r = 0; r < 4; r++)
        {
            why += " [";
            for (int c = 0; c < 4; c++) why += (c ? " " : "") + std::to_string(m[4 * c + r]);
            why += "]";
        }
        why += ")";
        return false;
    }
    // Position, forward and up in world space through the inverse view
    // matrix, as the reference camera maps them (perspectivecamera.cpp:174-240).
    auto apply = [&](double x, double y, double z, double w, double* o) {
        for (int r = 0; r < 3; r++) o[r] = inv[r] * x + inv[4 + r] * y + inv[8 + r] * z + inv[12 + r] * w;
    };
    auto normalize = [&](double* a) { const double l = std::sqrt(dot(a, a)); for (int k = 0; k < 3; k++) a[k] /= l; };
    double eye[3], f[3];
    apply(0, 0, 0, 1, eye);
    apply(0, 0, -1, 0, f);
    apply(0, 1, 0, 0, u);
    normalize(f);
    normalize(u);
    const double tan10 = std::tan(10.0 * 3.14159265358979323846 / 180.0);
    Math::Vec2 raster;
    const Math::Vec3 p(static_cast<Math::Float>(eye[0]), static_cast<Math::Float>(eye[1]), static_cast<Math::Float>(eye[2]));
    // (unnormalised: only the direction's camera-space ratios matter)
    const Math::Vec3 dir(static_cast<Math::Float>(f[0] + tan10 * u[0]), static_cast<Math::Float>(f[1] + tan10 * u[1]),
                         static_cast<Math::Float>(f[2] + tan10 * u[2]));
    cam->RayToRasterPosition(p, dir, raster);
    const double y = 2.0 * double(raster.y) - 1.0;
    if (!(y > 0))
    {
        why = "cannot recover the camera's field of view";
        return false;
    }
    d.has_camera = 1;
    for (int k = 0; k < 3; k++)
    {
        d.camera_eye[k] = static_cast<float>(eye[k]);
        d.camera_center[k] = static_cast<float>(eye[k] + f[k]);
        d.camera_up[k] = static_cast<float>(u[k]);
    }
    d.camera_fovy_degrees = static_cast<float>(2.0 * std::atan(tan10 / y) * 180.0 / 3.14159265358979323846);
    d.film_width = film->Width();
    d.film_height = film->Height();
    return true;
}

}  // namespace

class GPUScene final : public Scene
{
public:

    LM_COMPONENT_IMPL_DEF("plugin.gpu");

public:

    GPUScene() {}
    virtual ~GPUScene() override
    {
        if (handle) lmgpu_scene_destroy(handle);
        if (renderHandle) lmgpu_scene_destroy(renderHandle);
    }

public:

    virtual bool Configure(const ConfigNode& node) override
    {
        std::string layoutName;
        node.ChildValueOrDefault("layout", std::string("bvh"), layoutName);
        if (layoutName == "bvh") layout = LMGPU_LAYOUT_BVH2;
        else if (layoutName == "qbvh") layout = LMGPU_LAYOUT_BVH4;
        else
        {
            LM_LOG_ERROR("Invalid value for 'layout' (expected 'bvh' or 'qbvh')");
            return false;
        }
        return true;
    }

    virtual bool Build() override
    {
        if (!primitives)
        {
            LM_LOG_ERROR("Scene has no primitives");
            return false;
        }
        std::vector<LmgpuPrimitiveDesc> descs;
        std::vector<int> meshPrimitive;
        Describe(descs, transforms, triangles, meshPrimitive);
        LmgpuSceneDesc desc = {};
        desc.primitives = descs.data();
        desc.num_primitives = static_cast<int32_t>(descs.size());
        desc.layout = layout;
        signal_ReportBuildProgress(0, false);
        if (lmgpu_scene_create(&desc, &handle) != LMGPU_OK)
        {
            LM_LOG_ERROR(std::string("GPU scene build failed: ") + lmgpu_last_error());
            handle = nullptr;
            return false;
        }
        LmgpuSceneInfo info;
        lmgpu_scene_info(handle, &info);
        aabb.min = Math::Vec3(Math::Float(info.bounds_min[0]), Math::Float(info.bounds_min[1]), Math::Float(info.bounds_min[2]));
        aabb.max = Math::Vec3(Math::Float(info.bounds_max[0]), Math::Float(info.bounds_max[1]), Math::Float(info.bounds_max[2]));
        signal_ReportBuildProgress(1, true);
        return true;
    }

    virtual bool IntersectTriangles(Ray& ray, Intersection& isect) const override
    {
        if (!handle) return false;
        const float r[8] = {
            static_cast<float>(ray.o.x), static_cast<float>(ray.o.y), static_cast<float>(ray.o.z),
            static_cast<float>(ray.d.x), static_cast<float>(ray.d.y), static_cast<float>(ray.d.z),
            static_cast<float>(ray.minT), static_cast<float>(ray.maxT) };
        int32_t id = -1;
        float t = 0, u = 0, v = 0;
        {
            std::lock_guard<std::mutex> lock(mutex);
            if (lmgpu_intersect_host(handle, r, 1, &id, &t, &u, &v) != LMGPU_OK)
            {
                LM_LOG_ERROR(std::string("GPU intersection failed: ") + lmgpu_last_error());
                return false;
            }
        }
        if (id < 0) return false;
        ray.maxT = Math::Float(t);
        const auto& tri = triangles[id];
        StoreIntersectionFromBarycentricCoords(tri.first, tri.second, ray, Math::Vec2(Math::Float(u), Math::Float(v)), isect);
        return true;
    }

    virtual AABB GetAABBTriangles() const override { return aabb; }

    virtual boost::signals2::connection Connect_ReportBuildProgress(const std::function<void(double, bool)>& func) override
    {
        return signal_ReportBuildProgress.connect(func);
    }

public:

    // The device scene for rendering: the same primitives with their BSDFs,
    // lights and camera described to the core (the helpers above), built on
    // the first call (Build() touches only the geometry, so a scene used for
    // intersections alone never evaluates its BSDFs). False, with the
    // reason, when the scene has content the core does not render.
    bool PrepareRender(std::string& why) const
    {
        std::lock_guard<std::mutex> lock(renderMutex);
        if (renderHandle) return true;
        if (!renderError.empty()) { why = renderError; return false; }
        if (!handle) { why = "scene not built"; return false; }
        LmgpuSceneDesc desc = {};
        std::vector<LmgpuAreaLightDesc> areaLights;
        std::map<const Light*, int> lightIndex;
        for (int i = 0; i < primitives->NumLights(); i++)
        {
            const Light* l = primitives->LightByIndex(i);
            const std::string type = l->ComponentImplTypeName();
            if (type != "area" && type != "env.const")
            {
                renderError = "light '" + type + "' has no GPU counterpart";
                why = renderError;
                return false;
            }
            const Math::Vec3 Le = LuminanceOf(l);
            if (type == "env.const")
            {
                desc.has_env_light = 1;
                desc.env_luminance[0] = float(Le.x); desc.env_luminance[1] = float(Le.y); desc.env_luminance[2] = float(Le.z);
            }
            else
            {
                lightIndex[l] = static_cast<int>(areaLights.size());
                areaLights.push_back(LmgpuAreaLightDesc{ { float(Le.x), float(Le.y), float(Le.z) } });
            }
        }
        std::vector<LmgpuPrimitiveDesc> descs;
        std::vector<std::vector<float>> xforms;
        std::vector<std::pair<int, int>> tris;
        std::vector<int> meshPrimitive;
        Describe(descs, xforms, tris, meshPrimitive);
        std::vector<LmgpuMaterialDesc> materials;
        std::map<const BSDF*, int> materialIndex;
        for (size_t k = 0; k < descs.size(); k++)
        {
            const Primitive* p = primitives->PrimitiveByIndex(meshPrimitive[k]);
            if (p->bsdf)
            {
                auto it = materialIndex.find(p->bsdf);
                if (it == materialIndex.end())
                {
                    LmgpuMaterialDesc md = {};
                    if (!MaterialOf(p->bsdf, md, renderError))
                    {
                        why = renderError;
                        return false;
                    }
                    it = materialIndex.emplace(p->bsdf, static_cast<int>(materials.size())).first;
                    materials.push_back(md);
                }
                descs[k].material = it->second;
            }
            if (p->light)
            {
                auto it = lightIndex.find(p->light);
                descs[k].area_light = it == lightIndex.end() ? -1 : it->second;
            }
        }
        desc.primitives = descs.data();
        desc.num_primitives = static_cast<int32_t>(descs.size());
        desc.materials = materials.data();
        desc.num_materials = static_cast<int32_t>(materials.size());
        desc.area_lights = areaLights.data();
        desc.num_area_lights = static_cast<int32_t>(areaLights.size());
        desc.layout = layout;
        if (!CameraOf(*primitives, desc, renderError))
        {
            why = renderError;
            return false;
        }
        LmgpuScene* h = nullptr;
        if (lmgpu_scene_create(&desc, &h) != LMGPU_OK)
        {
            why = std::string("GPU scene build failed: ") + lmgpu_last_error();
            return false;
        }
        renderHandle = h;
        filmWidth = desc.film_width;
        filmHeight = desc.film_height;
        return true;
    }

    LmgpuScene* RenderHandle() const { return renderHandle; }
    int FilmWidth() const { return filmWidth; }
    int FilmHeight() const { return filmHeight; }

private:

    // One descriptor per primitive that has a mesh, in primitive order (the
    // core numbers triangles primitive-major in that order, like the
    // reference's TriAccel array, scene.bvh.cpp:210-247), without materials
    // or lights; with the transforms they point to, the core triangle ->
    // (primitive, face) map and the descriptor -> primitive map.
    void Describe(std::vector<LmgpuPrimitiveDesc>& descs, std::vector<std::vector<float>>& transforms,
                  std::vector<std::pair<int, int>>& triangles, std::vector<int>& meshPrimitive) const
    {
        transforms.clear();
        triangles.clear();
        meshPrimitive.clear();
        const int n = primitives->NumPrimitives();
        transforms.reserve(n);
        for (int i = 0; i < n; i++)
        {
            const Primitive* p = primitives->PrimitiveByIndex(i);
            if (!p->mesh) continue;
            std::vector<float> m(16);
            for (int c = 0; c < 4; c++)
                for (int r = 0; r < 4; r++)
                    m[4 * c + r] = static_cast<float>(p->transform[c][r]);   // column-major, like Math::Mat4
            transforms.push_back(std::move(m));
            LmgpuPrimitiveDesc d = {};
            d.positions = p->mesh->Positions();
            d.normals = p->mesh->Normals();
            d.texcoords = p->mesh->TexCoords();
            d.faces = p->mesh->Faces();
            d.num_vertices = p->mesh->NumVertices();
            d.num_faces = p->mesh->NumFaces() / 3;      // NumFaces() counts indices
            d.transform = transforms.back().data();
            d.material = -1;
            d.area_light = -1;
            descs.push_back(d);
            meshPrimitive.push_back(i);
            for (int f = 0; f < d.num_faces; f++) triangles.emplace_back(i, f);
        }
    }

private:

    LmgpuScene* handle = nullptr;                  // geometry only: intersections
    int layout = LMGPU_LAYOUT_BVH2;
    AABB aabb;
    std::vector<std::vector<float>> transforms;
    std::vector<std::pair<int, int>> triangles;    // core triangle id -> (primitive index, face index)
    mutable LmgpuScene* renderHandle = nullptr;    // with BSDFs, lights and camera: renders
    mutable std::string renderError;
    mutable int filmWidth = 0, filmHeight = 0;
    mutable std::mutex mutex, renderMutex;
    boost::signals2::signal<void(double, bool)> signal_ReportBuildProgress;

};

// ------------------------------------------------------------ renderers ----

class GPURenderer : public Renderer
{
public:

    explicit GPURenderer(int32_t technique) : technique(technique) {}

public:

    // The reference renderers' keys (pathtrace.cpp:122-154); the sampler's
    // rng_seed seeds the core's counter-based random numbers. Absent or
    // negative (the random sampler's default is -1, randomsampler.cpp:54-60)
    // means a seed from the system, as the reference takes one from the clock.
    virtual bool Configure(const ConfigNode& node, const Assets& assets, const Scene& scene, const RenderProcessScheduler& sched) override
    {
        node.ChildValueOrDefault("rr_depth", 1, rrDepth);
        node.ChildValueOrDefault("max_path_vertices", -1, maxPathVertices);
        long long s = -1;
        const auto samplerNode = node.Child("sampler");
        if (!samplerNode.Empty()) samplerNode.ChildValueOrDefault("rng_seed", -1LL, s);
        seed = s >= 0 ? static_cast<uint64_t>(s) : static_cast<uint64_t>(std::random_device{}());
        return true;
    }

    virtual bool Preprocess(const Scene& scene, const RenderProcessScheduler& sched) override
    {
        std::string why;
        const auto* s = dynamic_cast<const GPUScene*>(&scene);
        if (!s)
        {
            LM_LOG_ERROR("Renderer '" + Type() + "' needs a 'plugin.gpu' scene");
            return false;
        }
        if (!s->PrepareRender(why))
        {
            LM_LOG_ERROR("Renderer '" + Type() + "' cannot render this scene: " + why);
            return false;
        }
        return true;
    }

    virtual bool Postprocess(const Scene& scene, const RenderProcessScheduler& sched) const override { return true; }

    virtual RenderProcess* CreateRenderProcess(const Scene& scene, int threadID, int numThreads) override;

    virtual boost::signals2::connection Connect_ReportProgress(const std::function<void(double, bool)>& func) override
    {
        return signal_ReportProgress.connect(func);
    }

public:

    // Renders samples [offset, offset + n) of the scene's camera; `rescaled`
    // receives the film rescaled by W * H / n (row y = 0 first).
    bool RenderSamples(const GPUScene& scene, long long offset, long long n, std::vector<float>& rescaled) const
    {
        LmgpuRenderParams p = {};
        p.technique = technique;
        p.rr_depth = rrDepth;
        p.max_path_vertices = maxPathVertices;
        p.sampling = LMGPU_SAMPLING_UNIFORM;        // raster positions as the reference samples them
        p.seed = seed;
        p.num_samples = n;
        p.sample_offset = offset;
        std::string why;
        if (!scene.PrepareRender(why))       // Preprocess prepares it; a caller that skipped it gets it here
        {
            LM_LOG_ERROR("Renderer '" + Type() + "' cannot render this scene: " + why);
            return false;
        }
        rescaled.assign(static_cast<size_t>(scene.FilmWidth()) * scene.FilmHeight() * 3, 0.0f);
        LmgpuRenderStats stats;
        if (lmgpu_render(scene.RenderHandle(), &p, rescaled.data(), &stats) != LMGPU_OK)
        {
            LM_LOG_ERROR(std::string("GPU render failed: ") + lmgpu_last_error());
            return false;
        }
        return true;
    }

protected:

    int32_t technique;
    int rrDepth = 1;
    int maxPathVertices = -1;
    uint64_t seed = 0;
    boost::signals2::signal<void(double, bool)> signal_ReportProgress;

};

// A render process under a per-sample scheduler: ProcessSingleSample counts,
// GetFilm renders the samples counted so far (its own range of sample
// indices) and adds their un-rescaled sum to the process's film, which the
// scheduler accumulates and rescales (sched.mt.cpp:240-250).
class GPURenderProcess final : public SamplingBasedRenderProcess
{
public:

    GPURenderProcess(const GPURenderer& renderer, const GPUScene& scene, Film* film, long long firstSample)
        : renderer(renderer), scene(scene), film(film), next(firstSample) {}

    virtual void ProcessSingleSample(const Scene&) override { pending++; }

    virtual const Film* GetFilm() const override
    {
        if (pending > 0)
        {
            std::vector<float> rescaled;
            if (!renderer.RenderSamples(scene, next, pending, rescaled))
                throw std::runtime_error("GPU render failed");
            auto* bf = dynamic_cast<BitmapFilm*>(film.get());
            auto& data = bf->Bitmap().InternalData();
            const double k = double(pending) / (double(bf->Width()) * double(bf->Height()));
            for (size_t i = 0; i < data.size() && i < rescaled.size(); i++)
                data[i] += Math::Float(double(rescaled[i]) * k);
            next += pending;
            pending = 0;
        }
        return film.get();
    }

private:

    const GPURenderer& renderer;
    const GPUScene& scene;
    std::unique_ptr<Film> film;
    mutable long long next;
    mutable long long pending = 0;

};

RenderProcess* GPURenderer::CreateRenderProcess(const Scene& scene, int threadID, int numThreads)
{
    const auto* s = dynamic_cast<const GPUScene*>(&scene);
    Film* film = scene.MainCamera() ? scene.MainCamera()->GetFilm() : nullptr;
    if (!s || !film || !dynamic_cast<BitmapFilm*>(film))
    {
        LM_LOG_ERROR("Renderer '" + Type() + "' needs a 'plugin.gpu' scene with a bitmap film");
        return nullptr;
    }
    // Each process draws its samples from its own range of indices.
    return new GPURenderProcess(*this, *s, film->Clone(), (static_cast<long long>(threadID) + 1) << 40);
}

class GPUPathtraceRenderer final : public GPURenderer
{
public:
    LM_COMPONENT_IMPL_DEF("gpu.pt");
    GPUPathtraceRenderer() : GPURenderer(LMGPU_RENDER_PT) {}
    virtual std::string Type() const override { return ImplTypeName(); }
};

class GPUDirectPathtraceRenderer final : public GPURenderer
{
public:
    LM_COMPONENT_IMPL_DEF("gpu.pt.direct");
    GPUDirectPathtraceRenderer() : GPURenderer(LMGPU_RENDER_PT_DIRECT) {}
    virtual std::string Type() const override { return ImplTypeName(); }
};

class GPUMISPathtraceRenderer final : public GPURenderer
{
public:
    LM_COMPONENT_IMPL_DEF("gpu.pt.mis");
    GPUMISPathtraceRenderer() : GPURenderer(LMGPU_RENDER_PT_MIS) {}
    virtual std::string Type() const override { return ImplTypeName(); }
};

// ------------------------------------------------------------ scheduler ----

class GPURenderProcessScheduler final : public SamplingBasedRenderProcessScheduler
{
public:

    LM_COMPONENT_IMPL_DEF("gpu");

public:

    virtual bool Configure(const ConfigNode& node, const Assets& assets) override
    {
        node.ChildValueOrDefault("num_samples", 1LL, numSamples);
        if (numSamples <= 0)
        {
            LM_LOG_ERROR("Invalid value for 'num_samples'");
            return false;
        }
        fallback.reset(ComponentFactory::Create<RenderProcessScheduler>("mt"));
        if (fallback && !fallback->Configure(node, assets)) return false;
        return true;
    }

    virtual void SetTerminationMode(TerminationMode mode, double time) override
    {
        terminationMode = mode;
        terminationTime = time;
        if (fallback) fallback->SetTerminationMode(mode, time);
    }

    virtual bool Render(Renderer& renderer, const Scene& scene) const override
    {
        auto* r = dynamic_cast<GPURenderer*>(&renderer);
        if (!r)
        {
            if (!fallback)
            {
                LM_LOG_ERROR("No 'mt' scheduler to render with renderer '" + renderer.Type() + "'");
                return false;
            }
            return fallback->Render(renderer, scene);
        }
        const auto* s = dynamic_cast<const GPUScene*>(&scene);
        std::string why;
        if (!s || !s->PrepareRender(why))
        {
            LM_LOG_ERROR("The 'gpu' scheduler needs a renderable 'plugin.gpu' scene" + (why.empty() ? std::string() : ": " + why));
            return false;
        }
        auto* film = scene.MainCamera() ? dynamic_cast<BitmapFilm*>(scene.MainCamera()->GetFilm()) : nullptr;
        if (!film)
        {
            LM_LOG_ERROR("The main camera has no bitmap film");
            return false;
        }

        // One call per num_samples batch: one in Samples mode, as many as fit
        // the time in Time mode (at least one). Un-rescaled sums accumulate
        // into the film, which is then rescaled by W * H / samples.
        signal_ReportProgress(0, false);
        const double WH = double(film->Width()) * double(film->Height());
        std::vector<double> sums(static_cast<size_t>(WH) * 3, 0.0);
        std::vector<float> rescaled;
        long long total = 0;
        const auto start = std::chrono::high_resolution_clock::now();
        for (;;)
        {
            if (!r->RenderSamples(*s, total, numSamples, rescaled)) return false;
            for (size_t i = 0; i < sums.size() && i < rescaled.size(); i++) sums[i] += double(rescaled[i]) * double(numSamples) / WH;
            total += numSamples;
            if (terminationMode != TerminationMode::Time) break;
            const double elapsed = std::chrono::duration<double>(std::chrono::high_resolution_clock::now() - start).count();
            if (elapsed >= terminationTime) break;
            signal_ReportProgress(elapsed / terminationTime, false);
        }
        auto& data = film->Bitmap().InternalData();
        const double scale = WH / double(total);
        for (size_t i = 0; i < data.size() && i < sums.size(); i++) data[i] = Math::Float((double(data[i]) + sums[i]) * scale);
        signal_ReportProgress(1, true);
        return true;
    }

    virtual long long NumSamples() const override { return numSamples; }

    virtual boost::signals2::connection Connect_ReportProgress(const std::function<void(double, bool)>& func) override
    {
        return signal_ReportProgress.connect(func);
    }

private:

    long long numSamples = 1;
    TerminationMode terminationMode = TerminationMode::Samples;
    double terminationTime = 0;
    std::unique_ptr<RenderProcessScheduler> fallback;
    boost::signals2::signal<void(double, bool)> signal_ReportProgress;

};

LM_COMPONENT_REGISTER_PLUGIN_IMPL(GPUScene, Scene);
LM_COMPONENT_REGISTER_PLUGIN_IMPL(GPUPathtraceRenderer, Renderer);
LM_COMPONENT_REGISTER_PLUGIN_IMPL(GPUDirectPathtraceRenderer, Renderer);
LM_COMPONENT_REGISTER_PLUGIN_IMPL(GPUMISPathtraceRenderer, Renderer);
LM_COMPONENT_REGISTER_PLUGIN_IMPL(GPURenderProcessScheduler, RenderProcessScheduler);

LM_NAMESPACE_END
