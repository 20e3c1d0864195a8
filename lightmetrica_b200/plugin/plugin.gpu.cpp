// plugin.gpu.so — lightmetrica's Scene slot ("plugin.gpu") on the B200 core.
//
// A lightmetrica plugin in the reference's plugin ABI (plugin.common.h:82-103,
// plugin.common.cpp:97-110; the same slot plugin/plugin.embree fills): build
// it against lightmetrica's headers with LM_USE_SINGLE_PRECISION together
// with lightmetrica's plugin.common.cpp, link it to liblmgpu.so, and put it
// where ComponentFactory::LoadPlugins finds it (component.cpp:61-120). A scene
// document then selects it with <scene type="plugin.gpu">.
//
// Build() hands the primitives' meshes and transforms to lmgpu_scene_create,
// which builds the reference's binary SAH BVH on the host and uploads it;
// IntersectTriangles() answers one ray through lmgpu_intersect_host with the
// reference's closest hit bit for bit (same triangle, t and barycentrics), and
// fills the Intersection with the reference's own
// StoreIntersectionFromBarycentricCoords, exactly as BVHScene does
// (scene.bvh.cpp:390-403). The reference's renderers call IntersectTriangles
// from every OpenMP thread; the calls share the scene's staging buffers and
// take turns on a mutex. Whole renders and ray batches go through the C ABI
// (lmgpu_render, lmgpu_intersect) instead, one call per batch.
//
// Configuration: <layout>bvh</layout> (default; bit-exact) or qbvh (4-wide
// collapse of the same tree, also bit-exact).
#include <lightmetrica/scene.h>
#include <lightmetrica/primitive.h>
#include <lightmetrica/primitives.h>
#include <lightmetrica/trianglemesh.h>
#include <lightmetrica/confignode.h>
#include <lightmetrica/intersection.h>
#include <lightmetrica/ray.h>
#include <lightmetrica/logger.h>
#include <lightmetrica/plugin.common.h>

#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "lmgpu.h"

LM_NAMESPACE_BEGIN

class GPUScene final : public Scene
{
public:

    LM_COMPONENT_IMPL_DEF("plugin.gpu");

public:

    GPUScene() {}
    virtual ~GPUScene() override { if (handle) lmgpu_scene_destroy(handle); }

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

        // One descriptor per primitive that has a mesh, in primitive order:
        // the core numbers triangles primitive-major in that order, like the
        // reference's TriAccel array (scene.bvh.cpp:210-247).
        std::vector<LmgpuPrimitiveDesc> descs;
        transforms.clear();
        triangles.clear();
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
            for (int f = 0; f < d.num_faces; f++) triangles.emplace_back(i, f);
        }

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

private:

    LmgpuScene* handle = nullptr;
    int layout = LMGPU_LAYOUT_BVH2;
    AABB aabb;
    std::vector<std::vector<float>> transforms;
    std::vector<std::pair<int, int>> triangles;    // core triangle id -> (primitive index, face index)
    mutable std::mutex mutex;
    boost::signals2::signal<void(double, bool)> signal_ReportBuildProgress;

};

LM_COMPONENT_REGISTER_PLUGIN_IMPL(GPUScene, Scene);

LM_NAMESPACE_END
