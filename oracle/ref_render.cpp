// Oracle test infrastructure (not product code).
//
// Renders a scene with the reference's own renderer components, compiled
// unmodified (pathtrace.cpp, pathtrace.direct.cpp, pathtrace.mis.cpp, the
// `mt` scheduler, `hdr` film, `perspective` camera, `area` / `env.const`
// lights, `diffuse` / `mirror` / `plugin.diffusemirror` BSDFs, `bvh` scene).
// The harness only wires components together the way
// src/lightmetrica/main.cpp:255-612 and primitives.cpp:97-238 do, with an
// in-memory configuration tree instead of XML.
#include <lightmetrica/assets.h>
#include <lightmetrica/bitmap.h>
#include <lightmetrica/bitmapfilm.h>
#include <lightmetrica/bsdf.h>
#include <lightmetrica/camera.h>
#include <lightmetrica/component.h>
#include <lightmetrica/confignode.h>
#include <lightmetrica/emittershape.h>
#include <lightmetrica/film.h>
#include <lightmetrica/intersection.h>
#include <lightmetrica/light.h>
#include <lightmetrica/math.functions.h>
#include <lightmetrica/primitive.h>
#include <lightmetrica/primitives.h>
#include <lightmetrica/ray.h>
#include <lightmetrica/renderer.h>
#include <lightmetrica/sched.h>
#include <lightmetrica/scene.h>
#include <lightmetrica/trianglemesh.h>
#include <boost/any.hpp>
#include <chrono>
#include <cstdio>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <vector>
#include <omp.h>
#include "ref_tree.h"

using namespace lightmetrica;
using lmharness::HarnessNode;

extern "C" {
// Flat scene description (mirrored by ctypes in oracle/__init__.py).
struct RefRenderDesc {
    int num_prims;
    const float* const* positions;      // per primitive, 3 per vertex (world space)
    const float* const* normals;        // per primitive, 3 per vertex
    const unsigned int* const* faces;   // per primitive, 3 per triangle
    const int* num_vertices;
    const int* num_faces;
    const int* material;                // per primitive, -1 = none
    const int* light;                   // per primitive, area light index or -1
    int num_materials;
    const int* mat_type;                // 0 diffuse, 1 mirror, 2 diffuse-mirror
    const float* mat_R;                 // 3 per material
    int num_lights;
    const float* light_Le;              // 3 per area light
    int has_env;
    float env_Le[3];
    float eye[3], center[3], up[3];
    float fovy;
    int width, height;
    const char* renderer;               // "pt", "pt.direct", "pt.mis"
    int rr_depth;
    int max_path_vertices;
    int seed;
    long long num_samples;
    int num_threads;
    long long samples_per_block;
    const char* scene_type;             // accelerator ("bvh" when null), e.g. a plugin's "plugin.gpu"
    const char* sched_type;             // render process scheduler ("mt" when null), e.g. a plugin's "gpu"
};
}

namespace {

std::string fmt3(const float* v)
{
    std::ostringstream o;
    o.precision(9);
    o << v[0] << " " << v[1] << " " << v[2];
    return o.str();
}

class HarnessMesh : public TriangleMesh
{
public:
    LM_COMPONENT_IMPL_DEF("harness.mesh");
    int NumVertices() const override { return static_cast<int>(p.size() / 3); }
    int NumFaces() const override { return static_cast<int>(f.size()); }
    const Math::Float* Positions() const override { return p.data(); }
    const Math::Float* Normals() const override { return n.data(); }
    const Math::Float* TexCoords() const override { return nullptr; }
    const unsigned int* Faces() const override { return f.data(); }
    bool Load(const ConfigNode&, const Assets&) override { return true; }
    std::vector<Math::Float> p, n;
    std::vector<unsigned int> f;
};

class HarnessAssets : public Assets
{
public:
    LM_COMPONENT_IMPL_DEF("harness.assets");
    bool Load(const ConfigNode&) override { return true; }
    Asset* GetAssetByName(const std::string& name) const override
    {
        auto it = named.find(name);
        return it == named.end() ? nullptr : it->second;
    }
    boost::signals2::connection Connect_ReportProgress(const std::function<void(double, bool)>&) override
    {
        return boost::signals2::connection();
    }
    bool RegisterInterface(const std::string&, const std::string&, const std::vector<std::string>&) override { return true; }
    std::map<std::string, Asset*> named;
};

// Primitives with the wiring of PrimitivesImpl (primitives.cpp:97-238).
class HarnessPrimitives : public Primitives
{
public:
    LM_COMPONENT_IMPL_DEF("harness.primitives");
    bool Load(const ConfigNode&, const Assets&) override { return true; }
    void Reset() override {}
    int NumPrimitives() const override { return static_cast<int>(prims.size()); }
    const Primitive* PrimitiveByIndex(int i) const override { return prims[i].get(); }
    const Primitive* PrimitiveByID(const std::string&) const override { return nullptr; }
    const Camera* MainCamera() const override { return camera; }
    int NumLights() const override { return static_cast<int>(lights.size()); }
    const Light* LightByIndex(int i) const override { return lights[i]; }
    bool PostConfigure(const Scene& scene) override
    {
        if (env)
        {
            env->PostConfigure(scene);
            std::unique_ptr<EmitterShape> shape(env->CreateEmitterShape());
            if (shape) shapes.push_back(std::move(shape));
        }
        return true;
    }
    bool IntersectEmitterShapes(Ray& ray, Intersection& isect) const override
    {
        bool hit = false;
        size_t idx = 0;
        for (size_t i = 0; i < shapes.size(); i++)
        {
            Math::Float t;
            if (shapes[i]->Intersect(ray, t)) { ray.maxT = t; idx = i; hit = true; }
        }
        if (hit) shapes[idx]->StoreIntersection(ray, isect);
        return hit;
    }
    AABB GetAABBEmitterShapes() const override
    {
        AABB a;
        for (auto& s : shapes) a = a.Union(s->GetAABB());
        return a;
    }

    std::vector<std::unique_ptr<Primitive>> prims;
    std::vector<std::unique_ptr<HarnessMesh>> meshes;
    const Camera* camera = nullptr;
    std::vector<const Light*> lights;
    Light* env = nullptr;
    std::vector<std::unique_ptr<EmitterShape>> shapes;
};

// Forwards every query to the harness primitives without owning them. The
// counting scene's inner accelerator is loaded with this view, so that the
// harness primitives stay owned by the outer scene alone.
class PrimitivesView : public Primitives
{
public:
    LM_COMPONENT_IMPL_DEF("harness.primitives_view");
    explicit PrimitivesView(const Primitives* p) : p(p) {}
    bool Load(const ConfigNode&, const Assets&) override { return true; }
    bool PostConfigure(const Scene&) override { return true; }
    bool IntersectEmitterShapes(Ray& ray, Intersection& isect) const override { return p->IntersectEmitterShapes(ray, isect); }
    AABB GetAABBEmitterShapes() const override { return p->GetAABBEmitterShapes(); }
    void Reset() override {}
    int NumPrimitives() const override { return p->NumPrimitives(); }
    const Primitive* PrimitiveByIndex(int i) const override { return p->PrimitiveByIndex(i); }
    const Primitive* PrimitiveByID(const std::string& id) const override { return p->PrimitiveByID(id); }
    const Camera* MainCamera() const override { return p->MainCamera(); }
    int NumLights() const override { return p->NumLights(); }
    const Light* LightByIndex(int i) const override { return p->LightByIndex(i); }
    const Primitives* p;
};

// Scene "harness.counting": the reference's `bvh` scene with a count of the
// rays it traces. Every ray of the reference's renderers (camera, bounce and
// the shadow rays of RenderUtils::Visible) goes through Scene::Intersect,
// which calls IntersectTriangles exactly once (scene.cpp:67-72). One counter
// per OpenMP thread, each on its own cache line.
class CountingScene : public Scene
{
public:
    LM_COMPONENT_IMPL_DEF("harness.counting");
    static constexpr int MAX_THREADS = 1024;
    struct alignas(64) Counter { long long n = 0; };
    bool Configure(const ConfigNode& node) override { return inner->Configure(node); }
    bool Build() override { return inner->Build(); }
    bool IntersectTriangles(Ray& ray, Intersection& isect) const override
    {
        counts[omp_get_thread_num() & (MAX_THREADS - 1)].n++;
        return inner->IntersectTriangles(ray, isect);
    }
    AABB GetAABBTriangles() const override { return inner->GetAABBTriangles(); }
    boost::signals2::connection Connect_ReportBuildProgress(const std::function<void(double, bool)>& f) override
    {
        return inner->Connect_ReportBuildProgress(f);
    }
    long long Rays() const
    {
        long long n = 0;
        for (const auto& c : counts) n += c.n;
        return n;
    }
    void ResetCount() const
    {
        for (auto& c : counts) c.n = 0;
    }
    std::unique_ptr<Scene> inner;
    mutable Counter counts[MAX_THREADS];
};

// Everything a render needs, built once: components wired like
// main.cpp:255-612, the accelerator built, the renderer configured.
struct RefSession
{
    HarnessAssets assets;
    HarnessNode root;
    std::unique_ptr<Film> film;
    std::unique_ptr<Camera> camera;
    std::vector<std::unique_ptr<BSDF>> bsdfs;
    std::unique_ptr<BSDF> black;
    std::vector<std::unique_ptr<Light>> lights;
    std::unique_ptr<Light> env;
    std::unique_ptr<Scene> scene;
    std::unique_ptr<Renderer> renderer;
    CountingScene* counting = nullptr;
    std::string sched_type;
    long long samples_per_block = 100;
};

// Builds a session; returns 0 or the negative code lmref_render reports.
int build_session(const RefRenderDesc* d, RefSession& S, double* build_seconds)
{
    HarnessAssets& assets = S.assets;
    HarnessNode& root = S.root;

    // Film and camera
    S.film.reset(ComponentFactory::Create<Film>("hdr"));
    if (!S.film) return -1;
    {
        HarnessNode* n = root.Add("film");
        n->Add("width", std::to_string(d->width));
        n->Add("height", std::to_string(d->height));
        if (!S.film->Load(ConfigNode(n, nullptr), assets)) return -2;
    }
    assets.named["film"] = S.film.get();
    S.camera.reset(ComponentFactory::Create<Camera>("perspective"));
    {
        HarnessNode* n = root.Add("camera");
        std::ostringstream f;
        f.precision(9);
        f << d->fovy;
        n->Add("fovy", f.str());
        n->Add("film")->attributes["ref"] = "film";
        if (!S.camera->Load(ConfigNode(n, nullptr), assets)) return -3;
    }

    // BSDFs
    for (int i = 0; i < d->num_materials; i++)
    {
        const float* R = d->mat_R + 3 * i;
        if (d->mat_type[i] == 0)
        {
            S.bsdfs.emplace_back(ComponentFactory::Create<BSDF>("diffuse"));
            std::map<std::string, boost::any> params;
            params["color"] = Math::Vec3(Math::Float(R[0]), Math::Float(R[1]), Math::Float(R[2]));
            if (!S.bsdfs.back()->Load(params)) return -4;
        }
        else
        {
            const char* type = d->mat_type[i] == 1 ? "mirror" : "plugin.diffusemirror";
            S.bsdfs.emplace_back(ComponentFactory::Create<BSDF>(type));
            if (!S.bsdfs.back()) return -4;
            HarnessNode* n = root.Add("bsdf");
            n->Add(d->mat_type[i] == 1 ? "specular_reflectance" : "diffuse_reflectance", fmt3(R));
            if (!S.bsdfs.back()->Load(ConfigNode(n, nullptr), assets)) return -4;
        }
    }
    // Black diffuse for primitives without a material.
    S.black.reset(ComponentFactory::Create<BSDF>("diffuse"));
    {
        std::map<std::string, boost::any> params;
        params["color"] = Math::Vec3();
        S.black->Load(params);
    }

    // Lights
    for (int i = 0; i < d->num_lights; i++)
    {
        S.lights.emplace_back(ComponentFactory::Create<Light>("area"));
        HarnessNode* n = root.Add("light");
        n->Add("luminance", fmt3(d->light_Le + 3 * i));
        if (!S.lights.back()->Load(ConfigNode(n, nullptr), assets)) return -5;
    }
    if (d->has_env)
    {
        S.env.reset(ComponentFactory::Create<Light>("env.const"));
        HarnessNode* n = root.Add("env");
        n->Add("luminance", fmt3(d->env_Le));
        if (!S.env->Load(ConfigNode(n, nullptr), assets)) return -5;
    }

    // Primitives
    auto* P = new HarnessPrimitives;
    for (int i = 0; i < d->num_prims; i++)
    {
        std::unique_ptr<HarnessMesh> m(new HarnessMesh);
        for (int v = 0; v < 3 * d->num_vertices[i]; v++)
        {
            m->p.push_back(Math::Float(d->positions[i][v]));
            m->n.push_back(Math::Float(d->normals[i][v]));
        }
        for (int f = 0; f < 3 * d->num_faces[i]; f++) m->f.push_back(d->faces[i][f]);
        P->prims.emplace_back(new Primitive(Math::Mat4::Identity()));
        P->prims.back()->mesh = m.get();
        P->prims.back()->bsdf = d->material[i] >= 0 ? S.bsdfs[d->material[i]].get() : S.black.get();
        P->prims.back()->light = d->light[i] >= 0 ? S.lights[d->light[i]].get() : nullptr;
        P->meshes.push_back(std::move(m));
    }
    // Camera primitive: its transform is the view matrix (perspectivecamera.cpp:160-168).
    {
        auto v3 = [](const float* a) { return Math::Vec3(Math::Float(a[0]), Math::Float(a[1]), Math::Float(a[2])); };
        P->prims.emplace_back(new Primitive(Math::LookAt(v3(d->eye), v3(d->center), v3(d->up))));
        P->prims.back()->camera = S.camera.get();
        std::vector<Primitive*> refs{ P->prims.back().get() };
        S.camera->RegisterPrimitives(refs);
        P->camera = S.camera.get();
    }
    // Lights in the reference order: area lights, then the environment
    // (primitives.cpp:126-180).
    for (int li = 0; li < d->num_lights; li++)
    {
        std::vector<Primitive*> refs;
        for (auto& p : P->prims)
            if (p->light == S.lights[li].get()) refs.push_back(p.get());
        S.lights[li]->RegisterPrimitives(refs);
        P->lights.push_back(S.lights[li].get());
    }
    if (S.env)
    {
        P->lights.push_back(S.env.get());
        P->env = S.env.get();
    }

    // Scene
    const std::string scene_type = d->scene_type ? d->scene_type : "bvh";
    if (scene_type == "harness.counting")
    {
        auto* cs = new CountingScene;
        cs->inner.reset(ComponentFactory::Create<Scene>("bvh"));
        if (!cs->inner) { delete cs; delete P; return -7; }
        cs->inner->Load(new PrimitivesView(P));
        S.scene.reset(cs);
        S.counting = cs;
    }
    else
    {
        S.scene.reset(ComponentFactory::Create<Scene>(scene_type));
    }
    if (!S.scene) { delete P; return -7; }
    S.scene->Load(P);
    auto tb0 = std::chrono::high_resolution_clock::now();
    if (!S.scene->Configure(ConfigNode()) || !S.scene->Build() || !S.scene->PostConfigure()) return -6;
    auto tb1 = std::chrono::high_resolution_clock::now();
    if (build_seconds) *build_seconds = std::chrono::duration<double>(tb1 - tb0).count();

    S.sched_type = d->sched_type ? d->sched_type : "mt";
    S.samples_per_block = d->samples_per_block > 0 ? d->samples_per_block : 100;
    // The renderer is configured against a scheduler of this type (it reads
    // nothing from it, pathtrace*.cpp Configure).
    std::unique_ptr<RenderProcessScheduler> sched(ComponentFactory::Create<RenderProcessScheduler>(S.sched_type));
    if (!sched) return -7;
    S.renderer.reset(ComponentFactory::Create<Renderer>(d->renderer));
    if (!S.renderer) return -8;
    {
        HarnessNode* n = root.Add("renderer");
        n->Add("rr_depth", std::to_string(d->rr_depth));
        n->Add("max_path_vertices", std::to_string(d->max_path_vertices));
        HarnessNode* s = n->Add("sampler");
        s->attributes["type"] = "random";
        s->Add("rng", "standardmt");
        s->Add("rng_seed", std::to_string(d->seed));
        if (!S.renderer->Configure(ConfigNode(n, nullptr), assets, *S.scene, *sched)) return -8;
    }
    if (!S.renderer->Preprocess(*S.scene, *sched)) return -9;
    return 0;
}

// One RenderProcessScheduler::Render of `num_samples` samples on
// `num_threads` threads into the cleared master film; returns the seconds of
// sched.Render or a negative code.
double session_render(RefSession& S, long long num_samples, int num_threads, float* film_out, long long* rays)
{
    std::unique_ptr<RenderProcessScheduler> sched(ComponentFactory::Create<RenderProcessScheduler>(S.sched_type));
    if (!sched) return -7;
    {
        HarnessNode* n = S.root.Add("scheduler");
        n->Add("num_samples", std::to_string(num_samples));
        n->Add("num_threads", std::to_string(num_threads));
        n->Add("samples_per_block", std::to_string(S.samples_per_block));
        if (!sched->Configure(ConfigNode(n, nullptr), S.assets)) return -7;
        // The reference leaves terminationMode uninitialised (sched.mt.cpp:58)
        // and its application always sets it (main.cpp:500); so does this
        // harness, or the render loop's exit depends on heap contents.
        sched->SetTerminationMode(TerminationMode::Samples, 0);
    }
    S.film->Clear();
    if (S.counting) S.counting->ResetCount();
    auto t0 = std::chrono::high_resolution_clock::now();
    if (!sched->Render(*S.renderer, *S.scene)) return -10;
    auto t1 = std::chrono::high_resolution_clock::now();
    if (rays) *rays = S.counting ? S.counting->Rays() : -1;
    if (film_out)
    {
        auto* bf = dynamic_cast<BitmapFilm*>(S.film.get());
        const auto& data = bf->Bitmap().InternalData();
        for (size_t i = 0; i < data.size(); i++) film_out[i] = static_cast<float>(data[i]);
    }
    return std::chrono::duration<double>(t1 - t0).count();
}

}  // namespace

extern "C" {

// Renders with the reference's own components. film_out: W*H*3 floats,
// row y = 0 first (HDRBitmapFilm internal layout), rescaled as the `mt`
// scheduler leaves it. Returns the render time in seconds (sched.Render
// only), or a negative value on failure.
double lmref_render(const RefRenderDesc* d, float* film_out, double* build_seconds)
{
    RefSession S;
    const int rc = build_session(d, S, build_seconds);
    if (rc < 0) return rc;
    return session_render(S, d->num_samples, d->num_threads, film_out, nullptr);
}

// The same components built once for several renders: lmref_session_render
// renders `num_samples` samples into the cleared film (film_out may be
// NULL) and reports the rays the scene traced when the scene type is
// "harness.counting" (else -1). The renderer's sampler carries on from one
// render to the next, so successive renders draw fresh samples.
void* lmref_session_create(const RefRenderDesc* d, double* build_seconds, int* status)
{
    std::unique_ptr<RefSession> S(new RefSession);
    const int rc = build_session(d, *S, build_seconds);
    if (status) *status = rc;
    return rc < 0 ? nullptr : S.release();
}

double lmref_session_render(void* session, long long num_samples, int num_threads, float* film_out, long long* rays)
{
    if (!session) return -1;
    return session_render(*static_cast<RefSession*>(session), num_samples, num_threads, film_out, rays);
}

void lmref_session_destroy(void* session)
{
    delete static_cast<RefSession*>(session);
}

}
