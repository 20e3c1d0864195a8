// Oracle test infrastructure (not product code).
//
// C entry points that drive the reference's own hot-path classes, compiled
// unmodified from the reference tree by oracle/build_ref.sh into
// oracle/_ref/liblmref_{f,d}.so (float and double builds of Math::Float).
// Used only by tests/, by tests/golden/gen_golden.py and by bench.py's CPU
// baseline / reference arm.
//
// Scene set-up mirrors the reference's own test fixture
// (src/lightmetrica.test/test.scene.intersection.cpp:36-69, StubPrimitives):
// identity-transform primitives over caller-supplied triangle arrays. Each
// triangle is its own primitive so that the hit triangle index can be read
// back from Intersection::bsdf (the reference's Intersection carries no
// triangle id, include/lightmetrica/intersection.h:37-57); the BVH built over
// N one-face primitives is identical to the one over one N-face primitive
// because scene.bvh.cpp:210-247 numbers triangles primitive-major.
#include <lightmetrica/scene.h>
#include <lightmetrica/primitive.h>
#include <lightmetrica/primitives.h>
#include <lightmetrica/trianglemesh.h>
#include <lightmetrica/intersection.h>
#include <lightmetrica/ray.h>
#include <lightmetrica/aabb.h>
#include <lightmetrica/confignode.h>
#include <lightmetrica/component.h>
#include <lightmetrica/math.functions.h>
#include <chrono>
#include <cstdint>
#include <memory>
#include <random>
#include <thread>
#include <vector>
#include "ref_tree.h"

using namespace lightmetrica;

namespace {

// One-face view into shared vertex/face arrays.
class HarnessFaceMesh : public TriangleMesh
{
public:
	LM_COMPONENT_IMPL_DEF("harness.face");
	HarnessFaceMesh(const Math::Float* p, const Math::Float* n, const Math::Float* t, const unsigned int* f, int nv)
		: p_(p), n_(n), t_(t), f_(f), nv_(nv) {}
	int NumVertices() const override { return nv_; }
	int NumFaces() const override { return 3; }
	const Math::Float* Positions() const override { return p_; }
	const Math::Float* Normals() const override { return n_; }
	const Math::Float* TexCoords() const override { return t_; }
	const unsigned int* Faces() const override { return f_; }
	bool Load(const ConfigNode&, const Assets&) override { return false; }
private:
	const Math::Float* p_; const Math::Float* n_; const Math::Float* t_; const unsigned int* f_; int nv_;
};

class HarnessTrianglePrimitives : public Primitives
{
public:
	LM_COMPONENT_IMPL_DEF("harness.tris");
	bool Load(const ConfigNode&, const Assets&) override { return true; }
	void Reset() override {}
	int NumPrimitives() const override { return static_cast<int>(prims.size()); }
	const Primitive* PrimitiveByIndex(int i) const override { return prims[i].get(); }
	const Primitive* PrimitiveByID(const std::string&) const override { return nullptr; }
	const Camera* MainCamera() const override { return nullptr; }
	int NumLights() const override { return 0; }
	const Light* LightByIndex(int) const override { return nullptr; }
	bool PostConfigure(const Scene&) override { return true; }
	bool IntersectEmitterShapes(Ray&, Intersection&) const override { return false; }
	AABB GetAABBEmitterShapes() const override { return AABB(); }

	std::vector<Math::Float> positions, normals, texcoords;
	std::vector<unsigned int> faces;
	std::vector<std::unique_ptr<HarnessFaceMesh>> meshes;
	std::vector<std::unique_ptr<Primitive>> prims;
};

struct HarnessScene
{
	std::unique_ptr<Scene> scene;
	HarnessTrianglePrimitives* prims = nullptr;
};

}

extern "C" {

// Builds a reference scene ("bvh", "qbvh" or "naive") over world-space
// triangles. normals/texcoords may be null (normals then default to +z,
// texcoords to (0,0),(1,0),(0,1) per face corner so that the hit's uv equals
// the reference's barycentric pair b). Returns null on failure.
void* lmref_scene_create(const char* type, const float* positions, int num_vertices,
                         const float* normals, const float* texcoords,
                         const unsigned int* faces, int num_tris, double* build_seconds)
{
	auto* h = new HarnessScene;
	h->scene.reset(ComponentFactory::Create<Scene>(type));
	if (!h->scene) { delete h; return nullptr; }
	auto* P = new HarnessTrianglePrimitives;
	h->prims = P;

	P->positions.assign(positions, positions + 3 * (size_t)num_vertices);
	if (normals) P->normals.assign(normals, normals + 3 * (size_t)num_vertices);
	else for (int i = 0; i < num_vertices; i++) { P->normals.push_back(0); P->normals.push_back(0); P->normals.push_back(1); }

	// texcoords: either per vertex (caller) or per face corner (default).
	// The default needs distinct vertices per face corner, so faces are
	// re-indexed into a corner-expanded copy of the vertex arrays.
	if (texcoords)
	{
		P->texcoords.assign(texcoords, texcoords + 2 * (size_t)num_vertices);
		P->faces.assign(faces, faces + 3 * (size_t)num_tris);
	}
	else
	{
		std::vector<Math::Float> pos, nrm;
		static const Math::Float corner[3][2] = { {0, 0}, {1, 0}, {0, 1} };
		for (int f = 0; f < num_tris; f++)
			for (int c = 0; c < 3; c++)
			{
				unsigned int v = faces[3 * f + c];
				for (int k = 0; k < 3; k++) { pos.push_back(P->positions[3 * v + k]); nrm.push_back(P->normals[3 * v + k]); }
				P->texcoords.push_back(corner[c][0]);
				P->texcoords.push_back(corner[c][1]);
				P->faces.push_back(3 * f + c);
			}
		P->positions.swap(pos);
		P->normals.swap(nrm);
	}

	const int nv = static_cast<int>(P->positions.size() / 3);
	for (int f = 0; f < num_tris; f++)
	{
		P->meshes.emplace_back(new HarnessFaceMesh(P->positions.data(), P->normals.data(), P->texcoords.data(), &P->faces[3 * (size_t)f], nv));
		P->prims.emplace_back(new Primitive(Math::Mat4::Identity()));
		P->prims.back()->mesh = P->meshes.back().get();
		// Tag (never dereferenced by Intersect): triangle index + 1.
		P->prims.back()->bsdf = reinterpret_cast<BSDF*>(static_cast<uintptr_t>(f) + 1);
	}

	h->scene->Load(P);
	auto t0 = std::chrono::high_resolution_clock::now();
	bool ok = h->scene->Configure(ConfigNode()) && h->scene->Build();
	auto t1 = std::chrono::high_resolution_clock::now();
	if (build_seconds) *build_seconds = std::chrono::duration<double>(t1 - t0).count();
	if (!ok) { delete h; return nullptr; }
	return h;
}

void lmref_scene_destroy(void* p) { delete static_cast<HarnessScene*>(p); }

// Intersects n rays (AoS, 8 floats each: o.xyz, d.xyz, minT, maxT) with the
// scene through Scene::Intersect. tri_id[i] = hit triangle or -1; t_out[i]
// = the ray's maxT after the query (the hit distance); geom_out (optional,
// 17 floats per ray) = p, gn, sn, ss, st, uv. Returns the number of hits.
long long lmref_intersect(void* p, long long n, const float* rays, int* tri_id, float* t_out,
                          float* geom_out, int num_threads)
{
	auto* h = static_cast<HarnessScene*>(p);
	if (num_threads < 1) num_threads = 1;
	std::vector<long long> hits(num_threads, 0);
	auto work = [&](int tid)
	{
		long long b = n * tid / num_threads, e = n * (tid + 1) / num_threads;
		for (long long i = b; i < e; i++)
		{
			const float* r = rays + 8 * i;
			Ray ray;
			ray.o = Math::Vec3(Math::Float(r[0]), Math::Float(r[1]), Math::Float(r[2]));
			ray.d = Math::Vec3(Math::Float(r[3]), Math::Float(r[4]), Math::Float(r[5]));
			ray.minT = Math::Float(r[6]);
			ray.maxT = Math::Float(r[7]);
			Intersection isect;
			bool hit = h->scene->Intersect(ray, isect);
			tri_id[i] = hit ? static_cast<int>(reinterpret_cast<uintptr_t>(isect.bsdf) - 1) : -1;
			if (t_out) t_out[i] = hit ? static_cast<float>(ray.maxT) : 0.f;
			if (hit) hits[tid]++;
			if (geom_out)
			{
				float* g = geom_out + 17 * i;
				const auto& G = isect.geom;
				const Math::Vec3* vs[5] = { &G.p, &G.gn, &G.sn, &G.ss, &G.st };
				for (int k = 0; k < 5; k++)
					for (int c = 0; c < 3; c++) g[3 * k + c] = hit ? static_cast<float>((*vs[k])[c]) : 0.f;
				g[15] = hit ? static_cast<float>(G.uv.x) : 0.f;
				g[16] = hit ? static_cast<float>(G.uv.y) : 0.f;
			}
		}
	};
	std::vector<std::thread> ts;
	for (int t = 1; t < num_threads; t++) ts.emplace_back(work, t);
	work(0);
	for (auto& t : ts) t.join();
	long long total = 0;
	for (auto c : hits) total += c;
	return total;
}

int lmref_float_bytes() { return static_cast<int>(sizeof(Math::Float)); }

}

extern "C" {

// Regenerates the reference's StubTriangleMesh_Random vertex data
// (include/lightmetrica.test/stub.trianglemesh.h:184-225): 1000 triangles in
// [0,1]^3 from std::mt19937(42) and std::uniform_real_distribution<double>,
// converted to Math::Float, with the unnormalised face normal per corner.
// positions/normals: 9000 floats each.
void lmref_stub_random_mesh(float* positions, float* normals)
{
	std::mt19937 gen(42);
	std::uniform_real_distribution<double> dist;
	for (int i = 0; i < 1000; i++)
	{
		Math::Vec3 p[3];
		for (int c = 0; c < 3; c++)
		{
			Math::Float x = Math::Float(dist(gen));
			Math::Float y = Math::Float(dist(gen));
			Math::Float z = Math::Float(dist(gen));
			p[c] = Math::Vec3(x, y, z);
		}
		auto n = Math::Cross(p[1] - p[0], p[2] - p[0]);
		for (int c = 0; c < 3; c++)
			for (int k = 0; k < 3; k++)
			{
				positions[9 * i + 3 * c + k] = static_cast<float>(p[c][k]);
				normals[9 * i + 3 * c + k] = static_cast<float>(n[k]);
			}
	}
}

}
