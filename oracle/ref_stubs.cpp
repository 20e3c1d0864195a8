// Oracle test infrastructure (not product code).
//
// Link-time stand-ins for the parts of the reference runtime that its hot-path
// sources call but that depend on libraries absent here (Boost.Regex,
// pugixml, the logger thread):
//   - Logger            (reference include/lightmetrica/logger.h:36-232): no-op sinks
//     except the last error, kept for lmref_last_error.
//   - ComponentFactory  (reference include/lightmetrica/component.h:79-136): an
//     in-process registry map; plugins are linked in, not dlopen'ed.
//   - ConfigNode        (reference include/lightmetrica/confignode.h:37-194): backed
//     by a small in-memory tree (HarnessNode) instead of pugixml.
// Everything here is written for this harness; only the declarations it
// implements come from the reference headers.
#include <dlfcn.h>
#include <vector>
#include <lightmetrica/logger.h>
#include <lightmetrica/component.h>
#include <lightmetrica/confignode.h>
#include <lightmetrica/math.types.h>
#include <lightmetrica/math.functions.h>
#include <map>
#include <sstream>
#include <string>
#include <vector>
#include "ref_tree.h"

LM_NAMESPACE_BEGIN

// ---------------------------------------------------------------- Logger ----
// Errors are kept (the last one, for lmref_last_error); other levels are dropped.
static std::string& LastError()
{
	static thread_local std::string e;
	return e;
}
void Logger::Reset() {}
void Logger::Clear() {}
void Logger::Error(const std::string& message, const std::string&) { LastError() = message; }
void Logger::Warn(const std::string&, const std::string&) {}
void Logger::Info(const std::string&, const std::string&) {}
void Logger::Debug(const std::string&, const std::string&) {}
std::string Logger::FormattedDebugInfo(const char*, int) { return std::string(); }
unsigned int Logger::Indentation() { return 0; }
void Logger::SetIndentation(unsigned int) {}

// ------------------------------------------------------ ComponentFactory ----
std::map<std::string, ComponentFactory::CreateComponentFunc>& Registry()
{
	static std::map<std::string, ComponentFactory::CreateComponentFunc> r;
	return r;
}
namespace {
std::string Key(const std::string& i, const std::string& t) { return i + "::" + t; }
}

bool ComponentFactory::CheckRegistered(const std::string& interfaceType, const std::string& implType)
{
	return Registry().count(Key(interfaceType, implType)) > 0;
}

bool ComponentFactory::Register(const std::string& interfaceType, const std::string& implType, const CreateComponentFunc& func)
{
	auto k = Key(interfaceType, implType);
	if (Registry().count(k)) return false;
	Registry()[k] = func;
	return true;
}

// Plugins loaded by lmref_load_plugin: their exported entry points
// (plugin.common.cpp:97-110), asked after the internal registry, in load
// order, like the reference's factory (component.cpp:152-166).
struct LoadedPlugin {
	void* handle;
	Component* (*create)(const char* implType, const char* interfaceType);
	bool (*check)(const char* implType, const char* interfaceType);
};
static std::vector<LoadedPlugin>& Plugins()
{
	static std::vector<LoadedPlugin> p;
	return p;
}

Component* ComponentFactory::Create(const std::string& interfaceType, const std::string& implType)
{
	auto it = Registry().find(Key(interfaceType, implType));
	if (it != Registry().end()) return it->second();
	for (auto& p : Plugins())
		if (p.check(implType.c_str(), interfaceType.c_str())) return p.create(implType.c_str(), interfaceType.c_str());
	return nullptr;
}

void ComponentFactory::LoadPlugins(const std::string&) {}
void ComponentFactory::UnloadPlugins() {}

// ------------------------------------------------------------ ConfigNode ----
// ConfigNode::Impl holds a borrowed pointer into a HarnessNode tree.
class ConfigNode::Impl
{
public:
	const lmharness::HarnessNode* node = nullptr;
	const Config* config = nullptr;
};

ConfigNode::ConfigNode() : p(new Impl) {}
ConfigNode::~ConfigNode() { delete p; }
ConfigNode::ConfigNode(void* node, const Config* config) : p(new Impl)
{
	p->node = static_cast<const lmharness::HarnessNode*>(node);
	p->config = config;
}
ConfigNode::ConfigNode(const ConfigNode& o) : p(new Impl(*o.p)) {}
void ConfigNode::operator=(const ConfigNode& o) { *p = *o.p; }
ConfigNode::ConfigNode(ConfigNode&& o) : p(new Impl(*o.p)) {}
void ConfigNode::operator=(ConfigNode&& o) { *p = *o.p; }
const Config* ConfigNode::GetConfig() const { return p->config; }
bool ConfigNode::Empty() const { return p->node == nullptr; }

ConfigNode ConfigNode::Child(const std::string& name) const
{
	if (!p->node) return ConfigNode();
	for (auto& c : p->node->children)
		if (c->name == name) return ConfigNode((void*)c.get(), p->config);
	return ConfigNode();
}

ConfigNode ConfigNode::FirstChild() const
{
	if (!p->node || p->node->children.empty()) return ConfigNode();
	return ConfigNode((void*)p->node->children.front().get(), p->config);
}

ConfigNode ConfigNode::NextChild() const
{
	if (!p->node || !p->node->parent) return ConfigNode();
	auto& sib = p->node->parent->children;
	for (size_t i = 0; i + 1 < sib.size(); i++)
		if (sib[i].get() == p->node) return ConfigNode((void*)sib[i + 1].get(), p->config);
	return ConfigNode();
}

ConfigNode ConfigNode::NextChild(const std::string& name) const
{
	if (!p->node || !p->node->parent) return ConfigNode();
	auto& sib = p->node->parent->children;
	bool after = false;
	for (auto& s : sib)
	{
		if (after && s->name == name) return ConfigNode((void*)s.get(), p->config);
		if (s.get() == p->node) after = true;
	}
	return ConfigNode();
}

std::string ConfigNode::Name() const { return p->node ? p->node->name : std::string(); }
std::string ConfigNode::Value() const { return p->node ? p->node->value : std::string(); }

std::string ConfigNode::AttributeValue(const std::string& name) const
{
	if (!p->node) return std::string();
	auto it = p->node->attributes.find(name);
	return it == p->node->attributes.end() ? std::string() : it->second;
}

namespace {
template <class T> std::vector<T> ParseList(const std::string& s)
{
	std::istringstream in(s);
	std::vector<T> r;
	T v;
	while (in >> v) r.push_back(v);
	return r;
}
}

template <> std::string ConfigNode::Value<std::string>() const { return Value(); }
template <> int ConfigNode::Value<int>() const { return std::stoi(Value()); }
template <> long long ConfigNode::Value<long long>() const { return std::stoll(Value()); }
template <> bool ConfigNode::Value<bool>() const { auto v = Value(); return v == "true" || v == "1"; }
template <> Math::Float ConfigNode::Value<Math::Float>() const
{
	auto v = ParseList<double>(Value());
	return v.empty() ? Math::Float(0) : Math::Float(v[0]);
}
template <> Math::Vec3 ConfigNode::Value<Math::Vec3>() const
{
	auto v = ParseList<double>(Value());
	if (v.size() == 1) return Math::Vec3(Math::Float(v[0]));
	if (v.size() < 3) return Math::Vec3();
	return Math::Vec3(Math::Float(v[0]), Math::Float(v[1]), Math::Float(v[2]));
}
template <> Math::Mat4 ConfigNode::Value<Math::Mat4>() const
{
	auto v = ParseList<double>(Value());
	if (v.size() != 16) return Math::Mat4::Identity();
	auto col = [&](int c) { return Math::Vec4(Math::Float(v[4 * c]), Math::Float(v[4 * c + 1]), Math::Float(v[4 * c + 2]), Math::Float(v[4 * c + 3])); };
	return Math::Mat4(col(0), col(1), col(2), col(3));
}
template <> std::vector<Math::Float> ConfigNode::Value<std::vector<Math::Float>>() const
{
	std::vector<Math::Float> r;
	for (double x : ParseList<double>(Value())) r.push_back(Math::Float(x));
	return r;
}
template <> std::vector<unsigned int> ConfigNode::Value<std::vector<unsigned int>>() const
{
	return ParseList<unsigned int>(Value());
}

LM_NAMESPACE_END

// --------------------------------------------------------------- Assets -----
// Resolves <node ref="name"/> through the concrete Assets' GetAssetByName
// (reference declaration: include/lightmetrica/assets.h:117).
#include <lightmetrica/assets.h>
#include <lightmetrica/plugin.common.h>
LM_NAMESPACE_BEGIN
Asset* Assets::ResolveReferenceToAsset(const ConfigNode& node, const std::string&) const
{
	if (node.Empty()) return nullptr;
	return GetAssetByName(node.AttributeValue("ref"));
}

// Plugins are linked into the harness, so plugin registration goes straight
// to the in-process registry (reference declaration: plugin.common.h:46).
bool PluginManager::Register(const std::string& interfaceType, const std::string& implType, const CreateComponentFunc& func)
{
	return ComponentFactory::Register(interfaceType, implType, func);
}
LM_NAMESPACE_END

// Loads a plugin the way the reference does (dlopen with RTLD_LAZY |
// RTLD_LOCAL, dynamiclibrary.cpp:78) and adds it to the factory's search.
// Returns 0, or -1 with the loader's message in *error.
extern "C" int lmref_load_plugin(const char* path, const char** error)
{
	static std::string msg;
	void* h = dlopen(path, RTLD_LAZY | RTLD_LOCAL);
	if (!h) { msg = dlerror(); if (error) *error = msg.c_str(); return -1; }
	lightmetrica::LoadedPlugin p;
	p.handle = h;
	p.create = reinterpret_cast<lightmetrica::Component* (*)(const char*, const char*)>(dlsym(h, "LM_Plugin_CreateInstance"));
	p.check = reinterpret_cast<bool (*)(const char*, const char*)>(dlsym(h, "LM_Plugin_CheckRegistered"));
	if (!p.create || !p.check) { msg = "missing plugin entry points"; if (error) *error = msg.c_str(); return -1; }
	lightmetrica::Plugins().push_back(p);
	return 0;
}

// 1 if the factory (internal registry, then loaded plugins) can create
// implType of interfaceType; the instance is created and destroyed.
extern "C" int lmref_component_available(const char* interfaceType, const char* implType)
{
	lightmetrica::Component* c = lightmetrica::ComponentFactory::Create(interfaceType, implType);
	if (!c) return 0;
	delete c;
	return 1;
}

// Diagnostics: the registered component keys ("interface::impl"), newline-separated.
extern "C" const char* lmref_registered_components()
{
	static std::string out;
	out.clear();
	for (auto& kv : lightmetrica::Registry()) out += kv.first + "\n";
	return out.c_str();
}

// The last message logged at error level by the calling thread (reference
// components and plugins report their failures this way).
extern "C" const char* lmref_last_error()
{
	return lightmetrica::LastError().c_str();
}
