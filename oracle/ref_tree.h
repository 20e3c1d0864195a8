// Oracle test infrastructure (not product code).
// In-memory configuration tree that backs the harness's ConfigNode stand-in.
#pragma once
#include <map>
#include <memory>
#include <string>
#include <vector>

namespace lmharness {

struct HarnessNode
{
	std::string name;
	std::string value;
	std::map<std::string, std::string> attributes;
	std::vector<std::unique_ptr<HarnessNode>> children;
	HarnessNode* parent = nullptr;

	HarnessNode* Add(const std::string& n, const std::string& v = std::string())
	{
		children.emplace_back(new HarnessNode);
		auto* c = children.back().get();
		c->name = n;
		c->value = v;
		c->parent = this;
		return c;
	}
};

}
