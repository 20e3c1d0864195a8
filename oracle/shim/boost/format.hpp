// Minimal stand-in for boost::format: arguments are appended, separated by
// spaces. Only used for log messages, which the oracle harness discards.
#pragma once
#include <sstream>
#include <string>
namespace boost {
class format {
public:
    explicit format(const std::string& s) : s_(s) {}
    template <class T> format& operator%(const T& v) { std::ostringstream o; o << ' ' << v; s_ += o.str(); return *this; }
    std::string str() const { return s_; }
private:
    std::string s_;
};
inline std::string str(const format& f) { return f.str(); }
}
