// Minimal stand-in for boost::signals2 (signal/connection with connect and call).
#pragma once
#include <functional>
#include <vector>
namespace boost { namespace signals2 {
class connection { public: connection() {} void disconnect() {} bool connected() const { return false; } };
template <class Sig> class signal;
template <class R, class... A> class signal<R(A...)> {
public:
    connection connect(const std::function<R(A...)>& f) { slots_.push_back(f); return connection(); }
    void operator()(A... a) const { for (auto& s : slots_) s(a...); }
private:
    std::vector<std::function<R(A...)>> slots_;
};
}}
