// Minimal stand-in for boost::any / any_cast (copyable type-erased value).
#pragma once
#include <memory>
#include <typeinfo>
#include <stdexcept>
namespace boost {
class bad_any_cast : public std::bad_cast { public: const char* what() const noexcept override { return "bad_any_cast"; } };
class any {
    struct base { virtual ~base() {} virtual base* clone() const = 0; virtual const std::type_info& type() const = 0; };
    template <class T> struct holder : base { T v; holder(const T& x) : v(x) {} base* clone() const override { return new holder(v); } const std::type_info& type() const override { return typeid(T); } };
    std::unique_ptr<base> p_;
public:
    any() {}
    template <class T> any(const T& v) : p_(new holder<T>(v)) {}
    any(const any& o) : p_(o.p_ ? o.p_->clone() : nullptr) {}
    any& operator=(const any& o) { p_.reset(o.p_ ? o.p_->clone() : nullptr); return *this; }
    template <class T> any& operator=(const T& v) { p_.reset(new holder<T>(v)); return *this; }
    bool empty() const { return !p_; }
    const std::type_info& type() const { return p_ ? p_->type() : typeid(void); }
    template <class T> friend T any_cast(const any&);
};
template <class T> T any_cast(const any& a) {
    if (!a.p_ || a.p_->type() != typeid(T)) throw bad_any_cast();
    return static_cast<any::holder<T>*>(a.p_.get())->v;
}
}
