// Minimal stand-in for the boost::filesystem calls in the reference's
// scheduler (progress-image directory handling).
#pragma once
#include <string>
#include <sys/stat.h>
namespace boost { namespace filesystem {
class path {
public:
    path() {}
    path(const std::string& s) : s_(s) {}
    path(const char* s) : s_(s) {}
    std::string string() const { return s_; }
    bool has_extension() const { return s_.find_last_of('.') != std::string::npos && s_.find_last_of('.') > (s_.find_last_of('/') == std::string::npos ? 0 : s_.find_last_of('/')); }
    path extension() const { return has_extension() ? path(s_.substr(s_.find_last_of('.'))) : path(); }
    bool operator==(const char* o) const { return s_ == o; }
    bool operator!=(const char* o) const { return s_ != o; }
    path parent_path() const { auto k = s_.find_last_of('/'); return k == std::string::npos ? path() : path(s_.substr(0, k)); }
    bool empty() const { return s_.empty(); }
    path operator/(const std::string& o) const { return path(s_ + "/" + o); }
    path operator/(const path& o) const { return path(s_ + "/" + o.s_); }
private:
    std::string s_;
};
inline bool exists(const path& p) { struct stat st; return ::stat(p.string().c_str(), &st) == 0; }
inline bool create_directory(const path& p) { return ::mkdir(p.string().c_str(), 0755) == 0; }
}}
