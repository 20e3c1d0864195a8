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
    path operator/(const std::string& o) const { return path(s_ + "/" + o); }
    path operator/(const path& o) const { return path(s_ + "/" + o.s_); }
private:
    std::string s_;
};
inline bool exists(const path& p) { struct stat st; return ::stat(p.string().c_str(), &st) == 0; }
inline bool create_directory(const path& p) { return ::mkdir(p.string().c_str(), 0755) == 0; }
}}
