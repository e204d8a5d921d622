// Stand-in for SdfPath (oracle build of the reference sources; test infrastructure).
#pragma once
#include <functional>
#include <string>

#include "pxr/pxr.h"

PXR_NAMESPACE_OPEN_SCOPE

class SdfPath {
  public:
    SdfPath() = default;
    explicit SdfPath(std::string s) : _s(std::move(s)) {}
    bool IsEmpty() const { return _s.empty(); }
    const std::string &GetString() const { return _s; }
    const char *GetText() const { return _s.c_str(); }
    bool operator==(const SdfPath &o) const { return _s == o._s; }
    bool operator!=(const SdfPath &o) const { return _s != o._s; }
    bool operator<(const SdfPath &o) const { return _s < o._s; }
    struct Hash {
        size_t operator()(const SdfPath &p) const { return std::hash<std::string>()(p._s); }
    };
    static const SdfPath &EmptyPath() {
        static SdfPath e;
        return e;
    }

  private:
    std::string _s;
};
PXR_NAMESPACE_CLOSE_SCOPE

namespace std {
template <> struct hash<pxr::SdfPath> {
    size_t operator()(const pxr::SdfPath &p) const { return pxr::SdfPath::Hash()(p); }
};
}  // namespace std
