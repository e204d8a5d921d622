// Stand-in for SdfAssetPath (oracle build of the reference sources; test infrastructure).
#pragma once
#include <string>

#include "pxr/pxr.h"

PXR_NAMESPACE_OPEN_SCOPE

class SdfAssetPath {
  public:
    SdfAssetPath() = default;
    explicit SdfAssetPath(std::string p) : _p(std::move(p)) {}
    const std::string &GetAssetPath() const { return _p; }
    const std::string &GetResolvedPath() const { return _p; }
    bool operator==(const SdfAssetPath &o) const { return _p == o._p; }
    bool operator!=(const SdfAssetPath &o) const { return _p != o._p; }

  private:
    std::string _p;
};

PXR_NAMESPACE_CLOSE_SCOPE
