// Stand-in for pxr/base/tf/token.h (oracle build of the reference sources; test
// infrastructure): an interned string compared by value.
#pragma once
#include <string>

#include "pxr/pxr.h"

PXR_NAMESPACE_OPEN_SCOPE

class TfToken {
  public:
    TfToken() = default;
    explicit TfToken(std::string s) : _s(std::move(s)) {}
    const std::string &GetString() const { return _s; }
    bool operator==(const TfToken &o) const { return _s == o._s; }
    bool operator!=(const TfToken &o) const { return _s != o._s; }
    bool operator<(const TfToken &o) const { return _s < o._s; }

  private:
    std::string _s;
};

PXR_NAMESPACE_CLOSE_SCOPE
