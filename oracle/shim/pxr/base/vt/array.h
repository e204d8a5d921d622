// Stand-in for VtArray (oracle build of the reference sources; test infrastructure).
#pragma once
#include <vector>

#include "pxr/base/gf/gf_shim.h"

PXR_NAMESPACE_OPEN_SCOPE

template <typename T> class VtArray : public std::vector<T> {
  public:
    using std::vector<T>::vector;
};
using VtVec2fArray = VtArray<GfVec2f>;
using VtVec3fArray = VtArray<GfVec3f>;
using VtVec3iArray = VtArray<GfVec3i>;
using VtMatrix4dArray = VtArray<GfMatrix4d>;
using VtIntArray = VtArray<int>;

PXR_NAMESPACE_CLOSE_SCOPE
