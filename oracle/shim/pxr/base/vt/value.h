// Stand-in for pxr/base/vt/value.h (oracle build of the reference sources; test
// infrastructure): only what frame_buffer_target.h names (an empty value that
// compares equal to another empty value).
#pragma once

#include "pxr/pxr.h"

PXR_NAMESPACE_OPEN_SCOPE

class VtValue {
  public:
    VtValue() = default;
    bool IsEmpty() const { return true; }
    bool operator==(const VtValue &) const { return true; }
};

PXR_NAMESPACE_CLOSE_SCOPE
