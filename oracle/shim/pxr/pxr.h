// Stand-in for pxr/pxr.h (oracle build of the reference sources; test infrastructure).
#pragma once
namespace pxr {}
#define PXR_NS pxr
#define PXR_NAMESPACE_OPEN_SCOPE namespace pxr {
#define PXR_NAMESPACE_CLOSE_SCOPE }
#define PXR_NAMESPACE_USING_DIRECTIVE using namespace pxr;
