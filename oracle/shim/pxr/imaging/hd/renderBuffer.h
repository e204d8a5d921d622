// Stand-in for pxr/imaging/hd/renderBuffer.h and the HdFormat helpers of
// pxr/imaging/hd/types.h (oracle build of the reference sources; test
// infrastructure), written from OpenUSD's documented interface: a format is a
// component type and a component count; HdGetComponentFormat /
// HdGetComponentCount split it, HdDataSizeOfFormat is count x component size.
#pragma once
#include <cstddef>
#include <cstdint>

#include "pxr/pxr.h"
#include "pxr/usd/sdf/path.h"

PXR_NAMESPACE_OPEN_SCOPE

// Each component type is followed by its 2-, 3- and 4-component variants.
enum HdFormat {
    HdFormatInvalid = -1,
    HdFormatUNorm8 = 0, HdFormatUNorm8Vec2, HdFormatUNorm8Vec3, HdFormatUNorm8Vec4,
    HdFormatSNorm8, HdFormatSNorm8Vec2, HdFormatSNorm8Vec3, HdFormatSNorm8Vec4,
    HdFormatFloat16, HdFormatFloat16Vec2, HdFormatFloat16Vec3, HdFormatFloat16Vec4,
    HdFormatFloat32, HdFormatFloat32Vec2, HdFormatFloat32Vec3, HdFormatFloat32Vec4,
    HdFormatInt32, HdFormatInt32Vec2, HdFormatInt32Vec3, HdFormatInt32Vec4,
    HdFormatCount
};

inline HdFormat HdGetComponentFormat(HdFormat f) {
    return (f < 0 || f >= HdFormatCount) ? HdFormatInvalid : (HdFormat)((int)f & ~3);
}
inline size_t HdGetComponentCount(HdFormat f) { return (f < 0 || f >= HdFormatCount) ? 0 : (size_t)(((int)f & 3) + 1); }
inline size_t HdDataSizeOfFormat(HdFormat f) {
    switch (HdGetComponentFormat(f)) {
        case HdFormatUNorm8:
        case HdFormatSNorm8: return HdGetComponentCount(f);
        case HdFormatFloat16: return 2 * HdGetComponentCount(f);
        case HdFormatFloat32:
        case HdFormatInt32: return 4 * HdGetComponentCount(f);
        default: return 0;
    }
}

class GfVec3i;

class HdRenderBuffer {
  public:
    explicit HdRenderBuffer(SdfPath const &id) : _id(id) {}
    virtual ~HdRenderBuffer() = default;
    virtual bool Allocate(GfVec3i const &dimensions, HdFormat format, bool multiSampled) = 0;
    virtual unsigned int GetWidth() const = 0;
    virtual unsigned int GetHeight() const = 0;
    virtual unsigned int GetDepth() const = 0;
    virtual HdFormat GetFormat() const = 0;
    virtual bool IsMultiSampled() const = 0;
    virtual void *Map() = 0;
    virtual void Unmap() = 0;
    virtual bool IsMapped() const = 0;
    virtual void Resolve() = 0;
    virtual bool IsConverged() const = 0;
    SdfPath const &GetId() const { return _id; }

  protected:
    virtual void _Deallocate() = 0;

  private:
    SdfPath _id;
};

PXR_NAMESPACE_CLOSE_SCOPE
