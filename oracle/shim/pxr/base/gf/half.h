// Stand-in for pxr/base/gf/half.h (oracle build of the reference sources; test
// infrastructure): a 16-bit IEEE 754 binary16 value made from a float by
// rounding to nearest, ties to even; overflow gives infinity, NaN stays a
// (quiet) NaN. Written from the IEEE 754 definition of the format.
#pragma once
#include <cstdint>
#include <cstring>

#include "pxr/pxr.h"

PXR_NAMESPACE_OPEN_SCOPE

class GfHalf {
  public:
    GfHalf() = default;
    explicit GfHalf(float f) : _h(FromFloat(f)) {}
    uint16_t bits() const { return _h; }

  private:
    static uint16_t FromFloat(float f) {
        uint32_t x;
        std::memcpy(&x, &f, 4);
        const uint16_t sign = (uint16_t)((x >> 16) & 0x8000u);
        const uint32_t exp = (x >> 23) & 0xffu;
        uint32_t man = x & 0x7fffffu;
        if (exp == 0xffu) return (uint16_t)(sign | 0x7c00u | (man ? 0x200u | (man >> 13) : 0u));
        const int e = (int)exp - 127 + 15;  // binary16 biased exponent
        if (e >= 31) return (uint16_t)(sign | 0x7c00u);
        if (e <= 0) {  // subnormal or zero: shift the 24-bit significand right, round to nearest even
            if (e < -10) return sign;
            man |= 0x800000u;
            const int shift = 14 - e;  // 24-bit significand -> 10-bit field
            const uint32_t half_ulp = 1u << (shift - 1);
            const uint32_t rest = man & ((1u << shift) - 1u);
            uint32_t m = man >> shift;
            if (rest > half_ulp || (rest == half_ulp && (m & 1u))) ++m;
            return (uint16_t)(sign | m);
        }
        uint32_t m = man >> 13;
        const uint32_t rest = man & 0x1fffu;
        uint32_t h = ((uint32_t)e << 10) | m;
        if (rest > 0x1000u || (rest == 0x1000u && (m & 1u))) ++h;  // may carry into the exponent (to inf)
        return (uint16_t)(sign | h);
    }
    uint16_t _h = 0;
};

PXR_NAMESPACE_CLOSE_SCOPE
