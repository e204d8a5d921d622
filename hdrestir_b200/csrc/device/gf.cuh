// Vector arithmetic with the exact rounding behaviour the reference gets from
// OpenUSD Gf (GfVec3f / GfVec2f / GfMatrix4d) and libstdc++ on x86-64:
//  * component arithmetic, dot and cross products are float operations in
//    source order; the build passes -fmad=false so nothing is contracted;
//  * GfVec3f::operator*=(double s) evaluates each component as
//    float(double(x) * s), and operator/(double s) multiplies by the double
//    reciprocal 1.0/s (so a division by a float length is NOT a float divide);
//  * GetNormalized() divides by max(length, 1e-10f) through that double path;
//  * std::max / std::min / std::clamp are the ternaries of the standard, which
//    differ from fmaxf/fminf on NaN and signed zero.
// Every helper is __host__ __device__ so host-side scene preparation and the
// kernels round identically.
#pragma once

#include <math.h>
#include <stdint.h>

#if defined(__CUDACC__)
#define HDR_HD __host__ __device__ __forceinline__
#else
#define HDR_HD inline
#endif

namespace hdr {

// (float)M_PI: the reference's shading code casts the <cmath> double constant
constexpr float kPiF = 3.14159265358979323846f;

struct V3 {
    float x, y, z;
};
struct V2 {
    float x, y;
};
struct D3 {
    double x, y, z;
};

HDR_HD float smaxf(float a, float b) { return (a < b) ? b : a; }   // std::max
HDR_HD float sminf(float a, float b) { return (b < a) ? b : a; }   // std::min
HDR_HD int smaxi(int a, int b) { return (a < b) ? b : a; }
HDR_HD int smini(int a, int b) { return (b < a) ? b : a; }
HDR_HD float sclampf(float v, float lo, float hi) { return (v < lo) ? lo : ((hi < v) ? hi : v); }
HDR_HD int sclampi(int v, int lo, int hi) { return (v < lo) ? lo : ((hi < v) ? hi : v); }

HDR_HD V3 v3(float x, float y, float z) { return V3{x, y, z}; }
HDR_HD V3 v3s(float s) { return V3{s, s, s}; }
HDR_HD V3 operator+(V3 a, V3 b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; }
HDR_HD V3 operator-(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
HDR_HD V3 operator-(V3 a) { return V3{-a.x, -a.y, -a.z}; }
// GfVec3f * float / float * GfVec3f: Gf promotes the scalar to double, but the
// product of two floats is exact in double, so the single rounding to float is
// the IEEE float product.
HDR_HD V3 operator*(V3 a, float s) { return V3{a.x * s, a.y * s, a.z * s}; }
HDR_HD V3 operator*(float s, V3 a) { return V3{a.x * s, a.y * s, a.z * s}; }
// GfCompMult
HDR_HD V3 cmul(V3 a, V3 b) { return V3{a.x * b.x, a.y * b.y, a.z * b.z}; }
// GfVec3f *= double
HDR_HD V3 mul_d(V3 a, double s) {
    return V3{(float)((double)a.x * s), (float)((double)a.y * s), (float)((double)a.z * s)};
}
// GfVec3f / double  (== *this * (1.0 / s))
HDR_HD V3 div_d(V3 a, double s) { return mul_d(a, 1.0 / s); }
HDR_HD float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
HDR_HD V3 cross(V3 a, V3 b) {
    return V3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
HDR_HD float length_sq(V3 a) { return dot(a, a); }
#if defined(__CUDA_ARCH__)
HDR_HD float hdr_sqrtf(float x) { return __fsqrt_rn(x); }
#else
HDR_HD float hdr_sqrtf(float x) { return __builtin_sqrtf(x); }
#endif
HDR_HD float length(V3 a) { return hdr_sqrtf(dot(a, a)); }
// GfVec3f::GetNormalized(eps = GF_MIN_VECTOR_LENGTH = 1e-10)
HDR_HD V3 normalized(V3 a) {
    const float len = length(a);
    return div_d(a, (double)((len > 1e-10f) ? len : 1e-10f));
}
HDR_HD float comp(V3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }

HDR_HD V2 operator+(V2 a, V2 b) { return V2{a.x + b.x, a.y + b.y}; }
HDR_HD V2 operator*(V2 a, float s) { return V2{a.x * s, a.y * s}; }

// GfMatrix4f::Transform (row vector, w = 1, then GfProject).
HDR_HD V3 m4f_transform(const float *m, V3 v) {
    const float x = v.x * m[0] + v.y * m[4] + v.z * m[8] + m[12];
    const float y = v.x * m[1] + v.y * m[5] + v.z * m[9] + m[13];
    const float z = v.x * m[2] + v.y * m[6] + v.z * m[10] + m[14];
    const float w = v.x * m[3] + v.y * m[7] + v.z * m[11] + m[15];
    const float inv = (w != 0.0f) ? 1.0f / w : 1.0f;
    return V3{inv * x, inv * y, inv * z};
}
// GfMatrix4f::TransformDir (upper 3x3, row vector).
HDR_HD V3 m4f_transform_dir(const float *m, V3 v) {
    return V3{v.x * m[0] + v.y * m[4] + v.z * m[8], v.x * m[1] + v.y * m[5] + v.z * m[9],
              v.x * m[2] + v.y * m[6] + v.z * m[10]};
}
// GfMatrix4d::Transform on GfVec3d (w = 1, GfProject in double).
HDR_HD D3 m4d_transform(const double *m, D3 v) {
    const double x = v.x * m[0] + v.y * m[4] + v.z * m[8] + m[12];
    const double y = v.x * m[1] + v.y * m[5] + v.z * m[9] + m[13];
    const double z = v.x * m[2] + v.y * m[6] + v.z * m[10] + m[14];
    const double w = v.x * m[3] + v.y * m[7] + v.z * m[11] + m[15];
    const double inv = (w != 0.0) ? 1.0 / w : 1.0;
    return D3{inv * x, inv * y, inv * z};
}
HDR_HD V3 d3_to_f(D3 a) { return V3{(float)a.x, (float)a.y, (float)a.z}; }
HDR_HD D3 f3_to_d(V3 a) { return D3{(double)a.x, (double)a.y, (double)a.z}; }

// Inverse of a 4x4 (row-major) by cofactor expansion in double; singular
// matrices yield a scale of FLT_MAX like GfMatrix4d::GetInverse. Shared by the
// host scene builder and the device instance update, so both give the same bits.
HDR_HD void gf_inverse4d(const double *m, double *out) {
    const double s0 = m[0] * m[5] - m[4] * m[1];
    const double s1 = m[0] * m[6] - m[4] * m[2];
    const double s2 = m[0] * m[7] - m[4] * m[3];
    const double s3 = m[1] * m[6] - m[5] * m[2];
    const double s4 = m[1] * m[7] - m[5] * m[3];
    const double s5 = m[2] * m[7] - m[6] * m[3];
    const double c5 = m[10] * m[15] - m[14] * m[11];
    const double c4 = m[9] * m[15] - m[13] * m[11];
    const double c3 = m[9] * m[14] - m[13] * m[10];
    const double c2 = m[8] * m[15] - m[12] * m[11];
    const double c1 = m[8] * m[14] - m[12] * m[10];
    const double c0 = m[8] * m[13] - m[12] * m[9];
    const double det = s0 * c5 - s1 * c4 + s2 * c3 + s3 * c2 - s4 * c1 + s5 * c0;
    if (!(fabs(det) > 0.0)) {
        for (int i = 0; i < 16; ++i) out[i] = 0.0;
        out[0] = out[5] = out[10] = 3.402823466e+38;
        out[15] = 1.0;
        return;
    }
    const double r = 1.0 / det;
    out[0] = (m[5] * c5 - m[6] * c4 + m[7] * c3) * r;
    out[1] = (-m[1] * c5 + m[2] * c4 - m[3] * c3) * r;
    out[2] = (m[13] * s5 - m[14] * s4 + m[15] * s3) * r;
    out[3] = (-m[9] * s5 + m[10] * s4 - m[11] * s3) * r;
    out[4] = (-m[4] * c5 + m[6] * c2 - m[7] * c1) * r;
    out[5] = (m[0] * c5 - m[2] * c2 + m[3] * c1) * r;
    out[6] = (-m[12] * s5 + m[14] * s2 - m[15] * s1) * r;
    out[7] = (m[8] * s5 - m[10] * s2 + m[11] * s1) * r;
    out[8] = (m[4] * c4 - m[5] * c2 + m[7] * c0) * r;
    out[9] = (-m[0] * c4 + m[1] * c2 - m[3] * c0) * r;
    out[10] = (m[12] * s4 - m[13] * s2 + m[15] * s0) * r;
    out[11] = (-m[8] * s4 + m[9] * s2 - m[11] * s0) * r;
    out[12] = (-m[4] * c3 + m[5] * c1 - m[6] * c0) * r;
    out[13] = (m[0] * c3 - m[1] * c1 + m[2] * c0) * r;
    out[14] = (-m[12] * s3 + m[13] * s1 - m[14] * s0) * r;
    out[15] = (m[8] * s3 - m[9] * s1 + m[10] * s0) * r;
}

HDR_HD void gf_inverse4f(const float *m, float *out) {
    double md[16], od[16];
    for (int i = 0; i < 16; ++i) md[i] = (double)m[i];
    gf_inverse4d(md, od);
    for (int i = 0; i < 16; ++i) out[i] = (float)od[i];
}

}  // namespace hdr
