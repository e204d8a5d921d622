// Minimal stand-in for the OpenUSD Gf types the reference's hot-path sources
// use, so those sources compile in place for the oracle build (TEST
// INFRASTRUCTURE; not part of the product). Written from OpenUSD's documented
// semantics:
//  * GfVecNf arithmetic is float in source order; scalar multiply/divide take a
//    double (operator*=(double), operator/=(double) == *= (1.0 / s));
//  * GetNormalized/Normalize divide by max(length, eps = 1e-10);
//  * GfMatrix4{f,d} use the row-vector convention (translation in row 3),
//    Transform() projects through w, TransformDir() uses the upper 3x3;
//  * GetInverse() is a cofactor expansion in double (FLT_MAX scale when singular).
// OpenUSD itself is not available, so results are pinned to these semantics.
#pragma once

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstddef>
#include <cstring>

#include "pxr/pxr.h"

PXR_NAMESPACE_OPEN_SCOPE

class GfVec3d;
class GfVec4d;
class GfMatrix4d;

template <typename T, int N, typename Derived> struct GfVecBase {
    T _data[N];
    T &operator[](size_t i) { return _data[i]; }
    const T &operator[](size_t i) const { return _data[i]; }
    T *data() { return _data; }
    const T *data() const { return _data; }
    Derived &self() { return static_cast<Derived &>(*this); }
    const Derived &self() const { return static_cast<const Derived &>(*this); }
    bool operator==(const Derived &o) const {
        for (int i = 0; i < N; ++i)
            if (!(_data[i] == o._data[i])) return false;
        return true;
    }
    bool operator!=(const Derived &o) const { return !(*this == o); }
    Derived operator-() const {
        Derived r;
        for (int i = 0; i < N; ++i) r._data[i] = -_data[i];
        return r;
    }
    Derived &operator+=(const Derived &o) {
        for (int i = 0; i < N; ++i) _data[i] += o._data[i];
        return self();
    }
    Derived &operator-=(const Derived &o) {
        for (int i = 0; i < N; ++i) _data[i] -= o._data[i];
        return self();
    }
    Derived &operator*=(double s) {
        for (int i = 0; i < N; ++i) _data[i] *= s;
        return self();
    }
    Derived &operator/=(double s) { return *this *= (1.0 / s); }
    friend Derived operator+(const Derived &a, const Derived &b) { return Derived(a) += b; }
    friend Derived operator-(const Derived &a, const Derived &b) { return Derived(a) -= b; }
    friend Derived operator*(const Derived &a, double s) { return Derived(a) *= s; }
    friend Derived operator*(double s, const Derived &a) { return Derived(a) *= s; }
    friend Derived operator/(const Derived &a, double s) { return a * (1.0 / s); }
    // dot product, as Gf defines operator* between vectors
    friend T operator*(const Derived &a, const Derived &b) {
        T r = a._data[0] * b._data[0];
        for (int i = 1; i < N; ++i) r = r + a._data[i] * b._data[i];
        return r;
    }
    T GetLengthSq() const { return self() * self(); }
    T GetLength() const { return std::sqrt(GetLengthSq()); }
    T Normalize(T eps = (T)1e-10) {
        T len = GetLength();
        *this /= (len > eps) ? len : eps;
        return len;
    }
    Derived GetNormalized(T eps = (T)1e-10) const {
        Derived r(self());
        r.Normalize(eps);
        return r;
    }
};

class GfVec2f : public GfVecBase<float, 2, GfVec2f> {
  public:
    GfVec2f() { _data[0] = _data[1] = 0.0f; }
    explicit GfVec2f(float v) { _data[0] = _data[1] = v; }
    GfVec2f(float x, float y) { _data[0] = x, _data[1] = y; }
};

class GfVec2i : public GfVecBase<int, 2, GfVec2i> {
  public:
    GfVec2i() { _data[0] = _data[1] = 0; }
    explicit GfVec2i(int v) { _data[0] = _data[1] = v; }
    GfVec2i(int x, int y) { _data[0] = x, _data[1] = y; }
};

class GfVec3i : public GfVecBase<int, 3, GfVec3i> {
  public:
    GfVec3i() { _data[0] = _data[1] = _data[2] = 0; }
    explicit GfVec3i(int v) { _data[0] = _data[1] = _data[2] = v; }
    GfVec3i(int x, int y, int z) { _data[0] = x, _data[1] = y, _data[2] = z; }
};

class GfVec3f : public GfVecBase<float, 3, GfVec3f> {
  public:
    GfVec3f() { _data[0] = _data[1] = _data[2] = 0.0f; }
    explicit GfVec3f(float v) { _data[0] = _data[1] = _data[2] = v; }
    GfVec3f(float x, float y, float z) { _data[0] = x, _data[1] = y, _data[2] = z; }
    explicit GfVec3f(const GfVec3d &o);
};

class GfVec3d : public GfVecBase<double, 3, GfVec3d> {
  public:
    GfVec3d() { _data[0] = _data[1] = _data[2] = 0.0; }
    explicit GfVec3d(double v) { _data[0] = _data[1] = _data[2] = v; }
    GfVec3d(double x, double y, double z) { _data[0] = x, _data[1] = y, _data[2] = z; }
    GfVec3d(const GfVec3f &o) { _data[0] = o[0], _data[1] = o[1], _data[2] = o[2]; }
};
inline GfVec3f::GfVec3f(const GfVec3d &o) {
    _data[0] = (float)o[0];
    _data[1] = (float)o[1];
    _data[2] = (float)o[2];
}

class GfVec4f : public GfVecBase<float, 4, GfVec4f> {
  public:
    GfVec4f() { _data[0] = _data[1] = _data[2] = _data[3] = 0.0f; }
    explicit GfVec4f(float v) { _data[0] = _data[1] = _data[2] = _data[3] = v; }
    GfVec4f(float x, float y, float z, float w) { _data[0] = x, _data[1] = y, _data[2] = z, _data[3] = w; }
};

class GfVec4d : public GfVecBase<double, 4, GfVec4d> {
  public:
    GfVec4d() { _data[0] = _data[1] = _data[2] = _data[3] = 0.0; }
    GfVec4d(double x, double y, double z, double w) { _data[0] = x, _data[1] = y, _data[2] = z, _data[3] = w; }
};

inline float GfDot(const GfVec3f &a, const GfVec3f &b) { return a * b; }
inline double GfDot(const GfVec3d &a, const GfVec3d &b) { return a * b; }
inline float GfDot(const GfVec2f &a, const GfVec2f &b) { return a * b; }
inline float GfDot(const GfVec4f &a, const GfVec4f &b) { return a * b; }
inline GfVec3f GfCross(const GfVec3f &a, const GfVec3f &b) {
    return GfVec3f(a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]);
}
inline GfVec3d GfCross(const GfVec3d &a, const GfVec3d &b) {
    return GfVec3d(a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]);
}
inline GfVec3f GfCompMult(const GfVec3f &a, const GfVec3f &b) { return GfVec3f(a[0] * b[0], a[1] * b[1], a[2] * b[2]); }
inline GfVec3f GfCompDiv(const GfVec3f &a, const GfVec3f &b) { return GfVec3f(a[0] / b[0], a[1] / b[1], a[2] / b[2]); }
inline GfVec3f GfProject(const GfVec4f &v) {
    float inv = (v[3] != 0.0f) ? 1.0f / v[3] : 1.0f;
    return GfVec3f(inv * v[0], inv * v[1], inv * v[2]);
}
inline GfVec3d GfProject(const GfVec4d &v) {
    double inv = (v[3] != 0.0) ? 1.0 / v[3] : 1.0;
    return GfVec3d(inv * v[0], inv * v[1], inv * v[2]);
}

namespace gf_shim_detail {
inline void inverse4(const double *m, double *o) {
    double s0 = m[0] * m[5] - m[4] * m[1], s1 = m[0] * m[6] - m[4] * m[2], s2 = m[0] * m[7] - m[4] * m[3];
    double s3 = m[1] * m[6] - m[5] * m[2], s4 = m[1] * m[7] - m[5] * m[3], s5 = m[2] * m[7] - m[6] * m[3];
    double c5 = m[10] * m[15] - m[14] * m[11], c4 = m[9] * m[15] - m[13] * m[11], c3 = m[9] * m[14] - m[13] * m[10];
    double c2 = m[8] * m[15] - m[12] * m[11], c1 = m[8] * m[14] - m[12] * m[10], c0 = m[8] * m[13] - m[12] * m[9];
    double det = s0 * c5 - s1 * c4 + s2 * c3 + s3 * c2 - s4 * c1 + s5 * c0;
    if (!(std::fabs(det) > 0.0)) {
        for (int i = 0; i < 16; ++i) o[i] = 0.0;
        o[0] = o[5] = o[10] = FLT_MAX;
        o[15] = 1.0;
        return;
    }
    double r = 1.0 / det;
    o[0] = (m[5] * c5 - m[6] * c4 + m[7] * c3) * r;
    o[1] = (-m[1] * c5 + m[2] * c4 - m[3] * c3) * r;
    o[2] = (m[13] * s5 - m[14] * s4 + m[15] * s3) * r;
    o[3] = (-m[9] * s5 + m[10] * s4 - m[11] * s3) * r;
    o[4] = (-m[4] * c5 + m[6] * c2 - m[7] * c1) * r;
    o[5] = (m[0] * c5 - m[2] * c2 + m[3] * c1) * r;
    o[6] = (-m[12] * s5 + m[14] * s2 - m[15] * s1) * r;
    o[7] = (m[8] * s5 - m[10] * s2 + m[11] * s1) * r;
    o[8] = (m[4] * c4 - m[5] * c2 + m[7] * c0) * r;
    o[9] = (-m[0] * c4 + m[1] * c2 - m[3] * c0) * r;
    o[10] = (m[12] * s4 - m[13] * s2 + m[15] * s0) * r;
    o[11] = (-m[8] * s4 + m[9] * s2 - m[11] * s0) * r;
    o[12] = (-m[4] * c3 + m[5] * c1 - m[6] * c0) * r;
    o[13] = (m[0] * c3 - m[1] * c1 + m[2] * c0) * r;
    o[14] = (-m[12] * s3 + m[13] * s1 - m[14] * s0) * r;
    o[15] = (m[8] * s3 - m[9] * s1 + m[10] * s0) * r;
}
}  // namespace gf_shim_detail

class GfMatrix4f;

class GfMatrix4d {
  public:
    double _mtx[4][4];
    GfMatrix4d() { std::memset(_mtx, 0, sizeof(_mtx)); }
    explicit GfMatrix4d(double s) {
        std::memset(_mtx, 0, sizeof(_mtx));
        _mtx[0][0] = _mtx[1][1] = _mtx[2][2] = _mtx[3][3] = s;
    }
    explicit GfMatrix4d(int s) : GfMatrix4d((double)s) {}
    explicit GfMatrix4d(const double m[4][4]) { std::memcpy(_mtx, m, sizeof(_mtx)); }
    explicit GfMatrix4d(const GfMatrix4f &m);
    double *operator[](int i) { return _mtx[i]; }
    const double *operator[](int i) const { return _mtx[i]; }
    double *data() { return &_mtx[0][0]; }
    const double *data() const { return &_mtx[0][0]; }
    GfMatrix4d GetInverse(double *det = nullptr, double eps = 0.0) const {
        (void)det;
        (void)eps;
        GfMatrix4d r;
        gf_shim_detail::inverse4(&_mtx[0][0], &r._mtx[0][0]);
        return r;
    }
    GfVec3d Transform(const GfVec3d &v) const {
        return GfProject(GfVec4d(v[0] * _mtx[0][0] + v[1] * _mtx[1][0] + v[2] * _mtx[2][0] + _mtx[3][0],
                                 v[0] * _mtx[0][1] + v[1] * _mtx[1][1] + v[2] * _mtx[2][1] + _mtx[3][1],
                                 v[0] * _mtx[0][2] + v[1] * _mtx[1][2] + v[2] * _mtx[2][2] + _mtx[3][2],
                                 v[0] * _mtx[0][3] + v[1] * _mtx[1][3] + v[2] * _mtx[2][3] + _mtx[3][3]));
    }
    GfVec3d TransformDir(const GfVec3d &v) const {
        return GfVec3d(v[0] * _mtx[0][0] + v[1] * _mtx[1][0] + v[2] * _mtx[2][0],
                       v[0] * _mtx[0][1] + v[1] * _mtx[1][1] + v[2] * _mtx[2][1],
                       v[0] * _mtx[0][2] + v[1] * _mtx[1][2] + v[2] * _mtx[2][2]);
    }
    GfMatrix4d operator*(const GfMatrix4d &b) const {
        GfMatrix4d r;
        for (int i = 0; i < 4; ++i)
            for (int j = 0; j < 4; ++j)
                r._mtx[i][j] = _mtx[i][0] * b._mtx[0][j] + _mtx[i][1] * b._mtx[1][j] + _mtx[i][2] * b._mtx[2][j] +
                               _mtx[i][3] * b._mtx[3][j];
        return r;
    }
    bool operator==(const GfMatrix4d &o) const { return std::memcmp(_mtx, o._mtx, sizeof(_mtx)) == 0; }
    bool operator!=(const GfMatrix4d &o) const { return !(*this == o); }
};

class GfMatrix4f {
  public:
    float _mtx[4][4];
    GfMatrix4f() { std::memset(_mtx, 0, sizeof(_mtx)); }
    explicit GfMatrix4f(float s) {
        std::memset(_mtx, 0, sizeof(_mtx));
        _mtx[0][0] = _mtx[1][1] = _mtx[2][2] = _mtx[3][3] = s;
    }
    explicit GfMatrix4f(int s) : GfMatrix4f((float)s) {}
    explicit GfMatrix4f(const GfMatrix4d &m) {
        for (int i = 0; i < 4; ++i)
            for (int j = 0; j < 4; ++j) _mtx[i][j] = (float)m._mtx[i][j];
    }
    float *operator[](int i) { return _mtx[i]; }
    const float *operator[](int i) const { return _mtx[i]; }
    float *data() { return &_mtx[0][0]; }
    const float *data() const { return &_mtx[0][0]; }
    GfMatrix4f GetInverse(double *det = nullptr, double eps = 0.0) const {
        (void)det;
        (void)eps;
        double m[16], o[16];
        for (int i = 0; i < 16; ++i) m[i] = (double)(&_mtx[0][0])[i];
        gf_shim_detail::inverse4(m, o);
        GfMatrix4f r;
        for (int i = 0; i < 16; ++i) (&r._mtx[0][0])[i] = (float)o[i];
        return r;
    }
    GfVec3f Transform(const GfVec3f &v) const {
        return GfProject(GfVec4f(v[0] * _mtx[0][0] + v[1] * _mtx[1][0] + v[2] * _mtx[2][0] + _mtx[3][0],
                                 v[0] * _mtx[0][1] + v[1] * _mtx[1][1] + v[2] * _mtx[2][1] + _mtx[3][1],
                                 v[0] * _mtx[0][2] + v[1] * _mtx[1][2] + v[2] * _mtx[2][2] + _mtx[3][2],
                                 v[0] * _mtx[0][3] + v[1] * _mtx[1][3] + v[2] * _mtx[2][3] + _mtx[3][3]));
    }
    GfVec3f TransformDir(const GfVec3f &v) const {
        return GfVec3f(v[0] * _mtx[0][0] + v[1] * _mtx[1][0] + v[2] * _mtx[2][0],
                       v[0] * _mtx[0][1] + v[1] * _mtx[1][1] + v[2] * _mtx[2][1],
                       v[0] * _mtx[0][2] + v[1] * _mtx[1][2] + v[2] * _mtx[2][2]);
    }
    GfVec3f ExtractTranslation() const { return GfVec3f(_mtx[3][0], _mtx[3][1], _mtx[3][2]); }
    GfMatrix4f operator*(const GfMatrix4f &b) const {
        GfMatrix4f r;
        for (int i = 0; i < 4; ++i)
            for (int j = 0; j < 4; ++j)
                r._mtx[i][j] = _mtx[i][0] * b._mtx[0][j] + _mtx[i][1] * b._mtx[1][j] + _mtx[i][2] * b._mtx[2][j] +
                               _mtx[i][3] * b._mtx[3][j];
        return r;
    }
};
inline GfMatrix4d::GfMatrix4d(const GfMatrix4f &m) {
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) _mtx[i][j] = (double)m._mtx[i][j];
}

class GfRange3f {
  public:
    GfRange3f() { SetEmpty(); }
    GfRange3f(const GfVec3f &mn, const GfVec3f &mx) : _min(mn), _max(mx) {}
    void SetEmpty() {
        _min = GfVec3f(FLT_MAX, FLT_MAX, FLT_MAX);
        _max = GfVec3f(-FLT_MAX, -FLT_MAX, -FLT_MAX);
    }
    bool IsEmpty() const { return _min[0] > _max[0] || _min[1] > _max[1] || _min[2] > _max[2]; }
    const GfVec3f &GetMin() const { return _min; }
    const GfVec3f &GetMax() const { return _max; }
    GfVec3f GetSize() const { return _max - _min; }
    GfVec3f GetMidpoint() const { return 0.5 * _min + 0.5 * _max; }
    GfRange3f &ExtendBy(const GfVec3f &p) {
        for (int i = 0; i < 3; ++i) {
            if (p[i] < _min[i]) _min[i] = p[i];
            if (p[i] > _max[i]) _max[i] = p[i];
        }
        return *this;
    }
    GfRange3f &ExtendBy(const GfRange3f &r) {
        ExtendBy(r._min);
        ExtendBy(r._max);
        return *this;
    }

  private:
    GfVec3f _min, _max;
};

class GfRect2i {
  public:
    GfRect2i() = default;
    GfRect2i(const GfVec2i &mn, int w, int h) : _min(mn), _w(w), _h(h) {}
    int GetWidth() const { return _w; }
    int GetHeight() const { return _h; }

  private:
    GfVec2i _min;
    int _w = 0, _h = 0;
};

PXR_NAMESPACE_CLOSE_SCOPE
