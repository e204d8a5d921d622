// Spectral core: 4 wavelength samples in 360-830 nm.
// SampledWavelengths/SampledSpectrum: source/core/spectrum.h:8-149
// SpectrumToRGB / RGBToSpectrum / SpectrumLuminance: source/core/spectrum.cpp:26-109
// (Wyman-2013 CIE fit -> XYZ -> linear sRGB white-balanced to illuminant E;
//  Gaussian RGB uplift). The float expression order follows the reference;
// exp is CUDA's expf (glibc's expf differs by a few ulp at most).
#pragma once

#include "gf.cuh"

namespace hdr {

constexpr float kLambdaMin = 360.0f;
constexpr float kLambdaMax = 830.0f;

struct Lambda {
    float l[4];
};

struct Spec {
    float v[4];
};

HDR_HD Spec spec(float s) { return Spec{{s, s, s, s}}; }
HDR_HD Spec operator+(Spec a, Spec b) {
    return Spec{{a.v[0] + b.v[0], a.v[1] + b.v[1], a.v[2] + b.v[2], a.v[3] + b.v[3]}};
}
HDR_HD Spec operator*(Spec a, Spec b) {
    return Spec{{a.v[0] * b.v[0], a.v[1] * b.v[1], a.v[2] * b.v[2], a.v[3] * b.v[3]}};
}
HDR_HD Spec operator*(Spec a, float s) { return Spec{{a.v[0] * s, a.v[1] * s, a.v[2] * s, a.v[3] * s}}; }
HDR_HD bool is_black(Spec a) {
    for (int i = 0; i < 4; ++i)
        if (a.v[i] > 0.0f) return false;
    return true;
}
HDR_HD float spec_max(Spec a) {  // SampledSpectrum::Max (std::max fold)
    float m = a.v[0];
    for (int i = 1; i < 4; ++i) m = smaxf(m, a.v[i]);
    return m;
}

// SampledWavelengths::SampleUniform (spectrum.h:24-37)
HDR_HD Lambda sample_uniform_wavelengths(float u) {
    Lambda w;
    w.l[0] = kLambdaMin + u * (kLambdaMax - kLambdaMin);
    for (int i = 1; i < 4; ++i) {
        w.l[i] = w.l[0] + ((float)i * (kLambdaMax - kLambdaMin) / 4.0f);
        if (w.l[i] > kLambdaMax) w.l[i] -= (kLambdaMax - kLambdaMin);
    }
    return w;
}

#if defined(__CUDA_ARCH__)
#define HDR_EXPF expf
#define HDR_POWF powf
#define HDR_SINF sinf
#define HDR_COSF cosf
#define HDR_LOGF logf
#else
#define HDR_EXPF __builtin_expf
#define HDR_POWF __builtin_powf
#define HDR_SINF __builtin_sinf
#define HDR_COSF __builtin_cosf
#define HDR_LOGF __builtin_logf
#endif

HDR_HD float x_fit_1931(float w) {
    const float t1 = (w - 442.0f) * ((w < 442.0f) ? 0.0624f : 0.0374f);
    const float t2 = (w - 599.8f) * ((w < 599.8f) ? 0.0264f : 0.0323f);
    const float t3 = (w - 501.1f) * ((w < 501.1f) ? 0.0490f : 0.0382f);
    return 0.362f * HDR_EXPF(-0.5f * t1 * t1) + 1.056f * HDR_EXPF(-0.5f * t2 * t2) -
           0.065f * HDR_EXPF(-0.5f * t3 * t3);
}
HDR_HD float y_fit_1931(float w) {
    const float t1 = (w - 568.8f) * ((w < 568.8f) ? 0.0213f : 0.0247f);
    const float t2 = (w - 530.9f) * ((w < 530.9f) ? 0.0613f : 0.0322f);
    return 0.821f * HDR_EXPF(-0.5f * t1 * t1) + 0.286f * HDR_EXPF(-0.5f * t2 * t2);
}
HDR_HD float z_fit_1931(float w) {
    const float t1 = (w - 437.0f) * ((w < 437.0f) ? 0.0845f : 0.0278f);
    const float t2 = (w - 459.0f) * ((w < 459.0f) ? 0.0385f : 0.0725f);
    return 1.217f * HDR_EXPF(-0.5f * t1 * t1) + 0.681f * HDR_EXPF(-0.5f * t2 * t2);
}

// Per-wavelength CIE weights depend only on the wavelengths; a pixel computes
// them once per frame and reuses them for every SpectrumToRGB of that pixel.
struct CieTable {
    float x[4], y[4], z[4];
};
HDR_HD CieTable make_cie_table(const Lambda &w) {
    CieTable t;
    for (int i = 0; i < 4; ++i) {
        t.x[i] = x_fit_1931(w.l[i]);
        t.y[i] = y_fit_1931(w.l[i]);
        t.z[i] = z_fit_1931(w.l[i]);
    }
    return t;
}

// SpectrumToRGB (spectrum.cpp:26-63)
HDR_HD V3 spectrum_to_rgb(const Spec &s, const CieTable &t) {
    float X = 0.0f, Y = 0.0f, Z = 0.0f;
    float weight = (kLambdaMax - kLambdaMin) / 4.0f;
    weight /= 106.856f;
    for (int i = 0; i < 4; ++i) {
        const float val = s.v[i];
        X += val * t.x[i];
        Y += val * t.y[i];
        Z += val * t.z[i];
    }
    X *= weight;
    Y *= weight;
    Z *= weight;
    float r = 3.2404542f * X - 1.5371385f * Y - 0.4985314f * Z;
    float g = -0.9692660f * X + 1.8760108f * Y + 0.0415560f * Z;
    float b = 0.0556434f * X - 0.2040259f * Y + 1.0572252f * Z;
    r /= 1.198185f;
    g /= 0.950366f;
    b /= 0.907827f;
    return V3{smaxf(0.0f, r), smaxf(0.0f, g), smaxf(0.0f, b)};
}

// Gaussian uplift basis per wavelength (spectrum.cpp:66-98): exp terms depend
// only on the wavelength, so they are tabulated once per pixel as well.
struct UpliftTable {
    float r[4], g[4], b[4];
};
HDR_HD float uplift_gaussian(float x, float center, float sigma) {
    const float t = (x - center) / sigma;
    return HDR_EXPF(-0.5f * t * t);
}
HDR_HD UpliftTable make_uplift_table(const Lambda &w) {
    UpliftTable u;
    for (int i = 0; i < 4; ++i) {
        u.r[i] = uplift_gaussian(w.l[i], 615.0f, 20.0f);
        u.g[i] = uplift_gaussian(w.l[i], 540.0f, 20.0f);
        u.b[i] = uplift_gaussian(w.l[i], 460.0f, 20.0f);
    }
    return u;
}

// RGBToSpectrum (spectrum.cpp:72-103)
HDR_HD Spec rgb_to_spectrum(V3 rgb, const UpliftTable &u) {
    const float white = sminf(rgb.x, sminf(rgb.y, rgb.z));
    const V3 rem = V3{rgb.x - white, rgb.y - white, rgb.z - white};
    Spec s;
    for (int i = 0; i < 4; ++i) {
        float val = white;
        val += rem.x * u.r[i] * 1.295f;
        val += rem.y * u.g[i] * 1.556f;
        val += rem.z * u.b[i] * 1.382f;
        s.v[i] = smaxf(0.0f, val);
    }
    return s;
}

// SpectrumLuminance (spectrum.cpp:105-109)
HDR_HD float spectrum_luminance(const Spec &s, const CieTable &t) {
    const V3 rgb = spectrum_to_rgb(s, t);
    return smaxf(0.0f, 0.2126f * rgb.x + 0.7152f * rgb.y + 0.0722f * rgb.z);
}

// Per-pixel spectral context: wavelengths and the tables derived from them.
struct SpectralCtx {
    Lambda lambda;
    CieTable cie;
    UpliftTable up;
};
HDR_HD SpectralCtx make_spectral_ctx(float u) {
    SpectralCtx c;
    c.lambda = sample_uniform_wavelengths(u);
    c.cie = make_cie_table(c.lambda);
    c.up = make_uplift_table(c.lambda);
    return c;
}

}  // namespace hdr
