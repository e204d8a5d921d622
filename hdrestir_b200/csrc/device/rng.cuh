// Restir::Rng on the device (reference: source/core/rng.h:10-56).
//
// The reference seeds one std::mt19937_64 per pixel per frame
// (passes/integration_pass.cpp:210-211) and draws every random number with
// std::uniform_real_distribution<float>, i.e. libstdc++'s
// generate_canonical<float, 24>: one 64-bit output y, converted to float with
// round-to-nearest, times 2^-64, clamped below 1.
//
// A full MT19937-64 state is 312 words (2.5 KB): far too much per thread.
// Output k of the first twist only needs a few words of the seeding
// recurrence s[i] = 6364136223846793005 * (s[i-1] ^ (s[i-1] >> 62)) + i:
//   k <  156 : s[k+156] ^ T(s[k], s[k+1])
//   k <  311 : s[k] ^ T(s[k-156], s[k-155]) ^ T(s[k], s[k+1])
//   k == 311 : s[311] ^ T(s[155], s[156]) ^ T(s[311], new0),
//              new0 = s[156] ^ T(s[0], s[1])
// (T = the MT twist of the upper bit of a and the lower 31 bits of b), so the
// stream walks up to four seeding cursors in registers. Draws 312 and later,
// which no configured path reaches in practice, fall back to a full state in
// the caller-provided local array `spill`.
#pragma once

#include "gf.cuh"

namespace hdr {

constexpr uint64_t kMtMult = 6364136223846793005ULL;
constexpr uint64_t kMtMatrixA = 0xB5026F5AA96619E9ULL;
constexpr uint64_t kMtUpper = 0xFFFFFFFF80000000ULL;
constexpr uint64_t kMtLower = 0x7FFFFFFFULL;

HDR_HD uint64_t mt_seed_step(uint64_t prev, uint32_t i) { return kMtMult * (prev ^ (prev >> 62)) + (uint64_t)i; }
HDR_HD uint64_t mt_twist(uint64_t a, uint64_t b) {
    const uint64_t x = (a & kMtUpper) | (b & kMtLower);
    return (x >> 1) ^ ((x & 1ULL) ? kMtMatrixA : 0ULL);
}
HDR_HD uint64_t mt_temper(uint64_t y) {
    y ^= (y >> 29) & 0x5555555555555555ULL;
    y ^= (y << 17) & 0x71D67FFFEDA60000ULL;
    y ^= (y << 37) & 0xFFF7EEE000000000ULL;
    y ^= (y >> 43);
    return y;
}
// generate_canonical<float,24> for a 64-bit engine, then uniform_real_distribution(0,1).
HDR_HD float mt_to_float(uint64_t y) {
#if defined(__CUDA_ARCH__)
    float f = __ull2float_rn(y) * 5.42101086242752217e-20f;  // exactly 2^-64
#else
    float f = (float)y * 5.42101086242752217e-20f;
#endif
    return (f >= 1.0f) ? 0.99999994f : f;  // nextafter(1.0f, 0.0f)
}

// In-place regeneration of one full MT state block (used past 311 draws only).
HDR_HD void mt_full_twist(uint64_t *mt) {
    for (int k = 0; k < 312 - 156; ++k) mt[k] = mt[k + 156] ^ mt_twist(mt[k], mt[k + 1]);
    for (int k = 312 - 156; k < 311; ++k) mt[k] = mt[k - 156] ^ mt_twist(mt[k], mt[k + 1]);
    mt[311] = mt[155] ^ mt_twist(mt[311], mt[0]);
}

struct MtStream {
    uint64_t a;     // s[k]
    uint64_t b;     // s[k+1]
    uint64_t c;     // k < 156: s[k+156]; 156 <= k < 312: s[k-156]
    uint64_t d;     // 156 <= k < 312: s[k-155]
    uint64_t new0;  // first word after the first twist
    uint32_t k;     // index of the next output
    uint32_t seed;
    uint64_t *spill;  // 312-word local scratch, touched only from draw 312 on

    HDR_HD void init(uint32_t s, uint64_t *spill_buf) {
        seed = s;
        spill = spill_buf;
        k = 0;
        a = (uint64_t)s;
        b = mt_seed_step(a, 1);
        uint64_t x = b;
        for (uint32_t i = 2; i <= 156; ++i) x = mt_seed_step(x, i);
        c = x;
        d = 0;
        new0 = 0;
    }

    HDR_HD uint64_t next_raw() {
        uint64_t r;
        if (k < 156) {
            r = c ^ mt_twist(a, b);
            a = b;
            b = mt_seed_step(b, k + 2);
            c = mt_seed_step(c, k + 157);
            ++k;
            if (k == 156) {  // switch cursors: (a, b) continue at s[156], (c, d) restart at s[0]
                c = (uint64_t)seed;
                d = mt_seed_step(c, 1);
                new0 = a ^ mt_twist(c, d);
            }
        } else if (k < 311) {
            r = (a ^ mt_twist(c, d)) ^ mt_twist(a, b);
            a = b;
            b = mt_seed_step(b, k + 2);
            c = d;
            d = mt_seed_step(d, k - 154);
            ++k;
        } else if (k == 311) {
            r = (a ^ mt_twist(c, d)) ^ mt_twist(a, new0);
            ++k;
        } else if (spill == nullptr) {  // caller declared it never draws past 311
            r = 0;
            ++k;
        } else {
            const uint32_t idx = (k - 312) % 312;
            if (idx == 0) {
                if (k == 312) {  // rebuild the first twisted block
                    spill[0] = (uint64_t)seed;
                    for (uint32_t i = 1; i < 312; ++i) spill[i] = mt_seed_step(spill[i - 1], i);
                    mt_full_twist(spill);
                }
                mt_full_twist(spill);
            }
            r = spill[idx];
            ++k;
        }
        return mt_temper(r);
    }

    HDR_HD float next_float() { return mt_to_float(next_raw()); }
};

// A stream in three uint4 planes of n entries (entry i): the state of a
// stream below draw 312, handed from one kernel to the next.
__device__ __forceinline__ void store_stream(uint4 *st, size_t i, size_t n, const MtStream &r) {
    st[i] = make_uint4((unsigned)r.a, (unsigned)(r.a >> 32), (unsigned)r.b, (unsigned)(r.b >> 32));
    st[n + i] = make_uint4((unsigned)r.c, (unsigned)(r.c >> 32), (unsigned)r.d, (unsigned)(r.d >> 32));
    st[2 * n + i] = make_uint4((unsigned)r.new0, (unsigned)(r.new0 >> 32), r.k, r.seed);
}
__device__ __forceinline__ MtStream load_stream(const uint4 *st, size_t i, size_t n) {
    const uint4 p = st[i], q = st[n + i], w = st[2 * n + i];
    MtStream r;
    r.a = (uint64_t)p.x | ((uint64_t)p.y << 32);
    r.b = (uint64_t)p.z | ((uint64_t)p.w << 32);
    r.c = (uint64_t)q.x | ((uint64_t)q.y << 32);
    r.d = (uint64_t)q.z | ((uint64_t)q.w << 32);
    r.new0 = (uint64_t)w.x | ((uint64_t)w.y << 32);
    r.k = w.z;
    r.seed = w.w;
    r.spill = nullptr;
    return r;
}

}  // namespace hdr
