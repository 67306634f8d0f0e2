// Device helpers shared by the sweep, field and population kernels.
//
// The counter hash is the reference device engine's (glazier-cuda/src/lib.rs
// 33-50): SplitMix64's finaliser over seed ^ C1*site ^ C2*step ^ C3*stream.
// The step and stream parts are the same for every thread of a launch, so the
// host folds them into one 64-bit word per stream and a draw costs one
// 64x32-bit multiply plus the finaliser.
#pragma once

#include <cstdint>

namespace glz {

constexpr uint64_t kSiteMul = 0xD1B54A32D192ED03ULL;
constexpr uint64_t kStepMul = 0xA0761D6478BD642FULL;
constexpr uint64_t kStreamMul = 0xE7037ED1A0B428DBULL;

// The population step's draws take stream index 4*16, clear of the sweep's
// 4*colour + {0, 1} for colours 0..7.
constexpr int kPopulationStream = 16;

// Division of a 32-bit unsigned number by a divisor fixed for a launch, by a
// high multiply and two shifts (T. Granlund, P. L. Montgomery, "Division by
// Invariant Integers using Multiplication", PLDI 1994, section 4): with
// l = ceil(log2 d) and m = floor(2^32 (2^l - d) / d) + 1, the quotient of n is
// (t + ((n - t) >> min(l, 1))) >> max(l - 1, 0) for t = mulhi(m, n), exact
// for every n < 2^32 and 1 <= d <= 2^31.
struct Divider {
    uint32_t d = 1, m = 1, s1 = 0, s2 = 0;
};

inline Divider make_divider(uint32_t d) {
    Divider v;
    int l = 0;
    while ((1ull << l) < d) ++l;
    v.d = d;
    v.m = (uint32_t)(((1ull << 32) * ((1ull << l) - d)) / d + 1);
    v.s1 = l < 1 ? l : 1;
    v.s2 = l > 1 ? l - 1 : 0;
    return v;
}

__device__ __forceinline__ uint32_t udiv(const Divider &v, uint32_t n) {
    const uint32_t t = __umulhi(v.m, n);
    return (t + ((n - t) >> v.s1)) >> v.s2;
}

__host__ __device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

// seed ^ C2*step ^ C3*(4*colour + index): the launch-uniform part of a draw.
__host__ __device__ __forceinline__ uint64_t stream_key(uint64_t seed, int32_t step, int colour, int index) {
    return seed ^ (kStepMul * (uint64_t)(int64_t)step) ^ (kStreamMul * (uint64_t)(int64_t)(4 * colour + index));
}

__host__ __device__ __forceinline__ uint64_t draw(uint64_t key, uint32_t site) {
    return mix64(key ^ (kSiteMul * (uint64_t)site));
}

// A draw reduced mod N, the neighbourhood size, fixed at compile time: a
// power of two by its mask, any other through the 32-bit halves, as
// ((hi mod N) (2^32 mod N) + lo mod N) mod N, which needs no 64-bit division
// and is the same residue.
template <int N>
__host__ __device__ __forceinline__ int pick_of(uint64_t bits) {
    if constexpr ((N & (N - 1)) == 0) {
        return (int)(bits & (uint64_t)(N - 1));
    } else {
        constexpr uint32_t wrap32 = (uint32_t)((1ull << 32) % N);
        const uint32_t hi = (uint32_t)(bits >> 32) % (uint32_t)N, lo = (uint32_t)bits % (uint32_t)N;
        return (int)((hi * wrap32 + lo) % (uint32_t)N);
    }
}

// (bits >> 11) * 2^-53 rounded to f32: the reference computes the product in
// f64 and rounds once (lib.rs:48-50); rounding the 53-bit integer to f32 and
// scaling by a power of two rounds the same value once, so the bits agree.
__device__ __forceinline__ float to_f32(uint64_t bits) { return __ull2float_rn(bits >> 11) * 0x1p-53f; }

__device__ __forceinline__ double to_f64(uint64_t bits) { return __ull2double_rn(bits >> 11) * 0x1p-53; }

// exp for the Metropolis test, written from Cody and Waite's method (W. J.
// Cody, W. Waite, "Software Manual for the Elementary Functions", 1980):
// k = rint(x log2 e), r = x - k ln2 with ln 2 split hi + lo, e^r by the
// degree-7 Taylor polynomial in fused multiply-adds, scaled by 2^k through the
// exponent field. Only correctly rounded operations, so a host replay gets the
// same bits. Below -87 the result is zero: no draw in [0, 1) falls under it.
__device__ __forceinline__ float metropolis_exp(float x) {
    if (x < -87.0f) return 0.0f;
    if (x > 88.0f) return __int_as_float(0x7f800000);
    float k = rintf(__fmul_rn(x, 1.44269504088896341f));
    float r = __fmaf_rn(k, -0.693145751953125f, x);
    r = __fmaf_rn(k, -1.428606765330187e-06f, r);
    float p = 1.98412698e-04f;
    p = __fmaf_rn(p, r, 1.38888889e-03f);
    p = __fmaf_rn(p, r, 8.33333333e-03f);
    p = __fmaf_rn(p, r, 4.16666667e-02f);
    p = __fmaf_rn(p, r, 1.66666667e-01f);
    p = __fmaf_rn(p, r, 0.5f);
    p = __fmaf_rn(p, r, 1.0f);
    p = __fmaf_rn(p, r, 1.0f);
    int ki = (int)k;
    return __fmul_rn(p, __int_as_float((ki + 127) << 23));
}

// Natural log for the motility term's geometric means, written from the
// series ln m = 2 atanh(s) = 2 (s + s^3/3 + s^5/5 + s^7/7 + s^9/9 + ...),
// s = (m - 1) / (m + 1) (Abramowitz and Stegun 4.1.27), on a mantissa m
// reduced to [sqrt(1/2), sqrt(2)] so |s| < 0.172 and the terms past s^9 fall
// below f32 precision; the exponent adds e ln 2 with ln 2 split hi + lo. Only
// correctly rounded operations, so a host replay gets the same bits. For
// x > 0 and finite.
__device__ __forceinline__ float motility_log(float x) {
    int e = 0;
    if (x < 1.17549435e-38f) {  // subnormal: scale into the normal range
        x = __fmul_rn(x, 16777216.0f);
        e = -24;
    }
    const int bits = __float_as_int(x);
    e += ((bits >> 23) & 0xff) - 127;
    float m = __int_as_float((bits & 0x007fffff) | 0x3f800000);  // [1, 2)
    if (m > 1.41421356f) {
        m = __fmul_rn(m, 0.5f);
        e += 1;
    }
    const float s = __fdiv_rn(__fsub_rn(m, 1.0f), __fadd_rn(m, 1.0f));
    const float s2 = __fmul_rn(s, s);
    float p = 0.111111111f;
    p = __fmaf_rn(p, s2, 0.142857143f);
    p = __fmaf_rn(p, s2, 0.2f);
    p = __fmaf_rn(p, s2, 0.333333333f);
    p = __fmul_rn(p, s2);
    const float lm = __fmul_rn(__fmul_rn(2.0f, s), __fadd_rn(1.0f, p));
    const float fe = (float)e;
    return __fadd_rn(__fmaf_rn(fe, 0.693145751953125f, lm), __fmul_rn(fe, 1.428606765330187e-06f));
}

// A nematic field component in the per-cell sums, in units of 2^-32 rounded
// to nearest: the sums are exact and their order does not matter.
__device__ __forceinline__ long long nematic_fixed(float q) { return __double2ll_rn((double)q * 4294967296.0); }

// In-plane anisotropy ((c_xx - c_yy), 2 c_xy) / (c_xx + c_yy) of a cell of n
// sites from its exact moment sums (moments.rs anisotropy; the quantity the
// nematic term dots with the field): zero below two sites or for a vanishing
// trace.
template <int DIM>
__device__ __forceinline__ void anisotropy(long long n, const long long *m, double &a0, double &a1) {
    a0 = 0.0;
    a1 = 0.0;
    if (n < 2) return;
    const double dn = (double)n;
    const double mx = (double)m[0] / dn, my = (double)m[1] / dn;
    const double cxx = (double)m[DIM == 2 ? 2 : 3] / dn - mx * mx;
    const double cyy = (double)m[DIM == 2 ? 3 : 4] / dn - my * my;
    const double cxy = (double)m[DIM == 2 ? 4 : 6] / dn - mx * my;
    const double trace = cxx + cyy;
    if (!(trace > 1e-12)) return;
    a0 = (cxx - cyy) / trace;
    a1 = 2.0 * cxy / trace;
}

__host__ __device__ __forceinline__ int wrap(int v, int n) {
    int r = v % n;
    return r < 0 ? r + n : r;
}

// Minimum image of an integer offset on a periodic axis (moments.rs:36-46).
__host__ __device__ __forceinline__ int fold_int(int d, int span) {
    if (2 * d > span) return d - span;
    if (2 * d < -span) return d + span;
    return d;
}

// Per-cell (volume, surface) deltas packed in one 64-bit word so a commit is
// one atomic: the word holds surface * 2^32 + volume modulo 2^64, and a
// volume delta below 2^31 in size decodes exactly.
__device__ __forceinline__ unsigned long long pack_delta(int dv, int ds) {
    return ((unsigned long long)(long long)ds << 32) + (unsigned long long)(long long)dv;
}

__host__ __device__ __forceinline__ void unpack_delta(long long p, int &dv, int &ds) {
    dv = (int)(uint32_t)(uint64_t)p;
    ds = (int)((p - (long long)dv) >> 32);
}

}  // namespace glz
