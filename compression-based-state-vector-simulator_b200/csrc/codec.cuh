// Error-bounded quantiser of the block codec (host and device).
//
// Replaces the reference's log compander + nvCOMP Bitcomp lossy FP64 stage
// (src/cppsim/compand_kernel.cuh:5-30, compand_bitcomp_pipeline.cuh:14-62).
// That pipeline bounds every real component by |xhat - x| <= (eps_rel|x| +
// eps_abs)/2 (a round-to-nearest step of log1p(eps_rel) in the log domain,
// offset tau' = (1-2 eps_rel) eps_abs/eps_rel).  This quantiser meets the same
// pointwise bound with integer and exact floating-point operations only:
//
//   |x| <  2^e0 : c = rint(|x| * 2^L)                (2^-L <= eps_abs)
//   |x| >= 2^e0 : c = 2^m + (bits(|x|) rounded to m mantissa bits) - bits(2^e0)
//                                                     (2^-m <= eps_rel)
//   e0 = m - L, q = sign ? -c : c
//
// Both steps coincide in the binade [2^e0, 2^(e0+1)), so c is continuous and
// monotone in |x|.  The CPU oracle (oracle/codec_oracle.c) states the same map;
// the integer codes agree bit for bit.
//
// Chunk payload layout (32-lane vertical frame of reference): the 2^(C+1)
// components of a chunk (interleaved re, im) are split into 32 streams,
// stream l = components l, l+32, ...; u = q - base (base = chunk minimum) is
// packed LSB first in `width` bits per component into rows of 32-bit words,
// word r of stream l at index r*32 + l.  rows = ceil(per_lane*width/32),
// payload bytes = 128*rows.
#pragma once

#include <cstdint>
#include <cstring>
#include <cmath>

#include "internal.h"

namespace qs {

constexpr int64_t kCodeLimit = 0x3fffffff;

__host__ __device__ inline uint64_t payload_rows(int C, uint32_t width) {
    const uint64_t per_lane = (uint64_t(2) << C) / 32;
    return (per_lane * width + 31) / 32;
}

__host__ __device__ inline uint64_t payload_bytes(int C, uint32_t width) {
    return payload_rows(C, width) * 128;
}

__host__ __device__ inline uint32_t bit_length(uint32_t v) {
#ifdef __CUDA_ARCH__
    return 32u - __clz(v);
#else
    return v ? 32u - (uint32_t)__builtin_clz(v) : 0u;
#endif
}

// ---------------------------------------------------------------- float
__host__ __device__ inline int32_t quantize(float x, CodecParams p) {
    uint32_t bits;
#ifdef __CUDA_ARCH__
    bits = __float_as_uint(x);
#else
    std::memcpy(&bits, &x, 4);
#endif
    const uint32_t abits = bits & 0x7fffffffu;
    const bool neg = (bits >> 31) != 0;
    const int e0 = p.m - p.L;
    const uint32_t thr = uint32_t(e0 + 127) << 23;
    int64_t c;
    if (abits < thr) {
        float a;
#ifdef __CUDA_ARCH__
        // rint(a * 2^L) without a conversion instruction: a * 2^L < 2^23 here,
        // so fma(a, 2^L, 2^23) rounds it to an integer (nearest, ties to even)
        // in the low mantissa bits.
        a = __uint_as_float(abits);
        const float scale = __uint_as_float(uint32_t(p.L + 127) << 23);  // 2^L exactly
        const float r = __fmaf_rn(a, scale, 8388608.0f);
        c = (int64_t)(__float_as_uint(r) - 0x4b000000u);
#else
        std::memcpy(&a, &abits, 4);
        c = (int64_t)std::nearbyint(a * std::ldexp(1.0f, p.L));
#endif
    } else {
        const int sh = 23 - p.m;
        const uint64_t half = sh > 0 ? (uint64_t(1) << (sh - 1)) : 0;
        c = (int64_t)((uint64_t(abits) + half) >> sh) - (int64_t(e0 + 127) << p.m) + (int64_t(1) << p.m);
    }
    if (c > kCodeLimit) c = kCodeLimit;
    return (int32_t)(neg ? -c : c);
}

__host__ __device__ inline float dequantize_f32(int32_t q, CodecParams p) {
    const bool neg = q < 0;
    const int64_t c = neg ? -(int64_t)q : (int64_t)q;
    float a;
    if (c <= (int64_t(1) << p.m)) {
#ifdef __CUDA_ARCH__
        // (float)c for c <= 2^23 without a conversion instruction
        const float iscale = __uint_as_float(uint32_t(127 - p.L) << 23);  // 2^-L exactly
        const float cf = __uint_as_float(0x4b000000u + (uint32_t)c) - 8388608.0f;
        a = __fmul_rn(cf, iscale);
#else
        a = (float)c * std::ldexp(1.0f, -p.L);
#endif
    } else {
        const int e0 = p.m - p.L;
        const int sh = 23 - p.m;
        const uint32_t bits =
            (uint32_t)((uint64_t)(c - (int64_t(1) << p.m) + (int64_t(e0 + 127) << p.m)) << sh);
#ifdef __CUDA_ARCH__
        a = __uint_as_float(bits);
#else
        std::memcpy(&a, &bits, 4);
#endif
    }
    return neg ? -a : a;
}

// ---------------------------------------------------------------- double
__host__ __device__ inline int32_t quantize(double x, CodecParams p) {
    uint64_t bits;
#ifdef __CUDA_ARCH__
    bits = (uint64_t)__double_as_longlong(x);
#else
    std::memcpy(&bits, &x, 8);
#endif
    const uint64_t abits = bits & 0x7fffffffffffffffull;
    const bool neg = (bits >> 63) != 0;
    const int e0 = p.m - p.L;
    const uint64_t thr = uint64_t(e0 + 1023) << 52;
    int64_t c;
    if (abits < thr) {
        double a;
#ifdef __CUDA_ARCH__
        // rint(a * 2^L) via fma(a, 2^L, 2^52): exact integer in the low bits
        a = __longlong_as_double((long long)abits);
        const double scale = __longlong_as_double((long long)(uint64_t(p.L + 1023) << 52));
        const double r = __fma_rn(a, scale, 4503599627370496.0);
        c = (int64_t)((uint64_t)__double_as_longlong(r) - 0x4330000000000000ull);
#else
        std::memcpy(&a, &abits, 8);
        c = (int64_t)std::nearbyint(a * std::ldexp(1.0, p.L));
#endif
    } else {
        const int sh = 52 - p.m;
        const uint64_t half = uint64_t(1) << (sh - 1);
        c = (int64_t)((abits + half) >> sh) - (int64_t(e0 + 1023) << p.m) + (int64_t(1) << p.m);
    }
    if (c > kCodeLimit) c = kCodeLimit;
    return (int32_t)(neg ? -c : c);
}

__host__ __device__ inline double dequantize_f64(int32_t q, CodecParams p) {
    const bool neg = q < 0;
    const int64_t c = neg ? -(int64_t)q : (int64_t)q;
    double a;
    if (c <= (int64_t(1) << p.m)) {
#ifdef __CUDA_ARCH__
        // (double)c for c <= 2^24 without a conversion instruction
        const double iscale = __longlong_as_double((long long)(uint64_t(1023 - p.L) << 52));
        const double cf = __longlong_as_double((long long)(0x4330000000000000ull + (uint64_t)c)) - 4503599627370496.0;
        a = __dmul_rn(cf, iscale);
#else
        a = (double)c * std::ldexp(1.0, -p.L);
#endif
    } else {
        const int e0 = p.m - p.L;
        const int sh = 52 - p.m;
        const uint64_t bits = (uint64_t)(c - (int64_t(1) << p.m) + (int64_t(e0 + 1023) << p.m)) << sh;
#ifdef __CUDA_ARCH__
        a = __longlong_as_double((long long)bits);
#else
        std::memcpy(&a, &bits, 8);
#endif
    }
    return neg ? -a : a;
}

__host__ __device__ inline float dequantize(int32_t q, CodecParams p, float) { return dequantize_f32(q, p); }
__host__ __device__ inline double dequantize(int32_t q, CodecParams p, double) { return dequantize_f64(q, p); }

// ---------------------------------------------------------------- fast paths
// The same maps with 32-bit integer work only and no branches, for the hot
// kernels.  For doubles they need m <= kFastMantissaF64: then the log-region
// rounding bit and the kept mantissa bits all lie in the high word of the
// double, so the low word never contributes; for m above that the kernels
// call quantize()/dequantize_f64().  Bit-identical to the statements above
// (the CPU oracle checks the device codes).
constexpr int kFastMantissaF64 = 19;

__host__ __device__ inline uint32_t hi_word(double x) {
#ifdef __CUDA_ARCH__
    return (uint32_t)__double2hiint(x);
#else
    uint64_t b;
    std::memcpy(&b, &x, 8);
    return (uint32_t)(b >> 32);
#endif
}
__host__ __device__ inline uint32_t lo_word(double x) {
#ifdef __CUDA_ARCH__
    return (uint32_t)__double2loint(x);
#else
    uint64_t b;
    std::memcpy(&b, &x, 8);
    return (uint32_t)b;
#endif
}
__host__ __device__ inline double from_words(uint32_t hi, uint32_t lo) {
#ifdef __CUDA_ARCH__
    return __hiloint2double((int)hi, (int)lo);
#else
    const uint64_t b = ((uint64_t)hi << 32) | lo;
    double x;
    std::memcpy(&x, &b, 8);
    return x;
#endif
}
__host__ __device__ inline uint32_t f32_bits(float x) {
#ifdef __CUDA_ARCH__
    return __float_as_uint(x);
#else
    uint32_t b;
    std::memcpy(&b, &x, 4);
    return b;
#endif
}
__host__ __device__ inline float f32_from(uint32_t b) {
#ifdef __CUDA_ARCH__
    return __uint_as_float(b);
#else
    float x;
    std::memcpy(&x, &b, 4);
    return x;
#endif
}

// m <= kFastMantissaF64.
__host__ __device__ inline int32_t quantize_fast(double x, CodecParams p) {
    const uint32_t hi = hi_word(x), ahi = hi & 0x7fffffffu;
    const int e0 = p.m - p.L;
    const uint32_t thr = uint32_t(e0 + 1023) << 20;
    // linear region: rint(|x| 2^L) appears in the low word of fma(|x|, 2^L, 2^52)
    const double a = from_words(ahi, lo_word(x));
    const double scale = from_words(uint32_t(p.L + 1023) << 20, 0u);
#ifdef __CUDA_ARCH__
    const double r = __fma_rn(a, scale, 4503599627370496.0);
#else
    const double r = std::fma(a, scale, 4503599627370496.0);
#endif
    const uint32_t c_lin = lo_word(r);
    // log region: round the high word to m mantissa bits (the rounding bit is
    // bit 19 - m of the high word)
    const int shh = 20 - p.m;
    const uint32_t c_log = ((ahi + (1u << (shh - 1))) >> shh) - (uint32_t(e0 + 1023) << p.m) + (1u << p.m);
    uint32_t c = ahi < thr ? c_lin : c_log;
    if (ahi >= thr && c > (uint32_t)kCodeLimit) c = (uint32_t)kCodeLimit;
    const uint32_t sgn = (uint32_t)((int32_t)hi >> 31);
    return (int32_t)((c ^ sgn) - sgn);
}

// m <= kFastMantissaF64.
__host__ __device__ inline double dequantize_fast(int32_t q, CodecParams p) {
    const uint32_t sgn = (uint32_t)(q >> 31);
    const uint32_t c = ((uint32_t)q ^ sgn) - sgn;
    // linear region: c in the low word of 2^(52-L) (1 + c 2^-52), minus 2^(52-L)
    const uint32_t ehi = uint32_t(1075 - p.L) << 20;
    const double lin = from_words(ehi, c) - from_words(ehi, 0u);
    // log region: the code is the high word of the value, shifted
    const int e0 = p.m - p.L;
    const uint32_t lhi = (c + (uint32_t(e0 + 1023) << p.m) - (1u << p.m)) << (20 - p.m);
    const double a = c <= (1u << p.m) ? lin : from_words(lhi, 0u);
    return from_words(hi_word(a) | (sgn & 0x80000000u), lo_word(a));
}

__host__ __device__ inline int32_t quantize_fast(float x, CodecParams p) {
    const uint32_t bits = f32_bits(x), abits = bits & 0x7fffffffu;
    const int e0 = p.m - p.L;
    const uint32_t thr = uint32_t(e0 + 127) << 23;
    const float scale = f32_from(uint32_t(p.L + 127) << 23);
#ifdef __CUDA_ARCH__
    const float r = __fmaf_rn(f32_from(abits), scale, 8388608.0f);
#else
    const float r = std::fma(f32_from(abits), scale, 8388608.0f);
#endif
    const uint32_t c_lin = f32_bits(r) - 0x4b000000u;
    const int sh = 23 - p.m;
    const uint32_t half = sh > 0 ? (1u << (sh - 1)) : 0u;
    const uint32_t c_log = ((abits + half) >> sh) - (uint32_t(e0 + 127) << p.m) + (1u << p.m);
    uint32_t c = abits < thr ? c_lin : c_log;
    if (abits >= thr && c > (uint32_t)kCodeLimit) c = (uint32_t)kCodeLimit;
    const uint32_t sgn = (uint32_t)((int32_t)bits >> 31);
    return (int32_t)((c ^ sgn) - sgn);
}

__host__ __device__ inline float dequantize_fast_f32(int32_t q, CodecParams p) {
    const uint32_t sgn = (uint32_t)(q >> 31);
    const uint32_t c = ((uint32_t)q ^ sgn) - sgn;
    const uint32_t eb = uint32_t(150 - p.L) << 23;
    const float lin = f32_from(eb + c) - f32_from(eb);
    const int e0 = p.m - p.L;
    const uint32_t lb = (c + (uint32_t(e0 + 127) << p.m) - (1u << p.m)) << (23 - p.m);
    const float a = c <= (1u << p.m) ? lin : f32_from(lb);
    return f32_from(f32_bits(a) | (sgn & 0x80000000u));
}

// Dispatch on the precision and on the mantissa width (uniform per launch).
__host__ __device__ inline int32_t quantize_hot(double x, CodecParams p) {
    return p.m <= kFastMantissaF64 ? quantize_fast(x, p) : quantize(x, p);
}
__host__ __device__ inline int32_t quantize_hot(float x, CodecParams p) { return quantize_fast(x, p); }
__host__ __device__ inline double dequantize_hot(int32_t q, CodecParams p, double) {
    return p.m <= kFastMantissaF64 ? dequantize_fast(q, p) : dequantize_f64(q, p);
}
__host__ __device__ inline float dequantize_hot(int32_t q, CodecParams p, float) { return dequantize_fast_f32(q, p); }

// Quantiser parameters from the error bounds; false when eps_rel is out of
// range.  L is clamped so that 2^L, 2^-L and 2^e0 are normal numbers.
inline bool codec_params(bool f64, double eps_rel, double eps_abs, CodecParams *out) {
    if (!(eps_rel > 0.0) || !(eps_rel < 1.0)) return false;
    int m = (int)std::ceil(-std::log2(eps_rel));
    if (m < 1) m = 1;
    if (m > 24) return false;
    if (!f64 && m > 23) m = 23;
    const int bias = f64 ? 1023 : 127;
    int L = eps_abs > 0.0 ? (int)std::ceil(-std::log2(eps_abs)) : bias - 1;
    if (L > bias - 1) L = bias - 1;
    if (L < m - (bias - 2)) L = m - (bias - 2);
    out->m = m;
    out->L = L;
    return true;
}

}  // namespace qs
