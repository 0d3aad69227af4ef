/*
 * ORACLE / TEST INFRASTRUCTURE ONLY -- the CPU statement of the block codec.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
 * this library (built by oracle/Makefile into oracle/build/liboracle.so).
 * The product's CUDA codec (csrc/codec.cuh) must produce the same integer
 * codes and the same packed words as this file for the same FP inputs; the
 * quantiser is integer/exact-FP arithmetic only (no transcendental), so the
 * two agree bit for bit by construction, and the tests check that they do.
 *
 * What the codec replaces in the reference: the log compander plus nvCOMP
 * Bitcomp lossy FP64 (src/cppsim/compand_kernel.cuh:5-30,
 * src/cppsim/compand_bitcomp_pipeline.cuh:14-62).  With gamma = 1-2*eps_rel,
 * tau' = gamma*eps_abs/eps_rel and a quantiser step delta = log1p(eps_rel) in
 * the log domain, that pipeline bounds each real component by
 *     |xhat - x| <= (eps_rel*|x| + eps_abs) / 2      (round-to-nearest step).
 * This codec meets the same bound without log/exp:
 *   - |x| <  2^e0 : linear code  c = rint(|x| * 2^L),  2^-L <= eps_abs,
 *                    error <= 2^-(L+1) <= eps_abs/2
 *   - |x| >= 2^e0 : the IEEE bit pattern of |x| rounded to m mantissa bits,
 *                    2^-m <= eps_rel, relative error <= 2^-(m+1) <= eps_rel/2
 * with e0 = m - L, the binade in which both steps are equal, so the code is
 * continuous and monotone in |x|: c(2^e0) = 2^m.  The signed code is
 * q = sign ? -c : c.
 *
 * Chunk format (one chunk = 2^C amplitudes = N = 2^(C+1) real components,
 * interleaved re, im): frame of reference over the chunk, base = min q,
 * width w = bit length of (max q - min q); u = q - base is packed in w bits
 * with a 32-lane vertical layout: stream l (0..31) holds components
 * l, l+32, l+64, ...; each stream is packed LSB first into R =
 * ceil((N/32)*w/32) 32-bit words, and word r of stream l is stored at
 * payload word index r*32 + l.  Payload bytes = 128*R (a multiple of 128).
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

#define QS_CODE_LIMIT ((int64_t)0x3fffffff)

/* Derive the quantiser parameters (m, L) from the error bounds.
 * is_f64 selects the storage type (0 = float, 1 = double).
 * Returns 0 on success, -1 when eps_rel is outside (2^-24, 1). */
int qsor_codec_params(int is_f64, double eps_rel, double eps_abs,
                      int32_t *m_out, int32_t *L_out) {
    if (!(eps_rel > 0.0) || !(eps_rel < 1.0)) return -1;
    int m = (int)ceil(-log2(eps_rel));
    if (m < 1) m = 1;
    if (m > 24) return -1;
    if (!is_f64 && m > 23) m = 23;
    /* L is kept in [m - (bias-2), bias-1] so that 2^L and 2^-L are normal
     * numbers of the storage type and 2^e0 (e0 = m - L) is a normal binade. */
    int bias = is_f64 ? 1023 : 127;
    int L;
    if (eps_abs > 0.0) {
        L = (int)ceil(-log2(eps_abs));
    } else {
        L = bias - 1; /* no absolute bound: linear region ends at 2^(m-bias+1) */
    }
    if (L > bias - 1) L = bias - 1;
    if (L < m - (bias - 2)) L = m - (bias - 2);
    *m_out = m;
    *L_out = L;
    return 0;
}

static inline uint32_t f32_bits(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }
static inline float bits_f32(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }
static inline uint64_t f64_bits(double f) { uint64_t u; memcpy(&u, &f, 8); return u; }
static inline double bits_f64(uint64_t u) { double f; memcpy(&f, &u, 8); return f; }

int32_t qsor_quantize_f32(float x, int32_t m, int32_t L) {
    uint32_t bits = f32_bits(x);
    uint32_t abits = bits & 0x7fffffffu;
    int neg = (bits >> 31) & 1;
    int e0 = m - L;
    uint32_t thr = (uint32_t)(e0 + 127) << 23;
    int64_t c;
    if (abits < thr) {
        float a = bits_f32(abits);
        float scaled = a * ldexpf(1.0f, L); /* exact: power-of-two scale, L <= 126 */
        c = (int64_t)nearbyintf(scaled);
    } else {
        int sh = 23 - m;
        uint32_t half = sh > 0 ? (1u << (sh - 1)) : 0u;
        int64_t r = (int64_t)(((uint64_t)abits + half) >> sh);
        c = r - ((int64_t)(e0 + 127) << m) + ((int64_t)1 << m);
    }
    if (c > QS_CODE_LIMIT) c = QS_CODE_LIMIT;
    return (int32_t)(neg ? -c : c);
}

float qsor_dequantize_f32(int32_t q, int32_t m, int32_t L) {
    int neg = q < 0;
    int64_t c = neg ? -(int64_t)q : (int64_t)q;
    float a;
    if (c <= ((int64_t)1 << m)) {
        a = (float)c * ldexpf(1.0f, -L);
    } else {
        int e0 = m - L;
        int sh = 23 - m;
        uint64_t bits = (uint64_t)(c - ((int64_t)1 << m) + ((int64_t)(e0 + 127) << m)) << sh;
        a = bits_f32((uint32_t)bits);
    }
    return neg ? -a : a;
}

int32_t qsor_quantize_f64(double x, int32_t m, int32_t L) {
    uint64_t bits = f64_bits(x);
    uint64_t abits = bits & 0x7fffffffffffffffull;
    int neg = (int)((bits >> 63) & 1);
    int e0 = m - L;
    uint64_t thr = (uint64_t)(e0 + 1023) << 52;
    int64_t c;
    if (abits < thr) {
        double a = bits_f64(abits);
        double scaled = a * ldexp(1.0, L);
        c = (int64_t)nearbyint(scaled);
    } else {
        int sh = 52 - m;
        uint64_t half = 1ull << (sh - 1);
        uint64_t r = (abits + half) >> sh;
        int64_t base = (int64_t)(e0 + 1023) << m;
        int64_t d = (int64_t)r - base;
        c = d + ((int64_t)1 << m);
    }
    if (c > QS_CODE_LIMIT) c = QS_CODE_LIMIT;
    return (int32_t)(neg ? -c : c);
}

double qsor_dequantize_f64(int32_t q, int32_t m, int32_t L) {
    int neg = q < 0;
    int64_t c = neg ? -(int64_t)q : (int64_t)q;
    double a;
    if (c <= ((int64_t)1 << m)) {
        a = (double)c * ldexp(1.0, -L);
    } else {
        int e0 = m - L;
        int sh = 52 - m;
        uint64_t bits = (uint64_t)(c - ((int64_t)1 << m) + ((int64_t)(e0 + 1023) << m)) << sh;
        a = bits_f64(bits);
    }
    return neg ? -a : a;
}

/* Number of payload bytes of a chunk of 2^C amplitudes at width w. */
uint64_t qsor_payload_bytes(int32_t C, uint32_t w) {
    uint64_t per_lane = ((uint64_t)1 << (C + 1)) / 32;
    uint64_t rows = (per_lane * w + 31) / 32;
    return rows * 128;
}

static void pack_codes(const int32_t *q, uint64_t n, int32_t *base_out,
                       uint32_t *width_out, uint32_t *words) {
    int32_t lo = q[0], hi = q[0];
    for (uint64_t i = 1; i < n; ++i) {
        if (q[i] < lo) lo = q[i];
        if (q[i] > hi) hi = q[i];
    }
    uint32_t range = (uint32_t)((int64_t)hi - (int64_t)lo);
    uint32_t w = 0;
    while (w < 32 && (range >> w) != 0) ++w;
    *base_out = lo;
    *width_out = w;
    if (w == 0) return;
    uint64_t per_lane = n / 32;
    uint64_t rows = (per_lane * w + 31) / 32;
    memset(words, 0, rows * 32 * sizeof(uint32_t));
    for (uint32_t l = 0; l < 32; ++l) {
        uint64_t bitpos = 0;
        for (uint64_t i = 0; i < per_lane; ++i) {
            uint64_t u = (uint64_t)(uint32_t)(q[l + 32 * i] - lo);
            uint64_t r = bitpos >> 5, s = bitpos & 31;
            words[r * 32 + l] |= (uint32_t)(u << s);
            if (s + w > 32) words[(r + 1) * 32 + l] |= (uint32_t)(u >> (32 - s));
            bitpos += w;
        }
    }
}

static void unpack_codes(const uint32_t *words, uint64_t n, int32_t base,
                         uint32_t w, int32_t *q) {
    if (w == 0) {
        for (uint64_t i = 0; i < n; ++i) q[i] = base;
        return;
    }
    uint64_t per_lane = n / 32;
    uint64_t mask = (w == 32) ? 0xffffffffull : ((1ull << w) - 1);
    for (uint32_t l = 0; l < 32; ++l) {
        uint64_t bitpos = 0;
        for (uint64_t i = 0; i < per_lane; ++i) {
            uint64_t r = bitpos >> 5, s = bitpos & 31;
            uint64_t v = words[r * 32 + l] >> s;
            if (s + w > 32) v |= (uint64_t)words[(r + 1) * 32 + l] << (32 - s);
            q[l + 32 * i] = (int32_t)((uint32_t)base + (uint32_t)(v & mask));
            bitpos += w;
        }
    }
}

/* Encode one chunk of 2^C complex amplitudes (2^(C+1) interleaved floats).
 * words must hold qsor_payload_bytes(C, 32) bytes; scratch holds 2^(C+1)
 * int32.  Returns the payload byte count. */
uint64_t qsor_encode_chunk_f32(const float *vals, int32_t C, int32_t m, int32_t L,
                               int32_t *scratch, uint32_t *words,
                               int32_t *base_out, uint32_t *width_out) {
    uint64_t n = (uint64_t)1 << (C + 1);
    for (uint64_t i = 0; i < n; ++i) scratch[i] = qsor_quantize_f32(vals[i], m, L);
    pack_codes(scratch, n, base_out, width_out, words);
    return qsor_payload_bytes(C, *width_out);
}

uint64_t qsor_encode_chunk_f64(const double *vals, int32_t C, int32_t m, int32_t L,
                               int32_t *scratch, uint32_t *words,
                               int32_t *base_out, uint32_t *width_out) {
    uint64_t n = (uint64_t)1 << (C + 1);
    for (uint64_t i = 0; i < n; ++i) scratch[i] = qsor_quantize_f64(vals[i], m, L);
    pack_codes(scratch, n, base_out, width_out, words);
    return qsor_payload_bytes(C, *width_out);
}

void qsor_decode_chunk_f32(const uint32_t *words, int32_t C, int32_t base,
                           uint32_t w, int32_t m, int32_t L, int32_t *scratch,
                           float *out) {
    uint64_t n = (uint64_t)1 << (C + 1);
    unpack_codes(words, n, base, w, scratch);
    for (uint64_t i = 0; i < n; ++i) out[i] = qsor_dequantize_f32(scratch[i], m, L);
}

void qsor_decode_chunk_f64(const uint32_t *words, int32_t C, int32_t base,
                           uint32_t w, int32_t m, int32_t L, int32_t *scratch,
                           double *out) {
    uint64_t n = (uint64_t)1 << (C + 1);
    unpack_codes(words, n, base, w, scratch);
    for (uint64_t i = 0; i < n; ++i) out[i] = qsor_dequantize_f64(scratch[i], m, L);
}

/* Round trip of a whole array through the quantiser only (no packing). */
void qsor_roundtrip_f64(const double *x, uint64_t n, int32_t m, int32_t L, double *out) {
    for (uint64_t i = 0; i < n; ++i) out[i] = qsor_dequantize_f64(qsor_quantize_f64(x[i], m, L), m, L);
}

void qsor_roundtrip_f32(const float *x, uint64_t n, int32_t m, int32_t L, float *out) {
    for (uint64_t i = 0; i < n; ++i) out[i] = qsor_dequantize_f32(qsor_quantize_f32(x[i], m, L), m, L);
}
