// CPU check that the branch-free 32-bit codec paths of codec.cuh (used by the
// device kernels) give the same codes and decoded values, bit for bit, as the
// statement of the quantiser in the same header.  Built and run by
// tests/test_codec_fast.py with the host compiler.
#include "codec.cuh"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>

using namespace qs;

int main(int argc, char **argv) {
    const long iters = argc > 1 ? std::atol(argv[1]) : 200000;
    std::mt19937_64 rng(1);
    long bad = 0, n = 0;
    const double eps_rels[] = {1e-3, 1e-2, 0.3, 2e-5, 1.0 / (1 << 19), 1.0 / (1 << 18), 1e-1, 1.0 / (1 << 23)};
    const double eps_abss[] = {1e-7, 1e-4, 1e-13, 0.0, 1e-300, 1.0, 0.5};
    for (double er : eps_rels)
        for (double ea : eps_abss)
            for (int f64 = 0; f64 < 2; ++f64) {
                CodecParams p;
                if (!codec_params(f64, er, ea, &p)) continue;
                if (f64 && p.m > kFastMantissaF64) continue;
                for (long it = 0; it < iters; ++it) {
                    double mag = std::ldexp(1.0, (int)(rng() % 120) - 100) * (1.0 + (rng() % 1000000) / 1e6);
                    if (it % 97 == 0) mag = std::ldexp(1.0, p.m - p.L) * (1 + ((int)(rng() % 5) - 2) * 1e-16);
                    if (it % 101 == 0) mag = 0.0;
                    if (it % 103 == 0) mag = std::ldexp((double)(rng() % (1 << 20)), -p.L - 1);
                    const double x = (rng() & 1) ? -mag : mag;
                    ++n;
                    if (f64) {
                        const int32_t a = quantize(x, p), b = quantize_fast(x, p);
                        const double da = dequantize_f64(a, p), db = dequantize_fast(a, p);
                        if (a != b || std::memcmp(&da, &db, 8)) {
                            if (bad < 10) printf("f64 m=%d L=%d x=%a q=%d fast=%d\n", p.m, p.L, x, a, b);
                            ++bad;
                        }
                    } else {
                        const float xf = (float)x;
                        if (!std::isfinite(xf)) continue;
                        const int32_t a = quantize(xf, p), b = quantize_fast(xf, p);
                        const float da = dequantize_f32(a, p), db = dequantize_fast_f32(a, p);
                        if (a != b || std::memcmp(&da, &db, 4)) {
                            if (bad < 10) printf("f32 m=%d L=%d x=%a q=%d fast=%d\n", p.m, p.L, (double)xf, a, b);
                            ++bad;
                        }
                    }
                }
                // every code that a finite value can produce decodes identically
                const int32_t qmax = f64 ? quantize(1.7976931348623157e308, p) : quantize(3.4028234e38f, p);
                for (int32_t q = -(1 << 16); q <= (1 << 16); ++q) {
                    if (q > qmax || -q > qmax) continue;
                    ++n;
                    if (f64) {
                        const double da = dequantize_f64(q, p), db = dequantize_fast(q, p);
                        if (std::memcmp(&da, &db, 8)) ++bad;
                    } else {
                        const float da = dequantize_f32(q, p), db = dequantize_fast_f32(q, p);
                        if (std::memcmp(&da, &db, 4)) ++bad;
                    }
                }
            }
    printf("checked %ld values, %ld mismatches\n", n, bad);
    return bad != 0;
}
