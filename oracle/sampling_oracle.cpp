// ORACLE / TEST INFRASTRUCTURE ONLY -- the checker of the device sampling
// path; never linked by the product.
//
// CPU statement of CompressedQuantumState::sampling_blockwise
// (src/cppsim/compressed_state.hpp:1600-1681) for one rank, over a dense
// decoded vector (interleaved re, im) instead of decompressed blocks:
//   * block mass = sequential sum over the block of std::norm(a), skipped
//     (left 0) for blocks that are not stored (:1613-1620);
//   * total = sequential sum of the masses; not finite or not positive is an
//     error, returned as -1 (:1627-1633);
//   * shots split over blocks in order with std::binomial_distribution on
//     std::mt19937_64(seed), the last block taking the remainder
//     (:1635-1643);
//   * per block with shots: its cdf, draws uniform(0,1) * acc from
//     std::mt19937_64(seed + 1) (rank 0), std::lower_bound, clamped to the
//     block (:1644-1663);
//   * std::shuffle of the indices with the first generator (:1677-1678).
// The generators and distributions are libstdc++'s, as in the reference.
// Built with -ffp-contract=off: x*x + y*y is rounded after each operation.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <random>
#include <vector>

extern "C" int qsor_sampling_blockwise(const double *amps, uint32_t n, uint32_t B, const uint8_t *stored,
                                       uint32_t n_shots, uint32_t seed, uint64_t *out) {
    const uint64_t namps_per_block = uint64_t(1) << B;
    const uint64_t nblocks = uint64_t(1) << (n - B);
    const std::complex<double> *v = reinterpret_cast<const std::complex<double> *>(amps);
    std::vector<double> mass(nblocks, 0.0);
    for (uint64_t b = 0; b < nblocks; b++) {
        if (stored && !stored[b]) continue;
        double m = 0.0;
        for (uint64_t j = 0; j < namps_per_block; j++) m += std::norm(v[b * namps_per_block + j]);
        mass[b] = m;
    }
    double total = 0.0;
    for (double m : mass) total += m;
    if (!(total > 0.0) || !std::isfinite(total)) return -1;
    std::mt19937_64 rng(seed);
    std::vector<uint32_t> shots(mass.size(), 0);
    uint32_t left = n_shots;
    double rest = total;
    for (size_t g = 0; g < mass.size() && left > 0; g++) {
        double p = rest > 0 ? std::min(1.0, mass[g] / rest) : 0.0;
        std::binomial_distribution<uint32_t> bin(left, p);
        uint32_t k = (g + 1 == mass.size()) ? left : bin(rng);
        shots[g] = k;
        left -= k;
        rest -= mass[g];
    }
    std::vector<uint64_t> mine;
    std::mt19937_64 rng_local(static_cast<uint32_t>(seed + 1u));
    std::uniform_real_distribution<double> uni(0.0, 1.0);
    std::vector<double> cdf(namps_per_block);
    for (uint64_t b = 0; b < nblocks; b++) {
        const uint32_t k = shots[b];
        if (k == 0) continue;
        double acc = 0.0;
        for (uint64_t j = 0; j < namps_per_block; j++) {
            acc += std::norm(v[b * namps_per_block + j]);
            cdf[j] = acc;
        }
        const uint64_t base = b * namps_per_block;
        for (uint32_t s = 0; s < k; s++) {
            const double r = uni(rng_local) * acc;
            uint64_t j = std::lower_bound(cdf.begin(), cdf.end(), r) - cdf.begin();
            if (j >= namps_per_block) j = namps_per_block - 1;
            mine.push_back(base + j);
        }
    }
    std::shuffle(mine.begin(), mine.end(), rng);
    std::copy(mine.begin(), mine.end(), out);
    return 0;
}
