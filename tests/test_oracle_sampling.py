"""The sampling oracle (oracle/sampling_oracle.cpp), pinned on the CPU.

sampling_blockwise (src/cppsim/compressed_state.hpp:1600-1681) draws from
libstdc++'s std::mt19937_64.  The engine is restated here in Python from its
published definition (Matsumoto-Nishimura 64-bit Mersenne Twister) and
pinned by the C++ standard's known answer (the 10000th output of a
default-seeded std::mt19937_64 is 9981545732273789042).  With one block the
shot split draws nothing, so the oracle's multiset of samples must equal
lower_bound(cdf, u * mass) over the Python engine's uniforms, u = g / 2^64
(std::generate_canonical with a 64-bit engine).  The order is std::shuffle's
and is compared only as a multiset.
"""
import math

import numpy as np
import pytest

from oracle import sampling

_MASK = (1 << 64) - 1


class MT19937_64:
    N, M = 312, 156
    A = 0xB5026F5AA96619E9
    UPPER, LOWER = 0xFFFFFFFF80000000, 0x7FFFFFFF

    def __init__(self, seed: int = 5489):
        self.mt = [0] * self.N
        self.mt[0] = seed & _MASK
        for i in range(1, self.N):
            prev = self.mt[i - 1]
            self.mt[i] = (6364136223846793005 * (prev ^ (prev >> 62)) + i) & _MASK
        self.i = self.N

    def _twist(self):
        mt = self.mt
        for i in range(self.N):
            x = (mt[i] & self.UPPER) | (mt[(i + 1) % self.N] & self.LOWER)
            xa = x >> 1
            if x & 1:
                xa ^= self.A
            mt[i] = mt[(i + self.M) % self.N] ^ xa
        self.i = 0

    def __call__(self) -> int:
        if self.i >= self.N:
            self._twist()
        y = self.mt[self.i]
        self.i += 1
        y ^= (y >> 29) & 0x5555555555555555
        y ^= (y << 17) & 0x71D67FFFEDA60000
        y ^= (y << 37) & 0xFFF7EEE000000000
        y ^= y >> 43
        return y & _MASK


def test_mt19937_64_known_answer():
    g = MT19937_64()
    for _ in range(9999):
        g()
    assert g() == 9981545732273789042


def _uniform(g: MT19937_64) -> float:
    u = float(g()) / 2.0 ** 64
    return u if u < 1.0 else math.nextafter(1.0, 0.0)


@pytest.mark.parametrize("n,seed,shots", [(8, 3, 500), (10, 2 ** 32 - 1, 3000)])
def test_single_block_draws_match_restated_engine(n, seed, shots):
    rng = np.random.default_rng(n)
    v = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    v[rng.integers(0, 1 << n, size=20)] = 0          # zero-mass amplitudes are never drawn
    got = sampling.sampling_blockwise(v, n, shots, seed)
    cdf = np.cumsum(v.real * v.real + v.imag * v.imag)   # sequential sums, as std::norm in a loop
    g = MT19937_64((seed + 1) & 0xFFFFFFFF)
    r = np.array([_uniform(g) * cdf[-1] for _ in range(shots)])
    want = np.minimum(np.searchsorted(cdf, r, side="left"), v.size - 1)
    assert sorted(got) == sorted(int(x) for x in want)
    assert all(v[x] != 0 for x in got)


def test_block_split_statistics_and_determinism():
    rng = np.random.default_rng(4)
    n, B = 12, 5
    v = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    v *= np.repeat(rng.exponential(size=1 << (n - B)), 1 << B)   # uneven block masses
    a = sampling.sampling_blockwise(v, B, 100000, 11)
    assert a == sampling.sampling_blockwise(v, B, 100000, 11)
    assert a != sampling.sampling_blockwise(v, B, 100000, 12)
    assert len(a) == 100000 and min(a) >= 0 and max(a) < v.size
    p = np.abs(v) ** 2
    p /= p.sum()
    # per-block counts: the binomial split must follow the block masses
    pb = p.reshape(-1, 1 << B).sum(axis=1)
    cb = np.bincount(np.asarray(a) >> B, minlength=pb.size)
    e = pb * len(a)
    keep = e > 5
    chi = float(((cb[keep] - e[keep]) ** 2 / e[keep]).sum())
    k = int(keep.sum())
    assert chi < k + 6 * math.sqrt(2 * k), (chi, k)


def test_unstored_blocks_and_errors():
    n, B = 8, 4
    v = np.ones(1 << n, dtype=np.complex128)
    stored = np.zeros(1 << (n - B), dtype=np.uint8)
    stored[[2, 7]] = 1
    got = sampling.sampling_blockwise(v, B, 4000, 5, stored=stored)
    assert set(x >> B for x in got) == {2, 7}
    assert sampling.sampling_blockwise(v, B, 0, 5) == []
    e = np.zeros(1 << n, dtype=np.complex128)
    e[77] = 1j
    assert sampling.sampling_blockwise(e, B, 50, 1) == [77] * 50
    with pytest.raises(ValueError):
        sampling.sampling_blockwise(np.zeros(1 << n, dtype=np.complex128), B, 10, 1)
    for bad in (np.nan, np.inf):
        w = v.copy()
        w[3] = bad
        with pytest.raises(ValueError):
            sampling.sampling_blockwise(w, B, 10, 1)
    with pytest.raises(ValueError):
        sampling.sampling_blockwise(v, B, 10, 1, stored=np.zeros(1 << (n - B), dtype=np.uint8))
