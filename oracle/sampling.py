"""ORACLE (test infrastructure only): block-wise sampling of the compressed
state, CompressedQuantumState::sampling_blockwise
(src/cppsim/compressed_state.hpp:1600-1681), stated in C++ in
sampling_oracle.cpp (built into oracle/build/liboracle.so) because the
reference's draws come from libstdc++'s std::mt19937_64,
std::binomial_distribution, std::uniform_real_distribution and std::shuffle.
"""
from __future__ import annotations

from typing import List, Optional

import numpy as np

from . import codec


def sampling_blockwise(vec: np.ndarray, block_log2: int, n_shots: int, seed: int,
                       stored: Optional[np.ndarray] = None) -> List[int]:
    """Samples of a dense complex128 vector split into blocks of
    2^block_log2 amplitudes; `stored` (uint8 per block, 1 = stored) marks
    the blocks the reference keeps (others count as zero mass).  Raises
    ValueError where the reference raises std::domain_error."""
    v = np.ascontiguousarray(vec, dtype=np.complex128)
    n = int(v.size).bit_length() - 1
    assert v.size == 1 << n and 0 <= block_log2 <= n
    st = None if stored is None else np.ascontiguousarray(stored, dtype=np.uint8)
    if st is not None:
        assert st.size == 1 << (n - block_log2)
    out = np.zeros(max(1, int(n_shots)), dtype=np.uint64)
    rc = codec.lib().qsor_sampling_blockwise(v.ctypes.data, n, int(block_log2),
                                             None if st is None else st.ctypes.data,
                                             int(n_shots), int(seed) & 0xFFFFFFFF, out.ctypes.data)
    if rc != 0:
        raise ValueError("CompressedQuantumState::sampling_blockwise: "
                         "state has no finite positive probability mass")
    return [int(x) for x in out[:n_shots]]
