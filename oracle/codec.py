"""ORACLE (test infrastructure only): CPU statement of the block codec and an
emulation of the reference's lossy map.

* The block codec (codec_oracle.c, built into oracle/build/liboracle.so):
  quantiser params, value round trips, chunk encode/decode with the
  32-lane frame-of-reference layout.  The device codec must match it bit for
  bit.
* ref_compander_roundtrip: the reference's compander
  (src/cppsim/compand_kernel.cuh:5-30, compand_bitcomp_pipeline.cuh:14-62)
  with nvCOMP Bitcomp's lossy quantiser modelled as round-to-nearest at step
  delta = log1p(eps_rel).  nvCOMP 5.1.0.21 is a closed binary that is not
  present here; its lossless stage does not change values, so this model is
  what the reference's fidelity depends on.  It is an assumption, stated as
  such, not a pinned reproduction.
"""
from __future__ import annotations

import ctypes as ct
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "build", "liboracle.so")

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            env = dict(os.environ)
            subprocess.run(["make", "-C", HERE, "oracle"], check=True, capture_output=True, env=env)
        L = ct.CDLL(LIB_PATH)
        P = ct.c_void_p
        I32 = ct.c_int32
        L.qsor_codec_params.argtypes = [ct.c_int, ct.c_double, ct.c_double, ct.POINTER(I32), ct.POINTER(I32)]
        L.qsor_codec_params.restype = ct.c_int
        L.qsor_payload_bytes.argtypes = [I32, ct.c_uint32]
        L.qsor_payload_bytes.restype = ct.c_uint64
        L.qsor_quantize_f32.argtypes = [ct.c_float, I32, I32]
        L.qsor_quantize_f32.restype = I32
        L.qsor_quantize_f64.argtypes = [ct.c_double, I32, I32]
        L.qsor_quantize_f64.restype = I32
        L.qsor_dequantize_f32.argtypes = [I32, I32, I32]
        L.qsor_dequantize_f32.restype = ct.c_float
        L.qsor_dequantize_f64.argtypes = [I32, I32, I32]
        L.qsor_dequantize_f64.restype = ct.c_double
        for nm in ("qsor_encode_chunk_f32", "qsor_encode_chunk_f64"):
            f = getattr(L, nm)
            f.argtypes = [P, I32, I32, I32, P, P, ct.POINTER(I32), ct.POINTER(ct.c_uint32)]
            f.restype = ct.c_uint64
        for nm in ("qsor_decode_chunk_f32", "qsor_decode_chunk_f64"):
            f = getattr(L, nm)
            f.argtypes = [P, I32, I32, ct.c_uint32, I32, I32, P, P]
        L.qsor_roundtrip_f64.argtypes = [P, ct.c_uint64, I32, I32, P]
        L.qsor_roundtrip_f32.argtypes = [P, ct.c_uint64, I32, I32, P]
        L.qsor_sampling_blockwise.argtypes = [P, ct.c_uint32, ct.c_uint32, P, ct.c_uint32, ct.c_uint32, P]
        L.qsor_sampling_blockwise.restype = ct.c_int
        _lib = L
    return _lib


def params(f64: bool, eps_rel: float, eps_abs: float):
    m, L = ct.c_int32(), ct.c_int32()
    if lib().qsor_codec_params(1 if f64 else 0, eps_rel, eps_abs, ct.byref(m), ct.byref(L)) != 0:
        raise ValueError("eps_rel out of range")
    return m.value, L.value


def payload_bytes(C: int, width: int) -> int:
    return int(lib().qsor_payload_bytes(C, width))


def quantize(x: np.ndarray, m: int, L: int) -> np.ndarray:
    x = np.ascontiguousarray(x)
    f = lib().qsor_quantize_f64 if x.dtype == np.float64 else lib().qsor_quantize_f32
    return np.array([f(float(v), m, L) for v in x.reshape(-1)], dtype=np.int32).reshape(x.shape)


def roundtrip(x: np.ndarray, m: int, L: int) -> np.ndarray:
    """Quantise and dequantise every element (real arrays, f32 or f64)."""
    x = np.ascontiguousarray(x)
    out = np.empty_like(x)
    if x.dtype == np.float64:
        lib().qsor_roundtrip_f64(x.ctypes.data, x.size, m, L, out.ctypes.data)
    elif x.dtype == np.float32:
        lib().qsor_roundtrip_f32(x.ctypes.data, x.size, m, L, out.ctypes.data)
    else:
        raise TypeError(x.dtype)
    return out


def roundtrip_complex(v: np.ndarray, m: int, L: int, f64: bool = True) -> np.ndarray:
    v = np.ascontiguousarray(v, dtype=np.complex128)
    if f64:
        r = roundtrip(v.view(np.float64), m, L)
        return r.view(np.complex128)
    r = roundtrip(v.astype(np.complex64).view(np.float32), m, L)
    return r.view(np.complex64).astype(np.complex128)


def encode_chunk(vals: np.ndarray, C: int, m: int, L: int):
    """vals: 2^(C+1) real components (f32 or f64).  -> (words, base, width)."""
    vals = np.ascontiguousarray(vals)
    n = 2 << C
    assert vals.size == n
    words = np.zeros(n, dtype=np.uint32)
    scratch = np.zeros(n, dtype=np.int32)
    base, width = ct.c_int32(), ct.c_uint32()
    f = lib().qsor_encode_chunk_f64 if vals.dtype == np.float64 else lib().qsor_encode_chunk_f32
    nbytes = f(vals.ctypes.data, C, m, L, scratch.ctypes.data, words.ctypes.data, ct.byref(base), ct.byref(width))
    return words[: nbytes // 4].copy(), base.value, width.value


def decode_chunk(words: np.ndarray, C: int, base: int, width: int, m: int, L: int, f64: bool) -> np.ndarray:
    n = 2 << C
    w = np.zeros(n, dtype=np.uint32)
    w[: words.size] = words
    scratch = np.zeros(n, dtype=np.int32)
    out = np.zeros(n, dtype=np.float64 if f64 else np.float32)
    f = lib().qsor_decode_chunk_f64 if f64 else lib().qsor_decode_chunk_f32
    f(w.ctypes.data, C, base, width, m, L, scratch.ctypes.data, out.ctypes.data)
    return out


def ref_compander_roundtrip(x: np.ndarray, eps_rel: float, eps_abs: float) -> np.ndarray:
    """The reference's pointwise lossy map on real components (FP64)."""
    x = np.asarray(x, dtype=np.float64)
    gamma = 1.0 - 2.0 * eps_rel
    tau = gamma * (eps_abs / eps_rel) if eps_abs > 0 else 0.0
    delta = np.log1p(eps_rel)
    v = x * gamma
    sgn = np.where(v < 0.0, -1.0, 1.0)
    with np.errstate(divide="ignore"):
        y = sgn * np.log(np.abs(v) + tau)
    yq = np.round(y / delta) * delta
    s2 = np.where(yq < 0.0, 1.0, -1.0)
    a = np.exp(s2 * yq) - tau
    a = a / gamma
    a = np.clip(a, 0.0, 1.0)
    return s2 * a


def ref_compander_roundtrip_complex(v: np.ndarray, eps_rel: float, eps_abs: float) -> np.ndarray:
    v = np.asarray(v, dtype=np.complex128)
    return ref_compander_roundtrip(v.real, eps_rel, eps_abs) + 1j * ref_compander_roundtrip(v.imag, eps_rel, eps_abs)
