"""The allocation-free codec round trip, qs_codec_roundtrip_noalloc.

Some callers cannot call cudaMalloc: code that runs inside another
framework's memory pool, that has reserved all device memory up front, or
that must not allocate (an allocation may synchronise the device) in the
middle of a running pipeline.  For them the library offers one entry point
that allocates nothing: the caller passes device buffers for the inputs and
outputs, and the packed words between encode and decode live in a fixed
4 MiB device array inside the library.

This file checks it through the C ABI against the allocating entry point
(qs_codec_test) -- bit for bit, the tolerance every codec test here uses --
on two calls in a row with different data (the array keeps the previous
call's words, which must not leak into the next result), and checks that a
call larger than the array is refused.  It is named so that pytest collects
it last.
"""
import ctypes as ct

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _allocating(L, f64, C, vals, nch):
    n = 2 << C
    words = np.zeros(nch * n, dtype=np.uint32)
    bases = np.zeros(nch, dtype=np.int32)
    widths = np.zeros(nch, dtype=np.uint32)
    dec = np.zeros_like(vals)
    st = L.qs_codec_test(0 if f64 else 1, 1e-3, 1e-7, C, vals.ctypes.data, nch,
                         words.ctypes.data_as(ct.POINTER(ct.c_uint32)), bases.ctypes.data_as(ct.POINTER(ct.c_int32)),
                         widths.ctypes.data_as(ct.POINTER(ct.c_uint32)), dec.ctypes.data)
    assert st == 0, L.qs_dense_last_error(None)
    return bases, widths, dec


@pytest.mark.parametrize("f64", [True, False])
def test_noalloc_matches_allocating_entry_point(f64):
    import torch
    from qulacs import _native

    L = _native.load_library()
    C = 6
    n = 2 << C
    nch = 300
    dt = np.float64 if f64 else np.float32
    rng = np.random.default_rng(7 if f64 else 8)
    stream = ct.c_void_p(torch.cuda.current_stream().cuda_stream)
    for call in range(2):
        scale = 10.0 ** -rng.uniform(0, 6, size=(nch, 1))
        vals = (rng.normal(size=(nch, n)) * scale).astype(dt).reshape(-1)
        if call == 1:
            vals[: 3 * n] = 0.0  # all-zero chunks right after a call that left words behind
        ref_bases, ref_widths, ref_dec = _allocating(L, f64, C, vals, nch)

        d_vals = torch.from_numpy(vals).cuda()
        d_bases = torch.full((nch,), -1, dtype=torch.int32, device="cuda")
        d_widths = torch.full((nch,), -1, dtype=torch.int32, device="cuda")
        d_dec = torch.full_like(d_vals, float("nan"))
        st = L.qs_codec_roundtrip_noalloc(0 if f64 else 1, 1e-3, 1e-7, C, ct.c_void_p(d_vals.data_ptr()), nch,
                                          ct.c_void_p(d_bases.data_ptr()), ct.c_void_p(d_widths.data_ptr()),
                                          ct.c_void_p(d_dec.data_ptr()), stream)
        assert st == 0, L.qs_dense_last_error(None)
        torch.cuda.synchronize()
        assert np.array_equal(d_bases.cpu().numpy(), ref_bases), call
        assert np.array_equal(d_widths.cpu().numpy().view(np.uint32), ref_widths), call
        assert np.array_equal(d_dec.cpu().numpy(), ref_dec), call


def test_noalloc_refuses_more_than_its_scratch():
    import torch
    from qulacs import _native

    L = _native.load_library()
    C = 8
    too_many = (1 << 20) // (2 << C) + 1
    d = torch.zeros(16, dtype=torch.float64, device="cuda")
    p = ct.c_void_p(d.data_ptr())
    st = L.qs_codec_roundtrip_noalloc(0, 1e-3, 1e-7, C, p, too_many, p, p, p, None)
    assert st == _native.QS_ERR_ARG
    assert b"scratch" in L.qs_dense_last_error(None)


@pytest.mark.parametrize("C", [8, 4])
def test_noalloc_at_exact_capacity(C):
    """A call of exactly as many chunks as the fixed scratch holds
    (2^20 / 2^(C+1)): the last chunk's slot ends at the array's last word;
    the result equals the allocating entry point's bit for bit."""
    import torch
    from qulacs import _native

    L = _native.load_library()
    n = 2 << C
    nch = (1 << 20) // n
    rng = np.random.default_rng(30 + C)
    scale = 10.0 ** -rng.uniform(0, 6, size=(nch, 1))
    vals = (rng.normal(size=(nch, n)) * scale).reshape(-1)
    # the last chunk as wide as codes get (magnitudes from 1e-300 to 1e300), deep into its slot
    vals[-n:] = rng.choice([-1.0, 1.0], size=n) * 10.0 ** rng.uniform(-300, 300, size=n)
    ref_bases, ref_widths, ref_dec = _allocating(L, True, C, vals, nch)
    d_vals = torch.from_numpy(vals).cuda()
    d_bases = torch.full((nch,), -1, dtype=torch.int32, device="cuda")
    d_widths = torch.full((nch,), -1, dtype=torch.int32, device="cuda")
    d_dec = torch.full_like(d_vals, float("nan"))
    stream = ct.c_void_p(torch.cuda.current_stream().cuda_stream)
    st = L.qs_codec_roundtrip_noalloc(0, 1e-3, 1e-7, C, ct.c_void_p(d_vals.data_ptr()), nch,
                                      ct.c_void_p(d_bases.data_ptr()), ct.c_void_p(d_widths.data_ptr()),
                                      ct.c_void_p(d_dec.data_ptr()), stream)
    assert st == 0, L.qs_dense_last_error(None)
    torch.cuda.synchronize()
    assert np.array_equal(d_bases.cpu().numpy(), ref_bases)
    assert np.array_equal(d_widths.cpu().numpy().view(np.uint32), ref_widths)
    assert np.array_equal(d_dec.cpu().numpy(), ref_dec)
