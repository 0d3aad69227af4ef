"""The device kernels quantise with branch-free 32-bit paths (codec.cuh
quantize_fast / dequantize_fast*); on the CPU they must equal the statement
of the quantiser bit for bit over random values, region edges and every
producible code, for each precision and a range of error bounds."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "compression-based-state-vector-simulator_b200", "csrc")


def test_fast_codec_paths_match_statement(tmp_path):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no host C++ compiler")
    exe = tmp_path / "codec_fast_check"
    cmd = [gxx, "-O2", "-std=c++17", "-x", "c++", "-D__host__=", "-D__device__=", "-I", CSRC,
           "-I", "/usr/local/cuda/include", "-o", str(exe), os.path.join(HERE, "codec_fast_check.cpp")]
    env = dict(os.environ)
    env.pop("CXX", None)
    r = subprocess.run(cmd, capture_output=True, text=True, env=env)
    assert r.returncode == 0, r.stderr[-3000:]
    r = subprocess.run([str(exe), "60000"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:]
    assert "0 mismatches" in r.stdout
