"""The library's site decode (mag_b200/csrc/lattice.cuh) built for the host with g++:
its multiply-shift division by the chain extents against plain division, for
divisors 2..4096 and large ones on dividends across [0, 2^31), and every site of a
set of lattice shapes; on those shapes the neighbour indices of nb and nb_sel at steps
-2..2 along every direction (tests/cpp/decode_check.cpp)."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "decode_check.cpp")
BIN = os.path.join(ROOT, "tests", "cpp", "_build", "decode_check")
CUDA_INCLUDE = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include")


def test_site_decode_matches_plain_division():
    os.makedirs(os.path.dirname(BIN), exist_ok=True)
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", CUDA_INCLUDE, SRC, "-o", BIN], check=True,
                   capture_output=True, text=True)
    out = subprocess.run([BIN], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.strip() == "ok"
