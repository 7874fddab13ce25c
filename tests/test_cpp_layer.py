"""The C++ class layer (include/dyphur_b200.hpp): compiled with g++ against the
library, it runs the reference's frame loop and must reproduce the golden
hashes the reference build wrote."""
import os
import subprocess

import pytest

from test_oracle_pins import _golden_cases

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "frame_loop.cpp")
LIB_DIR = os.path.join(ROOT, "dyphur_b200", "lib")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


@pytest.fixture(scope="module")
def frame_loop(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("cpp") / "frame_loop")
    cmd = ["g++", "-std=c++20", "-O2", SRC, "-o", exe, f"-I{CUDA}/include", f"-L{LIB_DIR}", "-ldyphur_b200",
           f"-Wl,-rpath,{LIB_DIR}", f"-L{CUDA}/lib64", "-lcudart"]
    subprocess.run(cmd, check=True)
    return exe


def test_cpp_layer_compiles(frame_loop):
    assert os.path.exists(frame_loop)


@pytest.mark.gpu
@pytest.mark.parametrize("name,args", [
    ("determinism_8_f20", ["1", "2", "2", "2", "1.0", "0.0", "0", "20", "0"]),
    ("blocks_1025_f300_reference", ["0", "8", "16", "8", "0.85", "0.01", "1", "300", "0"]),
    ("blocks_1025_f300_serial", ["0", "8", "16", "8", "0.85", "0.01", "1", "300", "1"]),
])
def test_cpp_frame_loop_matches_golden(frame_loop, name, args):
    g = _golden_cases()[name]
    out = subprocess.run([frame_loop] + args, check=True, capture_output=True, text=True).stdout.split()
    assert out[0] == "hash" and out[1] == g["hash"], out
    assert int(out[3]) == g["pairs"] and int(out[5]) == g["contacts"], out
