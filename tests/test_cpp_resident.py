"""Build and run the C++ resident Session tests: over the deferred CPU transport
(no GPU) and over the B200 driver from make_cuda_session (GPU)."""
import os
import subprocess

import pytest

from ntt_gpu_b200 import build

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
OUT = os.path.join(ROOT, "tests", "cpp", "_bin")


def compile_test(name, extra):
    os.makedirs(OUT, exist_ok=True)
    exe = os.path.join(OUT, name)
    src = os.path.join(HERE, "cpp", name + ".cpp")
    oracle_dir = os.path.join(ROOT, "oracle")
    cmd = ["g++", "-std=c++20", "-O1", "-Wall", "-Wextra", "-I", os.path.join(ROOT, "ntt_gpu_b200", "host", "include"),
           src, *extra, "-L", oracle_dir, "-loracle", f"-Wl,-rpath,{oracle_dir}", "-o", exe]
    subprocess.run(cmd, check=True)
    return exe


def test_resident_runtime_over_cpu_transport(orc):
    exe = compile_test("resident_tests", [os.path.join(ROOT, "ntt_gpu_b200", "host", "src", "session.cpp")])
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr + r.stdout
    assert "RESIDENT HOST CHECKS PASSED" in r.stdout


@pytest.mark.gpu
def test_resident_session_over_b200_driver(orc, lib):
    build.build()
    exe = compile_test("gpu_session_tests", ["-L", build.LIB_DIR, "-lntt_b200_host", "-lntt_b200",
                                             f"-Wl,-rpath,{build.LIB_DIR}"])
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr + r.stdout
    assert "B200 SESSION CHECKS PASSED" in r.stdout
