"""The reference-side binding shown in INTEGRATION.md (section A) compiles
against the reference's own headers (when the reference tree is present) and
links against libntt_b200.so. No GPU."""
import os
import re
import subprocess

import pytest

from ntt_gpu_b200 import build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.environ.get("NTT_REFERENCE_TREE", "/root/reference")


def stub_source() -> str:
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    blocks = re.findall(r"```cpp\n(.*?)```", text, re.S)
    assert blocks, "INTEGRATION.md carries the binding"
    return blocks[0]


def test_binding_compiles_against_reference_headers(tmp_path):
    if not os.path.isdir(os.path.join(REF, "include", "ntt")):
        pytest.skip("reference tree not present")
    build.build()
    src = tmp_path / "resident_b200.cpp"
    src.write_text(stub_source())
    obj = tmp_path / "resident_b200.o"
    cmd = ["g++", "-std=c++20", "-c", "-Wall", "-I", os.path.join(ROOT, "oracle", "ref_shim"),
           "-I", os.path.join(REF, "include"), "-I", os.path.join(ROOT, "include"), str(src), "-o", str(obj)]
    subprocess.run(cmd, check=True)
    # link the binding with the reference runtime into a shared object to prove the symbols resolve
    so = tmp_path / "libbinding.so"
    cmd = ["g++", "-std=c++20", "-shared", "-fPIC", "-I", os.path.join(ROOT, "oracle", "ref_shim"),
           "-I", os.path.join(REF, "include"), "-I", os.path.join(ROOT, "include"), str(src),
           os.path.join(REF, "src", "resident.cpp"), "-L", build.LIB_DIR, "-lntt_b200", "-o", str(so),
           "-Wl,--no-undefined", f"-Wl,-rpath,{build.LIB_DIR}"]
    subprocess.run(cmd, check=True)
    assert so.exists()
