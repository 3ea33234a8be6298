"""The reference-side binding (ntt_gpu_b200/binding/resident_b200.cpp, shown
in INTEGRATION.md section A) compiles against the reference's own headers and
links, with the reference's unchanged src/resident.cpp, against
libntt_b200.so with no undefined symbol. Needs the reference tree (beside this
repository, or $NTT_REFERENCE_TREE); no GPU."""
import os
import re
import subprocess

import pytest

from ntt_gpu_b200 import build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.environ.get("NTT_REFERENCE_TREE", os.path.join(ROOT, "..", "reference"))
BINDING = os.path.join(ROOT, "ntt_gpu_b200", "binding", "resident_b200.cpp")


def test_integration_guide_shows_the_binding():
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    blocks = re.findall(r"```cpp\n(.*?)```", text, re.S)
    assert blocks, "INTEGRATION.md carries the binding"
    assert blocks[0].strip() == open(BINDING).read().strip()


def test_binding_compiles_against_reference_headers(tmp_path):
    if not os.path.isdir(os.path.join(REF, "include", "ntt")):
        pytest.skip("reference tree not present")
    build.build()
    so = tmp_path / "libbinding.so"
    cmd = ["g++", "-std=c++20", "-shared", "-fPIC", "-Wall", "-I", os.path.join(ROOT, "oracle", "ref_shim"),
           "-I", os.path.join(REF, "include"), "-I", os.path.join(ROOT, "include"), BINDING,
           os.path.join(REF, "src", "resident.cpp"), "-L", build.LIB_DIR, "-lntt_b200", "-o", str(so),
           "-Wl,--no-undefined", f"-Wl,-rpath,{build.LIB_DIR}"]
    subprocess.run(cmd, check=True)
    assert so.exists()
