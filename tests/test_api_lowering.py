"""The C++ operator surface (include/graptor_b200/api.h) compiled on the host
and its lowering checked without a GPU: relax / filter / record expressions
of the reference's analytics to the descriptor kinds, iif in the reference's
blend order, float rounding of vertex programs (tests/cpp/api_lowering.cc)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_api_lowering_table(tmp_path):
    cxx = shutil.which("g++")
    if not cxx:
        pytest.skip("no host C++ compiler")
    lib = os.path.join(ROOT, "graptor_b200")
    exe = str(tmp_path / "api_lowering")
    r = subprocess.run([cxx, "-std=c++17", "-O0", "-I", os.path.join(ROOT, "include"),
                        os.path.join(ROOT, "tests", "cpp", "api_lowering.cc"), "-o", exe, "-L", lib, "-lgg",
                        f"-Wl,-rpath,{lib}"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    r = subprocess.run([exe], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and "ok" in r.stdout, r.stdout + r.stderr
