"""The header-only C++20 API (include/vectorcache_b200.hpp) compiles against
the C ABI, and on a GPU a C++ program built with it shows the reference's
index-test properties (tests/cpp/flat_index_props.cpp)."""
import shutil
import subprocess

import pytest

from conftest import ROOT


def _compile(tmp_path):
    gxx = shutil.which("g++") or "/usr/bin/g++"
    exe = tmp_path / "flat_index_props"
    lib_dir = ROOT / "vectorcache_b200"
    cmd = [gxx, "-std=c++20", "-O1", str(ROOT / "tests" / "cpp" / "flat_index_props.cpp"),
           "-I", str(ROOT / "include"), "-L", str(lib_dir), "-lvectorcache_b200",
           f"-Wl,-rpath,{lib_dir}", "-o", str(exe)]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def test_cpp_api_compiles_and_links(tmp_path):
    from vectorcache_b200 import build

    build.build()
    assert _compile(tmp_path).exists()


@pytest.mark.gpu
def test_cpp_program_reference_properties(tmp_path):
    exe = _compile(tmp_path)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    assert out.stdout.startswith("OK")
