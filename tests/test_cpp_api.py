"""The header-only C++20 API (include/vectorcache_b200.hpp) compiles against
the C ABI, and on a GPU C++ programs built with it show the reference's
index-test properties (tests/cpp/flat_index_props.cpp) and the bucketed index /
serving properties (tests/cpp/bucketed_props.cpp)."""
import shutil
import subprocess

import pytest

from conftest import ROOT

PROGRAMS = ["flat_index_props", "bucketed_props"]


def _compile(tmp_path, name):
    gxx = shutil.which("g++") or "/usr/bin/g++"
    exe = tmp_path / name
    lib_dir = ROOT / "vectorcache_b200"
    cmd = [gxx, "-std=c++20", "-O1", str(ROOT / "tests" / "cpp" / f"{name}.cpp"),
           "-I", str(ROOT / "include"), "-L", str(lib_dir), "-lvectorcache_b200",
           f"-Wl,-rpath,{lib_dir}", "-o", str(exe)]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


@pytest.mark.parametrize("name", PROGRAMS)
def test_cpp_api_compiles_and_links(tmp_path, name):
    from vectorcache_b200 import build

    build.build()
    assert _compile(tmp_path, name).exists()


@pytest.mark.gpu
@pytest.mark.parametrize("name", PROGRAMS)
def test_cpp_program_properties(tmp_path, name):
    exe = _compile(tmp_path, name)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    assert out.stdout.startswith("OK")
