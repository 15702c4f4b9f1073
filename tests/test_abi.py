"""The C ABI library loads without a GPU, exports every entry point declared in
include/vectorcache_b200.h, and its host-side tables match the reference's."""
import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

import vectorcache_b200 as vcb
from conftest import ROOT, cuda_available


def declared_symbols():
    text = (ROOT / "include" / "vectorcache_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(tq_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    from vectorcache_b200 import build

    build.build()
    return vcb.load_library()


def test_library_exports_all_declared_symbols(lib):
    syms = declared_symbols()
    assert len(syms) >= 20
    raw = ctypes.CDLL(str(vcb.LIB_PATH))
    missing = [s for s in syms if not hasattr(raw, s)]
    assert not missing, missing


def test_host_tables_match_reference(lib, tables):
    for key in tables:
        if key.endswith("_centroids"):
            bits = int(key.split("_")[0][1:])
            dim = int(key.split("_")[1][1:])
            b, c = vcb.codebook(bits, dim)
            assert np.array_equal(c.view(np.uint32), tables[key].view(np.uint32)), key
            assert np.array_equal(b.view(np.uint32), tables[key.replace("centroids", "boundaries")].view(np.uint32))
    for dim in (8, 104, 128, 1536):
        s, p = vcb.rotation_tables(dim)
        assert np.array_equal(s, tables[f"d{dim}_signs"]) and np.array_equal(p, tables[f"d{dim}_perm"])


def test_argument_validation_matches_reference(lib):
    # rotation.cpp:140-145 / flat_index.cpp:92-98: dim % 8 == 0, 0 < dim <= 16384, bits in {2,3,4}.
    for dim, bits in [(0, 4), (100, 4), (16392, 4), (128, 1), (128, 5)]:
        with pytest.raises(vcb.InvalidArgument):
            vcb.TurboQuantIndex(dim, bits)
    with pytest.raises(vcb.InvalidArgument):
        vcb.codebook(5, 128)
    with pytest.raises(vcb.InvalidArgument):
        vcb.rotation_tables(12)


@pytest.mark.skipif(cuda_available(), reason="checks the no-GPU error path")
def test_no_device_is_an_error_not_a_fallback(lib):
    with pytest.raises(vcb.TurboQuantError) as e:
        vcb.TurboQuantIndex(128, 4)
    assert e.value.code in (vcb.TQ_ERR_CUDA, vcb.TQ_ERR_INVALID_ARGUMENT)
