"""File formats: .npy float32 matrices and VCEX exact-top-k files against
byte layouts built independently here (NumPy's own .npy writer/reader, and the
VCEX layout of tools/query-bench.cpp:180-340), plus index save/load and .npy
ingestion on the GPU."""
import struct

import numpy as np
import pytest

from vectorcache_b200 import formats


def test_npy_roundtrip_with_numpy(tmp_path):
    m = np.random.default_rng(0).standard_normal((37, 24)).astype(np.float32)
    p = tmp_path / "a.npy"
    formats.write_npy_f32(p, m)
    assert np.array_equal(np.load(p), m)  # numpy reads ours
    q = tmp_path / "b.npy"
    np.save(q, m)
    assert formats.npy_shape(q) == (37, 24)
    assert np.array_equal(formats.read_npy_f32(q), m)  # we read numpy's
    assert np.array_equal(formats.read_npy_f32(q, 5, 7), m[5:12])


def test_npy_rejects_wrong_dtype(tmp_path):
    p = tmp_path / "d.npy"
    np.save(p, np.zeros((3, 8), np.float64))
    with pytest.raises(ValueError):
        formats.npy_shape(p)


def _vcex_bytes(ids, index_n, seed, label, split, qsplit):
    nq, k = ids.shape
    b = b"VCEX" + struct.pack("<IQQQQ", 1, nq, k, index_n, seed)
    for s in (label, split, qsplit):
        b += struct.pack("<I", len(s)) + s.encode()
    return b + ids.astype("<u8").tobytes()


def test_vcex_layout_both_ways(tmp_path):
    ids = np.arange(30, dtype=np.uint64).reshape(3, 10) * 7
    p = tmp_path / "gt.bin"
    formats.write_vcex(p, ids, index_n=1000, seed=42, source_label="npy-x", split="test", query_split="holdout")
    assert p.read_bytes() == _vcex_bytes(ids, 1000, 42, "npy-x", "test", "holdout")
    q = tmp_path / "hand.bin"
    q.write_bytes(_vcex_bytes(ids[:2], 77, 9, "a", "", "bb"))
    meta, got = formats.read_vcex(q)
    assert meta == {"n_queries": 2, "k": 10, "index_n": 77, "seed": 9}
    assert np.array_equal(got, ids[:2])


@pytest.mark.gpu
def test_index_save_load_and_npy_ingest(tmp_path):
    import vectorcache_b200 as vcb
    from vectorcache_b200.synthetic import power_law

    dim, bits = 384, 4
    db = power_law(3000, dim, seed=11)
    q = power_law(12, dim, seed=12)
    a = vcb.TurboQuantIndex(dim, bits)
    a.calibrate(db[:700])
    npy = tmp_path / "db.npy"
    np.save(npy, db)
    a.add_npy(npy)
    a.prepare()
    want = a.search(q, 25)
    path = tmp_path / "index.vcb"
    a.save(path)
    b = vcb.TurboQuantIndex.load(path)
    assert b.size == 3000 and b.info()["calibrated"]
    got = b.search(q, 25)
    assert np.array_equal(got.ids, want.ids)
    assert np.array_equal(got.scores.view(np.uint32), want.scores.view(np.uint32))
    assert np.array_equal(b.codes_flat(), a.codes_flat())
    assert np.array_equal(b.alpha().view(np.uint32), a.alpha().view(np.uint32))
    # a loaded index keeps growing like any prepared one
    b.add(db[:10])
    assert b.size == 3010
    raw = bytearray(path.read_bytes())
    raw[100] ^= 0xFF
    bad = tmp_path / "bad.vcb"
    bad.write_bytes(bytes(raw))
    with pytest.raises(ValueError):
        vcb.TurboQuantIndex.load(bad)
