"""tq_index_search_device_noalloc: the search entry point that allocates no
device memory, for callers that may not call cudaMalloc while they serve
queries (a server that reserved all free HBM for its own pool, or a loop that
cannot take cudaMalloc's implicit synchronization). Its temporaries live in a
fixed 16 MiB array inside the library.

The test calls it through the C ABI twice in a row, with different query
batches, and checks each result bit for bit against the regular
tq_index_search_device on the same index; an over-size request must fail
cleanly. Further cases cover 3-bit and 2-bit indexes, k above 32 (eight
candidate lists per vector range) and a request whose candidate lists would
overflow the array unless the search uses fewer vector ranges. This file is collected last (name order) so that a run which stops at
the first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

import vectorcache_b200 as vcb
from vectorcache_b200.synthetic import power_law

pytestmark = pytest.mark.gpu

SCRATCH_BYTES = 16 << 20


def _search(lib, fn, h, q, k, torch):
    nq = q.shape[0]
    scores = torch.full((nq, k), float("nan"), dtype=torch.float32, device=q.device)
    ids = torch.full((nq, k), -1, dtype=torch.int64, device=q.device)
    ke = C.c_size_t(0)
    rc = fn(h, C.c_void_p(q.data_ptr()), C.c_size_t(nq), C.c_size_t(k), C.c_void_p(scores.data_ptr()),
            C.c_void_p(ids.data_ptr()), C.byref(ke), None)
    assert rc == 0, lib.tq_last_error().decode()
    lib.tq_index_synchronize(h)
    kk = ke.value
    return scores[:, :kk].cpu().numpy(), ids[:, :kk].cpu().numpy()


def _noalloc_fn(torch):
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    lib = vcb.load_library()
    fn = lib.tq_index_search_device_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_size_t, C.c_void_p, C.c_void_p,
                   C.POINTER(C.c_size_t), C.c_void_p]
    return lib, fn


def test_noalloc_search_matches_regular_search():
    torch = pytest.importorskip("torch")
    lib, fn = _noalloc_fn(torch)

    dim, bits, n = 768, 4, 20000
    db = power_law(n, dim, seed=31)
    idx = vcb.TurboQuantIndex(dim, bits)
    idx.calibrate(db[:2000])
    idx.add(db)
    idx.prepare()
    h = idx._h

    dev = torch.device("cuda", 0)
    batches = [(torch.from_numpy(power_law(40, dim, seed=32)).to(dev), 10),
               (torch.from_numpy(power_law(7, dim, seed=33)).to(dev), 17)]
    for q, k in batches:  # two calls in a row; the second must not see the first's leftovers
        want_s, want_i = _search(lib, lib.tq_index_search_device, h, q, k, torch)
        got_s, got_i = _search(lib, fn, h, q, k, torch)
        assert got_i.shape == want_i.shape == (q.shape[0], k)
        assert np.array_equal(got_i, want_i)
        assert np.array_equal(got_s.view(np.uint32), want_s.view(np.uint32))

    # A request larger than the fixed array is rejected before any work runs.
    nbg = dim // (8 // bits)
    too_many = SCRATCH_BYTES // (nbg * 32) + 1
    q_big = torch.zeros((too_many, dim), dtype=torch.float32, device=dev)
    out_s = torch.empty((too_many, 10), dtype=torch.float32, device=dev)
    out_i = torch.empty((too_many, 10), dtype=torch.int64, device=dev)
    ke = C.c_size_t(0)
    rc = fn(h, C.c_void_p(q_big.data_ptr()), C.c_size_t(too_many), C.c_size_t(10),
            C.c_void_p(out_s.data_ptr()), C.c_void_p(out_i.data_ptr()), C.byref(ke), None)
    assert rc == vcb.TQ_ERR_INVALID_ARGUMENT
    assert "no-alloc scratch" in lib.tq_last_error().decode()
    idx.close()


# (dim, bits, n, TQ+, [(queries, k), ...]). The last case needs 392 candidate
# lists of 64 x 200 entries (40 MB) under the regular plan, so the no-alloc
# search must cut the vector ranges to fit its 16 MiB array.
MORE_CASES = [
    (768, 3, 20000, True, [(40, 10), (9, 64)]),
    (1536, 2, 9000, True, [(33, 10), (5, 100)]),
    (256, 4, 30000, False, [(50, 100), (3, 256)]),
    (256, 4, 100000, False, [(64, 200), (64, 200)]),
]


@pytest.mark.parametrize("case", MORE_CASES, ids=lambda c: f"d{c[0]}_b{c[1]}_n{c[2]}")
def test_noalloc_bits_and_list_plans(case):
    torch = pytest.importorskip("torch")
    lib, fn = _noalloc_fn(torch)
    dim, bits, n, tq, batches = case
    db = power_law(n, dim, seed=dim + n)
    idx = vcb.TurboQuantIndex(dim, bits)
    if tq:
        idx.calibrate(db[:2000])
    idx.add(db)
    idx.prepare()
    dev = torch.device("cuda", 0)
    for j, (nq, k) in enumerate(batches):
        q = torch.from_numpy(power_law(nq, dim, seed=100 + j)).to(dev)
        want_s, want_i = _search(lib, lib.tq_index_search_device, idx._h, q, k, torch)
        got_s, got_i = _search(lib, fn, idx._h, q, k, torch)
        assert got_i.shape == want_i.shape == (nq, min(k, n))
        assert np.array_equal(got_i, want_i), (nq, k)
        assert np.array_equal(got_s.view(np.uint32), want_s.view(np.uint32)), (nq, k)
    idx.close()
