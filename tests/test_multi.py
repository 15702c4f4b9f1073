"""Multi-index launch on the GPU: one persistent, graph-captured scan over
indexes of uneven n, dim and bits with uneven batch sizes and k returns, for
every index, exactly the per-index search results (ids and scores bit for
bit); graph replays with new queries stay exact; the autotuner's choice does
not change results."""
import numpy as np
import pytest

import vectorcache_b200 as vcb
from vectorcache_b200.multi import MultiIndex
from vectorcache_b200.synthetic import gaussian_mixture, power_law

pytestmark = pytest.mark.gpu


def bits_equal(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return a.shape == b.shape and np.array_equal(a.view(np.uint8), b.view(np.uint8))


SPECS = [  # (dim, n, bits, nq, k, tq)
    (128, 30000, 4, 1, 10, False),
    (384, 9000, 3, 37, 64, True),
    (768, 12345, 2, 300, 10, True),
    (256, 70000, 4, 129, 1, False),
    (104, 2049, 3, 8, 100, False),
    (1536, 4000, 4, 17, 10, True),
]


@pytest.fixture(scope="module")
def indexes():
    out = []
    for j, (dim, n, bits, nq, k, tq) in enumerate(SPECS):
        db = power_law(n, dim, seed=j) if dim % 2 == 0 and j % 2 else gaussian_mixture(n, 1, dim, seed=j)[0]
        idx = vcb.TurboQuantIndex(dim, bits)
        if tq:
            idx.calibrate(db[:1000])
        idx.add(db)
        idx.prepare()
        out.append((idx, db))
    yield out
    for idx, _ in out:
        idx.close()


def _queries(j, dim, nq, seed):
    return power_law(nq, dim, seed=100 + 7 * j + seed)


@pytest.mark.parametrize("autotune", [False, True])
def test_multi_launch_equals_per_index_search(indexes, autotune):
    multi = MultiIndex([x for x, _ in indexes])
    multi.plan([s[3] for s in SPECS], [s[4] for s in SPECS], autotune=autotune)
    cfg = multi.config()
    assert cfg["items"] > 0 and cfg["ctas"] > 0
    if autotune:
        assert len(cfg["tuned_ms"]) >= 4 and 0 <= cfg["direct_indexes"] <= len(SPECS)
    for rep in range(2):  # the graph is replayed with new queries
        qs = [_queries(j, s[0], s[3], rep) for j, s in enumerate(SPECS)]
        for j, q in enumerate(qs):
            multi.set_queries(j, q)
        multi.launch()
        multi.synchronize()
        for j, ((idx, _), q) in enumerate(zip(indexes, qs)):
            got_s, got_i = multi.results(j)
            want = idx.search(q, SPECS[j][4])
            assert np.array_equal(got_i, want.ids), (j, rep)
            assert bits_equal(got_s, want.scores), (j, rep)
    # the same sequence without the graph
    multi.run_uncaptured()
    multi.synchronize()
    got_s, got_i = multi.results(2)
    want = indexes[2][0].search(qs[2], SPECS[2][4])
    assert np.array_equal(got_i, want.ids)
    multi.close()
