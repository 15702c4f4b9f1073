"""The scan planner's rules, on the host (no GPU): the tilings the measured
shapes run with, as tq_index_scan_plan reports them on a B200 (148 SMs).

* 10k queries: four queries per CTA over two vector ranges (whole 1M rows).
* One or two queries over at most two waves of 2048-vector blocks split by
  256-group batch; one query takes four CTAs per SM when that wastes less of
  the last wave (1M vectors), two otherwise (200k, 500k vectors).
* Larger one-query scans run whole rows: a register ring on four CTAs per SM
  for 2- and 4-bit codes (stages 0) while four CTAs' LUTs fit an SM (rows up
  to 3072 dims at 4 bits), shared-memory slots for wider rows, for 3-bit
  codes and for two queries.
"""
import pytest

import vectorcache_b200 as vcb

SMS = 148


def plan(n, nq, dim, bits, k=10):
    return vcb.scan_plan_shape(n, nq, dim, bits, k, SMS)


def test_ten_thousand_queries_four_per_cta():
    p = plan(1_000_000, 10_000, 1536, 4)
    assert p == {"q_per_cta": 4, "n_ranges": 2, "range_vectors": 501_760, "split_batches": 1, "stages": 0,
                 "split_ctas_per_sm": 0}


@pytest.mark.parametrize("n,dim,bits,batches,per_sm", [
    (1_000_000, 1536, 4, 3, 4),
    (1_000_000, 768, 3, 2, 4),
    (1_000_000, 1536, 2, 2, 4),
    (500_000, 1536, 4, 3, 2),
    (200_000, 1536, 4, 3, 2),
])
def test_one_query_batch_split(n, dim, bits, batches, per_sm):
    p = plan(n, 1, dim, bits)
    blocks = (n + 2047) // 2048
    assert p["q_per_cta"] == 1 and p["n_ranges"] == blocks and p["range_vectors"] == 2048
    assert p["split_batches"] == batches and p["stages"] == 0 and p["split_ctas_per_sm"] == per_sm


def test_two_queries_split_on_two_ctas_per_sm():
    p = plan(1_000_000, 2, 1536, 4)
    assert p["q_per_cta"] == 2 and p["split_batches"] == 3 and p["split_ctas_per_sm"] == 2


@pytest.mark.parametrize("n,nq,dim,bits,stages", [
    (4_000_000, 1, 1536, 4, 0),   # register ring, four CTAs per SM
    (4_000_000, 1, 1536, 2, 0),
    (10_000_000, 1, 768, 3, 6),   # shared-memory slots
    (4_000_000, 2, 1536, 4, 5),
    (4_000_000, 1, 3072, 4, 0),   # the widest rows whose four LUTs fit an SM
    (4_000_000, 1, 4096, 4, 6),   # wider: slots again
])
def test_whole_row_code_stream(n, nq, dim, bits, stages):
    p = plan(n, nq, dim, bits)
    assert p["split_batches"] == 1 and p["split_ctas_per_sm"] == 0 and p["q_per_cta"] == nq
    assert p["stages"] == stages


def test_ten_million_serving_index_ranges():
    p = plan(10_000_000, 1, 768, 3)
    assert p["n_ranges"] == 1628 and p["range_vectors"] == 6144


def test_k_above_register_list_never_splits():
    p = plan(1_000_000, 1, 1536, 4, k=64)
    assert p["split_batches"] == 1 and p["stages"] == 0


@pytest.mark.parametrize("args", [
    (0, 1, 1536, 4, 10, SMS),
    (1000, 0, 1536, 4, 10, SMS),
    (1000, 1, 1537, 4, 10, SMS),
    (1000, 1, 1536, 5, 10, SMS),
    (1000, 1, 1536, 4, 0, SMS),
    (1000, 1, 1536, 4, 257, SMS),
    (1000, 1, 1536, 4, 10, 0),
])
def test_invalid_shapes_rejected(args):
    with pytest.raises(vcb.TurboQuantError):
        vcb.scan_plan_shape(*args)
