"""The top-p selection behind the bucketed routing (tq_select_top_device)
against a numpy statement of its order: score descending, equal scores by lower
column, -inf and NaN never selected, short rows padded with (-inf, 0xffffffff).
Rows up to 32768 columns take the radix-select kernel, wider rows the streaming
sort; both are covered."""
import numpy as np
import pytest


def _expected(s: np.ndarray, p: int):
    rows, ncols = s.shape
    out_s = np.full((rows, p), -np.inf, np.float32)
    out_i = np.full((rows, p), 0xFFFFFFFF, np.uint32)
    cols = np.arange(ncols)
    for r in range(rows):
        ok = (s[r] > -np.inf) & ~np.isnan(s[r])
        c = cols[ok]
        order = c[np.lexsort((c, -s[r, c]))][:p]
        out_s[r, : len(order)] = s[r, order]
        out_i[r, : len(order)] = order
    return out_s, out_i


def _run(s: np.ndarray, p: int, ncols: int | None = None):
    import torch

    from vectorcache_b200.bucketed import select_top_device

    d = torch.from_numpy(s).cuda()
    rows = s.shape[0]
    ts = torch.empty((rows, p), dtype=torch.float32, device="cuda")
    ti = torch.empty((rows, p), dtype=torch.int32, device="cuda")
    select_top_device(d, p, ts, ti, ncols=ncols)
    torch.cuda.synchronize()
    return ts.cpu().numpy(), ti.cpu().numpy().view(np.uint32)


def _check(s, p, ncols=None):
    got_s, got_i = _run(s, p, ncols)
    exp_s, exp_i = _expected(s[:, : (ncols or s.shape[1])], p)
    assert np.array_equal(got_i, exp_i)
    assert np.array_equal(got_s.view(np.uint32), exp_s.view(np.uint32))


@pytest.mark.gpu
@pytest.mark.parametrize("ncols,p", [(3217, 512), (3217, 256), (700, 100), (40000, 2048), (40000, 37), (5, 1)])
def test_random_rows(ncols, p):
    rng = np.random.default_rng(ncols + p)
    _check(rng.standard_normal((48, ncols)).astype(np.float32), p)


@pytest.mark.gpu
@pytest.mark.parametrize("ncols", [3217, 40000])
def test_ties_infinities_nan_and_zero(ncols):
    rng = np.random.default_rng(7)
    s = np.round(rng.standard_normal((32, ncols)), 1).astype(np.float32)  # many equal scores
    s[0, :] = 0.5  # one tie group across the whole row
    s[1, ::2] = -0.0
    s[1, 1::2] = 0.0
    s[2, :] = -np.inf
    s[2, [3, 17, 40]] = [1.0, 2.0, 1.0]  # fewer selectable columns than p
    s[3, ::3] = np.nan
    s[4, :] = np.nan
    s[5, :] = -np.finfo(np.float32).max
    s[6, ::5] = np.inf
    for p in (1, 100, 512, 2048):
        _check(s, p)


@pytest.mark.gpu
def test_row_stride_wider_than_columns():
    rng = np.random.default_rng(3)
    s = rng.standard_normal((20, 4000)).astype(np.float32)
    _check(s, 300, ncols=3500)
