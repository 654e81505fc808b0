"""The bounded device waits, made to run out on purpose.

Every decoupled look-back (the filter's output offsets, the join probe's
chunk offsets, the sort's digit offsets) gives up after a bounded number of
polls of a not yet published earlier tile, raises GHB_ERR_TIMEOUT into the
context's status word and returns.  With the bound set to one poll through
ghb_ctx_set_spin_limit, a launch of many concurrently running tiles meets a
not-ready predecessor; the test checks that ghb_sync reports the timeout
(nothing hangs, every write stays inside the buffers), then that with the
default bound restored the same context gives the oracle's result.
"""
import numpy as np
import pytest

from ghive_b200 import abi, workloads
from ghive_b200._lib import GhbError
from oracle import oracle

pytestmark = pytest.mark.gpu

ATTEMPTS = 8


@pytest.fixture(scope="module")
def ctx():
    from ghive_b200.ops import Context
    c = Context(0)
    yield c
    c.close()


def dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _times_out(ctx, run):
    """Runs `run` with a one-poll bound until a call reports GHB_ERR_TIMEOUT."""
    ctx.set_spin_limit(1)
    try:
        for _ in range(ATTEMPTS):
            try:
                run()
            except GhbError as e:
                assert e.code == abi.ERR_TIMEOUT, e
                return True
        return False
    finally:
        ctx.set_spin_limit(0)


def test_filter_lookback_timeout_then_clean_call(ctx):
    g = np.random.default_rng(70)
    n = 20_000_000
    d = g.integers(0, 2526, n, dtype=np.int32)
    pred = abi.Pred.leaf(abi.FILTER_LT, 0, a=1263)
    dd = dev(d)
    assert _times_out(ctx, lambda: ctx.filter(pred, [dd]))
    outs, k = ctx.filter(pred, [dd])
    sel = oracle.filter_rows(pred, [d])
    assert k == len(sel)
    assert np.array_equal(outs[0][0].cpu().numpy(), d[sel])


def test_join_scan_timeout_then_clean_call(ctx):
    (bkey, bpay), (fk, _) = workloads.join_tables(100_000, 8_000_000, seed_idx=71)
    t = ctx.join_build(dev(bkey))
    dfk = dev(fk)
    assert _times_out(ctx, lambda: ctx.join_probe(t, dfk))
    r = ctx.join_probe(t, dfk)
    pr, br = oracle.hash_join(bkey, fk)
    assert r["rows"] == len(pr)
    assert np.array_equal(r["probe_rowid"].cpu().numpy(), pr)
    assert np.array_equal(r["build_rowid"].cpu().numpy(), br)
    t.free()


def test_sort_lookback_timeout_then_clean_call(ctx):
    d, k, rowid = workloads.sort_table(8_000_000, seed_idx=72)
    dd, dk, dr = dev(d), dev(k), dev(rowid)
    assert _times_out(ctx, lambda: ctx.sort([dd, dk], payload=[dr]))
    _, op, _ = ctx.sort([dd, dk], payload=[dr])
    perm = oracle.sort_perm([d, k], threads=8)
    assert np.array_equal(op[0][0].cpu().numpy(), rowid[perm])
