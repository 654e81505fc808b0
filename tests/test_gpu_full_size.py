"""GPU parity at the benchmark workloads' own sizes, through the same calls
the benchmark times.

- filter + GROUP BY over the 6M-row fact table (1000 groups), with native
  widths and with every integer 8 bytes wide (Hive's layout);
- the inner hash join of 1.5M unique build keys with a 60M-row probe, with
  the benchmark's output set (probe row id, int64 and double build payloads,
  no build row ids): the lean write pass.  Once with the dense surrogate keys
  the benchmark uses (direct table) and once with the same keys spread over
  the int64 range (hashed table);
- the 60M-row ORDER BY (d, k), stable, with uniform and Zipf(0.99) k;
- all 512 instances of the batched filter + group-by, in one batch.

Keys, counts, integer sums, MIN/MAX, join pairs and sort order bit-exact;
DOUBLE SUM/AVG within REL_TOL of the oracle's Hive-order sequential sum
(parity.REL_TOL), and the relative error of every double result against
the oracle's FP64 Neumaier compensated sum is stated and bounded by the
same tolerance.  The oracle's multi-threaded forms (all host threads) keep
the join and sort checks to seconds; they compute the same pairs and the
same stable order as the sequential ones.
"""
import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

from ghive_b200 import abi, workloads
from oracle import oracle
from parity import REL_TOL, compare_groupby, error_summary, host_cols

pytestmark = pytest.mark.gpu

THREADS = max(1, os.cpu_count() or 1)


@pytest.fixture(scope="module")
def ctx():
    from ghive_b200.ops import Context
    c = Context(0)
    yield c
    c.close()


def dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _types(cols, aggs):
    return [abi.agg_out_type(t, abi.TYPE_OF_DTYPE[np.dtype(cols[c].dtype)] if c >= 0 else abi.LONG)
            for t, c in aggs]


def test_fact_table_filter_groupby_6M(ctx):
    cols = workloads.fact_table(6_000_000, seed_idx=0)
    pred, aggs = workloads.fact_predicate(), workloads.AGGS_FACT
    ok, oa, comp = oracle.filter_groupby(pred, cols, [0], aggs, cap=1000, with_comp=True)
    gk, ga, g = ctx.filter_groupby(pred, [dev(c) for c in cols], [0], aggs, capacity=1000,
                                   max_groups=1000)
    assert g == 1000
    errs = compare_groupby(host_cols(gk), host_cols(ga), ok, oa, _types(cols, aggs), comp)
    s = error_summary(errs)
    print("fact table 6M: double SUM/AVG error vs compensated sum", s)
    assert s["results"] == 2000 and s["max_rel"] <= REL_TOL


def test_fact_table_hive_layout_6M(ctx):
    """The same query with every integer column 8 bytes wide, as Hive's
    LongColumnVector holds them (k and d widened to int64): LONG keys and
    LONG MIN/MAX."""
    k, qty, price, d = workloads.fact_table(6_000_000, seed_idx=0)
    cols = [k.astype(np.int64), qty, price, d.astype(np.int64)]
    pred, aggs = workloads.fact_predicate(), workloads.AGGS_FACT
    ok, oa, comp = oracle.filter_groupby(pred, cols, [0], aggs, cap=1000, with_comp=True)
    gk, ga, g = ctx.filter_groupby(pred, [dev(c) for c in cols], [0], aggs, capacity=1000,
                                   max_groups=1000)
    assert g == 1000
    errs = compare_groupby(host_cols(gk), host_cols(ga), ok, oa, _types(cols, aggs), comp)
    s = error_summary(errs)
    assert s["results"] == 2000 and s["max_rel"] <= REL_TOL


def _join_full(ctx, sparse):
    import torch
    n_build, n_probe = 1_500_000, 60_000_000
    (bkey, bpay), (fk, _) = workloads.join_tables(n_build, n_probe, seed_idx=1, sparse=sparse)
    from ghive_b200.ops import _Outs
    d_bpay = [dev(c) for c in bpay]
    t = ctx.join_build(dev(bkey), build_payload=d_bpay)
    rows, dup, slots = t.info()
    assert rows == n_build and dup == 1
    # the benchmark's outputs: probe row id and the two payloads, no NULL maps
    ob = _Outs([abi.LONG, abi.DOUBLE], n_probe, "cuda:0", with_nulls=False)
    op = _Outs([], n_probe, "cuda:0")
    prow = torch.empty(n_probe, dtype=torch.int32, device="cuda:0")
    d_rows = torch.zeros(1, dtype=torch.int64, device="cuda:0")
    ctx.join_probe(t, dev(fk), abi.INNER_JOIN, capacity=n_probe, rowids=False, sync=False,
                   outs=(ob, op, prow, None, d_rows))
    ctx.sync()
    k = int(d_rows.item())
    g_prow = prow[:k].cpu().numpy()
    g_long = ob.cols[0][0][:k].cpu().numpy()
    g_dbl = ob.cols[1][0][:k].cpu().numpy()
    t.free()
    e_prow, (e_long, e_dbl) = oracle.hash_join_mt(THREADS, bkey, fk, bpay)
    assert k == len(e_prow)
    # probe-row order on both sides; unique build keys: one pair per probe row,
    # so the sorted multisets are the arrays themselves
    assert np.all(np.diff(g_prow) > 0)
    assert np.array_equal(g_prow, e_prow)
    assert np.array_equal(g_long, e_long)
    assert np.array_equal(g_dbl.view(np.uint64), e_dbl.view(np.uint64))
    return slots


def test_join_1_5M_by_60M_lean_direct_table(ctx):
    slots = _join_full(ctx, sparse=False)
    assert slots == 1_500_000  # dense keys: slot = key - min


def test_join_1_5M_by_60M_lean_hashed_table(ctx):
    slots = _join_full(ctx, sparse=True)
    assert slots & (slots - 1) == 0  # hashed: power-of-two buckets


@pytest.mark.parametrize("zipf", [False, True])
def test_sort_60M(ctx, zipf):
    d, k, rowid = workloads.sort_table(60_000_000, zipf=zipf, seed_idx=2)
    ok, op, _ = ctx.sort([dev(d), dev(k)], payload=[dev(rowid)])
    g_rowid = op[0][0].cpu().numpy()
    g_d, g_k = ok[0][0].cpu().numpy(), ok[1][0].cpu().numpy()
    del ok, op
    perm = oracle.sort_perm([d, k], threads=THREADS)
    assert np.array_equal(g_rowid, perm)    # rowid = input position: stable order
    assert np.array_equal(g_d, d[perm]) and np.array_equal(g_k, k[perm])


def test_batched_512_instances(ctx):
    import torch
    specs = workloads.batched_specs(512, seed_idx=3)
    inst = workloads.batched_instances_device(specs, torch.device("cuda:0"))
    aggs = workloads.AGGS_FACT
    entries = [(workloads.batched_predicate(s["cut"]), it["cols"],
                max(1, min(s["groups"], s["rows"])) + 8, s["groups"]) for s, it in zip(specs, inst)]
    b = ctx.batch_groupby(entries, [0], aggs, autotune=True)
    b.launch()
    ctx.sync()
    counts = b.groups.cpu().numpy()
    types = [abi.LONG] * 2 + [abi.DOUBLE] * 2 + [abi.INT] * 2

    def check(i):
        s, it = specs[i], inst[i]
        cols = [c.cpu().numpy() for c in it["cols"]]
        pred = workloads.batched_predicate(s["cut"])
        ok, oa, comp = oracle.filter_groupby(pred, cols, [0], aggs, cap=entries[i][2],
                                             with_comp=True)
        gk, ga, g = b.results(i, counts)
        assert g == len(ok[0][0]), i
        return compare_groupby(host_cols(gk), host_cols(ga), ok, oa, types, comp)

    # the oracle calls release the GIL: one sequential (Hive-order) oracle per
    # instance, instances spread over the host threads, largest first
    order = sorted(range(len(specs)), key=lambda i: -specs[i]["rows"])
    with ThreadPoolExecutor(THREADS) as ex:
        errs = list(ex.map(check, order))
    s = error_summary(np.concatenate(errs))
    print("batched 512: double SUM/AVG error vs compensated sum", s)
    assert s["max_rel"] <= REL_TOL
    b.free()
