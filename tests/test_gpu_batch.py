"""GPU parity of the batched filter + group-by (one persistent launch over
many instances, replayed from a CUDA graph).

Every instance's result must equal the oracle's Hive group-by of that
instance alone, and the single-call operator's result on the same instance:
bit-exact for keys, counts, integer sums, MIN/MAX; DOUBLE SUM/AVG within
REL_TOL relative of the oracle's sequential sum.
"""
import numpy as np
import pytest

from ghive_b200 import abi, workloads
from oracle import oracle

pytestmark = pytest.mark.gpu

REL_TOL = 1e-12


@pytest.fixture(scope="module")
def ctx():
    from ghive_b200.ops import Context
    c = Context(0)
    yield c
    c.close()


def dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _np(x):
    return x.cpu().numpy() if hasattr(x, "cpu") else np.asarray(x)


def _canon(keys, aggs):
    """Rows ordered by key (NULL first); one key column at most."""
    if keys:
        v, nl = _np(keys[0][0]), _np(keys[0][1]).astype(bool)
        order = np.lexsort((np.where(nl, 0, v), ~nl))
        keys = [(v[order], nl[order])]
    else:
        order = slice(None)
    return keys, [(_np(v)[order], _np(nl).astype(bool)[order]) for v, nl in aggs]


def _assert_same(exp, got, types, what):
    (ek, ea), (gk, ga) = exp, got
    for (ev, en), (gv, gn) in zip(ek, gk):
        assert np.array_equal(en, gn), what
        assert np.array_equal(ev[~en], gv[~gn]), what
    for j, ((ev, en), (gv, gn)) in enumerate(zip(ea, ga)):
        assert np.array_equal(en, gn), (what, j)
        if types[j] == abi.DOUBLE:
            e, g = ev[~en], gv[~gn]
            assert np.all(np.abs(g - e) <= REL_TOL * np.maximum(np.abs(e), 1e-300)), (what, j)
        else:
            assert np.array_equal(ev[~en], gv[~gn]), (what, j)


def _types(cols, aggs):
    return [abi.agg_out_type(t, abi.TYPE_OF_DTYPE[np.dtype(cols[c].dtype)] if c >= 0 else abi.LONG)
            for t, c in aggs]


def _make(count, seed, max_rows, extra_small=True):
    inst = list(workloads.batched_instances(count, seed_idx=seed, min_rows=1_000, max_rows=max_rows))
    if extra_small:
        # an empty and a one-row instance ride along
        for rows in (0, 1):
            g = workloads.rng(seed, 99 + rows)
            inst.append({"rows": rows, "groups": 10, "theta": 0.0, "cut": 2000,
                         "cols": [g.integers(0, 10, rows, dtype=np.int64),
                                  g.integers(1, 51, rows, dtype=np.int64),
                                  g.integers(90000, 10500001, rows, dtype=np.int64) / 100.0,
                                  g.integers(0, 2526, rows, dtype=np.int32)]})
    return inst


def _run_batch(ctx, inst, keys, aggs, **kw):
    dcols = [[dev(c) for c in it["cols"]] for it in inst]
    specs = []
    for it, dc in zip(inst, dcols):
        cap = max(1, min(it["groups"], it["rows"])) + 8 if keys else 1
        specs.append((workloads.batched_predicate(it["cut"]), dc, cap, it["groups"] if keys else 0))
    b = ctx.batch_groupby(specs, keys, aggs, **kw)
    return b, dcols, specs


@pytest.mark.parametrize("autotune,use_graph", [(True, True), (False, False)])
def test_batch_matches_oracle_and_single_calls(ctx, autotune, use_graph):
    inst = _make(36, seed=31, max_rows=300_000)
    aggs = workloads.AGGS_FACT
    b, dcols, specs = _run_batch(ctx, inst, [0], aggs, autotune=autotune, use_graph=use_graph)
    b.launch()
    ctx.sync()
    counts = b.groups.cpu().numpy()
    for i, it in enumerate(inst):
        types = _types(it["cols"], aggs)
        pred = workloads.batched_predicate(it["cut"])
        ok, oa = oracle.filter_groupby(pred, it["cols"], [0], aggs)
        gk, ga, g = b.results(i, counts)
        assert g == len(ok[0][0]), i
        _assert_same(_canon(ok, oa), _canon(gk, ga), types, "instance %d vs oracle" % i)
        sk, sa, sg = ctx.filter_groupby(pred, dcols[i], [0], aggs, capacity=specs[i][2],
                                        max_groups=it["groups"])
        assert sg == g
        _assert_same(_canon(sk, sa), _canon(gk, ga), types, "instance %d vs single call" % i)
    desc = b.describe()
    assert desc["autotuned"] == autotune and desc["chunks"] >= len(inst) - 2
    b.free()


def test_batch_replays_are_identical(ctx):
    inst = _make(12, seed=32, max_rows=200_000)
    aggs = workloads.AGGS_FACT
    b, _, _ = _run_batch(ctx, inst, [0], aggs, autotune=False)
    results = []
    for _ in range(3):
        b.launch()
        ctx.sync()
        counts = b.groups.cpu().numpy()
        results.append([_canon(*b.results(i, counts)[:2]) for i in range(len(inst))])
    for r in results[1:]:
        for i, it in enumerate(inst):
            _assert_same(results[0][i], r[i], _types(it["cols"], aggs), "replay of %d" % i)
    b.free()


def test_batch_global_aggregate_with_empty_instances(ctx):
    inst = _make(8, seed=33, max_rows=50_000)
    aggs = [(abi.CNT, -1), (abi.SUM, 1), (abi.AVG, 2), (abi.MIN, 3), (abi.MAX, 0)]
    b, _, _ = _run_batch(ctx, inst, [], aggs, autotune=True)
    b.launch()
    ctx.sync()
    counts = b.groups.cpu().numpy()
    for i, it in enumerate(inst):
        ok, oa = oracle.filter_groupby(workloads.batched_predicate(it["cut"]), it["cols"], [], aggs)
        gk, ga, g = b.results(i, counts)
        assert g == 1
        _assert_same(_canon(ok, oa), _canon(gk, ga), _types(it["cols"], aggs), "instance %d" % i)
    b.free()


def test_batch_nullable_columns(ctx):
    g = workloads.rng(34)
    inst = []
    for i in range(6):
        n = int(g.integers(1, 40_000))
        k = g.integers(-50, 50, n, dtype=np.int64)
        k[g.random(n) < 0.02] = np.iinfo(np.int64).min     # the key whose image is the empty marker
        kn = g.random(n) < 0.05
        v = g.integers(-10**12, 10**12, n, dtype=np.int64)
        vn = g.random(n) < 0.1
        x = g.random(n) * 1e6
        xn = g.random(n) < 0.1
        d = g.integers(0, 2526, n, dtype=np.int32)
        inst.append({"rows": n, "groups": 110, "cut": 1800, "cols": [(k, kn), (v, vn), (x, xn), d]})
    aggs = [(abi.CNT, -1), (abi.CNT, 1), (abi.SUM, 1), (abi.AVG, 2), (abi.MIN, 1), (abi.MAX, 2)]
    specs, keep = [], []
    for it in inst:
        dc = [(dev(c[0]), dev(c[1].astype(np.uint8))) if isinstance(c, tuple) else dev(c)
              for c in it["cols"]]
        keep.append(dc)
        specs.append((workloads.batched_predicate(it["cut"]), dc, 128, 110))
    b = ctx.batch_groupby(specs, [0], aggs, autotune=True)
    b.launch()
    ctx.sync()
    counts = b.groups.cpu().numpy()
    types = [abi.LONG, abi.LONG, abi.LONG, abi.DOUBLE, abi.LONG, abi.DOUBLE]
    for i, it in enumerate(inst):
        ok, oa = oracle.filter_groupby(workloads.batched_predicate(it["cut"]), it["cols"], [0], aggs)
        gk, ga, gg = b.results(i, counts)
        assert gg == len(ok[0][0])
        _assert_same(_canon(ok, oa), _canon(gk, ga), types, "instance %d" % i)
    b.free()


def test_batch_capacity_error_then_clean_replay(ctx):
    from ghive_b200._lib import GhbError
    inst = _make(4, seed=35, max_rows=20_000, extra_small=False)
    aggs = workloads.AGGS_FACT
    dcols = [[dev(c) for c in it["cols"]] for it in inst]
    specs = [(workloads.batched_predicate(it["cut"]), dc, 4, 4) for it, dc in zip(inst, dcols)]
    b = ctx.batch_groupby(specs, [0], aggs, autotune=False)
    b.launch()
    with pytest.raises(GhbError) as e:
        ctx.sync()
    assert e.value.code == abi.ERR_CAPACITY
    b.free()
    # the context stays usable and a fresh batch on the same columns is right
    specs = [(s[0], s[1], max(1, min(it["groups"], it["rows"])) + 8, it["groups"])
             for s, it in zip(specs, inst)]
    b = ctx.batch_groupby(specs, [0], aggs, autotune=False)
    b.launch()
    ctx.sync()
    counts = b.groups.cpu().numpy()
    for i, it in enumerate(inst):
        ok, oa = oracle.filter_groupby(workloads.batched_predicate(it["cut"]), it["cols"], [0], aggs)
        gk, ga, g = b.results(i, counts)
        _assert_same(_canon(ok, oa), _canon(gk, ga), _types(it["cols"], aggs), "instance %d" % i)
    b.free()


def test_batch_rejects_mixed_signatures(ctx):
    from ghive_b200._lib import GhbError
    a = [dev(np.arange(10, dtype=np.int64)), dev(np.ones(10, dtype=np.int64))]
    c = [dev(np.arange(10, dtype=np.int64)), dev(np.ones(10, dtype=np.float64))]
    with pytest.raises(GhbError):
        ctx.batch_groupby([(None, a, 16, 10), (None, c, 16, 10)], [0], [(abi.SUM, 1)])


def test_device_generator_matches_host_distributions():
    import torch
    specs = workloads.batched_specs(4, seed_idx=36, max_rows=200_000)
    dev_inst = workloads.batched_instances_device(specs, "cuda")
    for s, it in zip(specs, dev_inst):
        keys, qty, price, d = it["cols"]
        assert keys.numel() == s["rows"] and d.dtype == torch.int32
        assert int(qty.min()) >= 1 and int(qty.max()) <= 50
        assert float(price.min()) >= 900.0 and float(price.max()) <= 105000.0
        assert int(d.min()) >= 0 and int(d.max()) < 2526
        assert len(torch.unique(keys)) <= s["groups"]
