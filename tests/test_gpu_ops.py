"""GPU parity: every operator through the C ABI against the CPU oracle.

Bit-exact for keys, counts, integer sums, MIN/MAX, filter rows, join pairs
(as sorted multisets) and sort order; DOUBLE SUM/AVG within 1e-12 relative
of the oracle's Hive-order sequential sum (REL_TOL below).
"""
import json
import os

import numpy as np
import pytest

from ghive_b200 import abi, workloads
from oracle import oracle

pytestmark = pytest.mark.gpu

REL_TOL = 1e-12
EDGE_SIZES = [0, 1, 31, 32, 33, 1023, 1024, 1025, 2047, 2049, 4095, 4097, 100_003]


@pytest.fixture(scope="module")
def ctx():
    from ghive_b200.ops import Context
    c = Context(0)
    yield c
    c.close()


def dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def devcol(c):
    from ghive_b200.ops import Sentinel
    if isinstance(c, Sentinel):
        return Sentinel(dev(c.values))
    if isinstance(c, tuple):
        return (dev(c[0]), dev(c[1].astype(np.uint8)))
    return dev(c)


def host(t):
    return t.cpu().numpy()


def oracle_col(c):
    from ghive_b200.ops import Sentinel
    return c.values if isinstance(c, Sentinel) else c


# ----------------------------------------------------------------- filter
def _check_filter(ctx, pred, cols, sentinel=False):
    ocols = [oracle_col(c) for c in cols]
    sel = oracle.filter_rows(pred, ocols) if not sentinel else \
        oracle.filter_rows(pred, ocols, n=None)
    outs, k = ctx.filter(pred, [devcol(c) for c in cols])
    assert k == len(sel)
    for c, (v, nl) in zip(cols, outs):
        vals = oracle_col(c)
        vals = vals[0] if isinstance(vals, tuple) else vals
        got = host(v)
        exp = vals[sel]
        assert np.array_equal(got.view(np.uint8), exp.view(np.uint8)) if exp.dtype == np.float64 \
            else np.array_equal(got, exp)
        if isinstance(c, tuple):
            assert np.array_equal(host(nl), c[1][sel].astype(bool))


@pytest.mark.parametrize("n", EDGE_SIZES)
def test_filter_edge_sizes(ctx, n):
    g = np.random.default_rng(n + 1)
    cols = [g.integers(0, 2526, n, dtype=np.int32), g.integers(-50, 50, n, dtype=np.int64),
            g.random(n)]
    _check_filter(ctx, abi.Pred.leaf(abi.FILTER_LT, 0, a=1263), cols)


def test_filter_every_mode_and_type(ctx):
    g = np.random.default_rng(5)
    n = 50_000
    cols = [g.integers(-100, 100, n, dtype=np.int32), g.integers(-100, 100, n, dtype=np.int64),
            np.round(g.normal(0, 50, n), 1)]
    for col in range(3):
        for mode in range(abi.FILTER_NOT_NULL + 1):
            lit = (-10.5, 20.0) if col == 2 or mode % 2 else (-10, 20)
            p = abi.Pred.leaf(mode, col, a=lit[0], b=lit[1])
            _check_filter(ctx, p, cols)


def test_filter_tree_and_column_compare(ctx):
    g = np.random.default_rng(6)
    n = 70_001
    cols = [g.integers(0, 100, n, dtype=np.int64), g.integers(0, 100, n, dtype=np.int64),
            g.integers(0, 3, n, dtype=np.int32), g.random(n) * 100]
    p = abi.Pred.or_(abi.Pred.and_(abi.Pred.leaf(abi.FILTER_GT, 0, col2=1),
                                   abi.Pred.leaf(abi.FILTER_EQ, 2, a=0.0)),
                     abi.Pred.leaf(abi.FILTER_EQ_RANGE, 3, a=10.0, b=12.5))
    _check_filter(ctx, p, cols)
    p2 = abi.Pred.leaf(abi.FILTER_LE, 3, col2=0)  # double vs long column
    _check_filter(ctx, p2, cols)


def test_filter_nulls_bytemap_and_sentinel(ctx):
    from ghive_b200.ops import Sentinel
    g = np.random.default_rng(7)
    n = 33_333
    v = g.integers(0, 1000, n, dtype=np.int64)
    isnull = g.random(n) < 0.2
    _check_filter(ctx, abi.Pred.leaf(abi.FILTER_GE, 0, a=500), [(v, isnull)])
    _check_filter(ctx, abi.Pred.leaf(abi.FILTER_NOT_NULL, 0), [(v, isnull)])
    s = v.copy()
    s[isnull] = np.iinfo(np.int64).max
    out, k = ctx.filter(abi.Pred.leaf(abi.FILTER_NOT_NULL, 0), [Sentinel(dev(s))])
    assert k == int((~isnull).sum())
    d = np.where(isnull, np.nan, g.random(n))
    out, k = ctx.filter(abi.Pred.leaf(abi.FILTER_LT, 0, a=0.5), [Sentinel(dev(d))])
    assert k == int(((d < 0.5) & ~np.isnan(d)).sum())


def test_filter_ghive_golden_rows(ctx):
    with open(os.path.join(os.path.dirname(__file__), "golden", "ghive_filter.json")) as f:
        case = json.load(f)["cases"][0]
    cols = [np.array(c[1], dtype={"long": np.int64, "double": np.float64, "int": np.int32}[c[0]])
            for c in case["columns"]]
    pred = abi.Pred.leaf(getattr(abi, case["mode"]), case["col"], a=float(case["literal"]))
    outs, k = ctx.filter(pred, [dev(c) for c in cols])
    rows = [tuple(("%f" % host(v)[i]) if t == abi.DOUBLE else str(host(v)[i])
                  for (v, _), t in zip(outs, case["expected_types"])) for i in range(k)]
    assert rows == [tuple(r) for r in case["expected_rows"]]


def test_filter_ranges_of_several_tiles(ctx):
    """5M rows: each CTA claims a range of several 2048-row tiles (one
    look-back per range), the last range and tile partial.  A one-leaf
    predicate (values loaded before the compares), a tree over a NULL-mapped
    column, and a capacity that runs out inside a range: the rows below it
    are written, the error carries the full count."""
    from ghive_b200._lib import GhbError
    g = np.random.default_rng(8)
    n = 5_000_003
    a = g.integers(0, 2526, n, dtype=np.int32)
    b = g.integers(-(1 << 40), 1 << 40, n, dtype=np.int64)
    bnull = g.random(n) < 0.1
    c = g.random(n)
    _check_filter(ctx, abi.Pred.leaf(abi.FILTER_LT, 0, a=1263), [a, (b, bnull), c])
    tree = abi.Pred.and_(abi.Pred.leaf(abi.FILTER_GE, 1, a=0),
                         abi.Pred.or_(abi.Pred.leaf(abi.FILTER_LT, 2, a=0.3), abi.Pred.leaf(abi.FILTER_EQ, 0, a=7)))
    _check_filter(ctx, tree, [a, (b, bnull), c])
    sel = oracle.filter_rows(tree, [a, (b, bnull), c])
    cap = len(sel) // 3
    from ghive_b200.ops import _Outs
    outs = _Outs([abi.INT, abi.LONG, abi.DOUBLE], cap, "cuda:0")
    with pytest.raises(GhbError) as e:
        ctx.filter(tree, [dev(a), (dev(b), dev(bnull.astype(np.uint8))), dev(c)], capacity=cap, outs=outs)
    assert e.value.code == abi.ERR_CAPACITY
    got = outs.rows(cap)
    assert np.array_equal(host(got[0][0]), a[sel[:cap]]) and np.array_equal(host(got[1][0]), b[sel[:cap]])


def test_filter_capacity_error_reports_required_rows(ctx):
    from ghive_b200._lib import GhbError
    n = 10_000
    cols = [np.arange(n, dtype=np.int64)]
    with pytest.raises(GhbError) as e:
        ctx.filter(abi.Pred.leaf(abi.FILTER_LT, 0, a=5000), [dev(cols[0])], capacity=100)
    assert e.value.code == abi.ERR_CAPACITY
    outs, k = ctx.filter(abi.Pred.leaf(abi.FILTER_LT, 0, a=5000), [dev(cols[0])])
    assert k == 5000  # the context stays usable after the error


# --------------------------------------------------------------- group-by
def _norm_rows(keys, aggs):
    """Rows as tuples sorted by key (NULL first)."""
    n = len(aggs[0][0]) if aggs else len(keys[0][0])
    rows = []
    for i in range(n):
        r = []
        for v, nl in keys + aggs:
            r.append(None if nl[i] else v[i].item())
        rows.append(tuple(r))
    nk = len(keys)
    return sorted(rows, key=lambda r: tuple((x is not None, x if x is not None else 0) for x in r[:nk]))


def _coltype(c):
    v = oracle_col(c)
    v = v[0] if isinstance(v, tuple) else v
    return abi.TYPE_OF_DTYPE[np.dtype(v.dtype)]


def _check_groupby(ctx, pred, cols, keys, aggs, max_groups=None):
    ocols = [oracle_col(c) for c in cols]
    ok, oa = oracle.filter_groupby(pred, ocols, keys, aggs)
    exp = _norm_rows(ok, oa)
    gk, ga, g = ctx.filter_groupby(pred, [devcol(c) for c in cols], keys, aggs,
                                   capacity=max(len(exp), 1) + 16, max_groups=max_groups)
    got = _norm_rows([(host(v), host(nl)) for v, nl in gk], [(host(v), host(nl)) for v, nl in ga])
    assert g == len(exp)
    types = [abi.agg_out_type(t, _coltype(cols[c]) if c >= 0 else abi.LONG) for t, c in aggs]
    for re_, rg in zip(exp, got):
        assert re_[:len(keys)] == rg[:len(keys)]
        for j, (e, x) in enumerate(zip(re_[len(keys):], rg[len(keys):])):
            if e is None or x is None:
                assert e is None and x is None
            elif types[j] == abi.DOUBLE:
                assert abs(x - e) <= REL_TOL * max(abs(e), 1e-300), (e, x)
            else:
                assert x == e
    return g


@pytest.mark.parametrize("n", EDGE_SIZES)
def test_groupby_fact_shape_edge_sizes(ctx, n):
    cols = workloads.fact_table(n, seed_idx=100 + n % 97, groups=1000)
    _check_groupby(ctx, workloads.fact_predicate(), cols, [0], workloads.AGGS_FACT, max_groups=1000)


def test_groupby_fact_shape_300k(ctx):
    cols = workloads.fact_table(300_000, seed_idx=7)
    g = _check_groupby(ctx, workloads.fact_predicate(), cols, [0], workloads.AGGS_FACT, max_groups=1000)
    assert g == 1000


@pytest.mark.parametrize("groups", [1, 7, 64, 5000, 200_000])
def test_groupby_cardinalities_and_skew(ctx, groups):
    g = np.random.default_rng(groups)
    n = 400_000
    keys = workloads.zipf_ranks(g, n, groups, 1.1) * 7919 - 1000
    cols = [keys, g.integers(1, 51, n, dtype=np.int64),
            g.integers(90000, 10500001, n) / 100.0, g.integers(0, 2526, n, dtype=np.int32)]
    _check_groupby(ctx, workloads.fact_predicate(), cols, [0], workloads.AGGS_FACT, max_groups=groups)


def test_groupby_no_keys_and_empty(ctx):
    cols = workloads.fact_table(123_457, seed_idx=9)
    _check_groupby(ctx, workloads.fact_predicate(), cols, [], workloads.AGGS_FACT)
    _check_groupby(ctx, abi.Pred.leaf(abi.FILTER_LT, 3, a=-1), cols, [], workloads.AGGS_FACT)
    _check_groupby(ctx, abi.Pred.leaf(abi.FILTER_LT, 3, a=-1), cols, [0], workloads.AGGS_FACT)


def test_groupby_nulls_keys_and_values(ctx):
    from ghive_b200.ops import Sentinel
    g = np.random.default_rng(11)
    n = 80_000
    k = g.integers(-5, 40, n, dtype=np.int64)
    kn = g.random(n) < 0.1
    v = g.integers(-1000, 1000, n, dtype=np.int64)
    vn = g.random(n) < 0.3
    vn[k == 3] = True  # an all-NULL group: SUM/AVG/MIN/MAX NULL, COUNT(col) 0
    dv = g.random(n) * 100
    dn = g.random(n) < 0.3
    aggs = [(abi.CNT, -1), (abi.CNT, 1), (abi.SUM, 1), (abi.AVG, 1), (abi.MIN, 1), (abi.MAX, 1),
            (abi.SUM, 2), (abi.AVG, 2), (abi.MIN, 2), (abi.MAX, 2)]
    _check_groupby(ctx, None, [(k, kn), (v, vn), (dv, dn)], [0], aggs, max_groups=64)
    ks = k.copy()
    ks[kn] = np.iinfo(np.int64).max
    # sentinel keys: NULL group holds the same rows
    ok, oa = oracle.filter_groupby(None, [(k, kn), v], [0], [(abi.SUM, 1)])
    gk, ga, gg = ctx.filter_groupby(None, [Sentinel(dev(ks)), dev(v)], [0], [(abi.SUM, 1)],
                                    capacity=128, max_groups=64)
    assert gg == len(ok[0][0])
    assert sum(host(nl).sum() for _, nl in gk) == 1


def test_groupby_key_types_and_extremes(ctx):
    g = np.random.default_rng(12)
    n = 50_000
    i64 = np.iinfo(np.int64)
    k = g.choice(np.array([i64.min, i64.min + 1, -1, 0, 1, i64.max - 1], dtype=np.int64), n)
    v = g.choice(np.array([i64.max, i64.min, 1, -1], dtype=np.int64), n)  # SUM wraps
    _check_groupby(ctx, None, [k, v], [0], [(abi.SUM, 1), (abi.MIN, 1), (abi.MAX, 1), (abi.CNT, -1)],
                   max_groups=8)
    kd = g.choice(np.array([-0.5, 0.0, 2.25, 1e300, -1e-300]), n)
    _check_groupby(ctx, None, [kd, v], [0], [(abi.SUM, 1), (abi.CNT, -1)], max_groups=8)
    ki = g.integers(np.iinfo(np.int32).min, np.iinfo(np.int32).max, n, dtype=np.int32) % 1000
    _check_groupby(ctx, None, [ki, v], [0], [(abi.MAX, 1)], max_groups=1000)


def test_groupby_hive_golden_cases(ctx):
    with open(os.path.join(os.path.dirname(__file__), "golden", "hive_groupby.json")) as f:
        cases = json.load(f)["cases"]
    ran = 0
    for case in cases:
        if case.get("key_type") == "string":
            continue
        vals = case["values"] * case.get("repeat", 1)
        vdt = np.float64 if case["value_type"] == "double" else np.int64
        v = np.array([0 if x is None else x for x in vals], dtype=vdt)
        vn = np.array([x is None for x in vals], dtype=bool)
        spec = (abi.CNT, -1) if case["agg"] == "count(*)" else \
            (abi.AGG_NAMES[case["agg"]], 1 if "keys" in case else 0)
        if "keys" not in case:
            gk, ga, g = ctx.filter_groupby(None, [(dev(v), dev(vn.astype(np.uint8)))], [], [spec],
                                           capacity=1)
            val, nl = ga[0]
            got = None if host(nl)[0] else host(val)[0].item()
            assert got == case["expected"], (case["test"], got, case["expected"])
        else:
            ks = case["keys"]
            k = np.array([0 if x is None else x for x in ks], dtype=np.int64)
            kn = np.array([x is None for x in ks], dtype=bool)
            gk, ga, g = ctx.filter_groupby(None, [(dev(k), dev(kn.astype(np.uint8))),
                                                  (dev(v), dev(vn.astype(np.uint8)))], [0], [spec],
                                           capacity=16, max_groups=8)
            got = sorted([(None if host(gk[0][1])[i] else host(gk[0][0])[i].item(),
                           None if host(ga[0][1])[i] else host(ga[0][0])[i].item())
                          for i in range(g)], key=lambda r: (r[0] is not None, r[0] or 0))
            exp = sorted([tuple(p) for p in case["expected"]], key=lambda r: (r[0] is not None, r[0] or 0))
            assert got == exp, case["test"]
        ran += 1
    assert ran >= 50


def test_groupby_ghive_golden_numeric(ctx):
    with open(os.path.join(os.path.dirname(__file__), "golden", "ghive_groupby.json")) as f:
        cases = json.load(f)["cases"]
    for case in cases:
        if any(case["columns"][k][0] == "string" for k in case["keys"]):
            continue
        cols = [np.array(c[1], dtype={"long": np.int64, "double": np.float64, "int": np.int32}[c[0]])
                for c in case["columns"]]
        aggs = [(abi.AGG_NAMES[t.lower()], c) for t, c in case["aggs"]]
        gk, ga, g = ctx.filter_groupby(None, [dev(c) for c in cols], case["keys"], aggs, capacity=64,
                                       max_groups=32)
        rows = sorted(tuple(("%f" % host(v)[i]) if t == abi.DOUBLE else str(host(v)[i])
                            for (v, _), t in zip(gk + ga, case["expected_types"])) for i in range(g))
        assert rows == sorted(tuple(r) for r in case["expected_rows"]), case["test"]


def test_groupby_repeat_is_stable(ctx):
    cols = workloads.fact_table(200_000, seed_idx=13)
    dc = [dev(c) for c in cols]
    first = None
    for _ in range(20):
        gk, ga, g = ctx.filter_groupby(workloads.fact_predicate(), dc, [0], workloads.AGGS_FACT,
                                       capacity=1000, max_groups=1000)
        rows = _norm_rows([(host(v), host(nl)) for v, nl in gk], [(host(v), host(nl)) for v, nl in ga])
        if first is None:
            first = rows
        else:
            for a, b in zip(first, rows):
                assert a[:3] == b[:3] and a[5:] == b[5:]
                assert abs(a[3] - b[3]) <= REL_TOL * abs(a[3])


# ------------------------------------------------------------------- join
def _check_join(ctx, bkey, pkey, jt=abi.INNER_JOIN, bpay=(), ppay=()):
    pr, br = oracle.hash_join(bkey, pkey, jt)
    dbp = [dev(c) for c in bpay]  # the table keeps these columns: they outlive it
    t = ctx.join_build(dev(bkey), build_payload=dbp)
    r = ctx.join_probe(t, dev(pkey), jt, probe_payload=[dev(c) for c in ppay])
    assert r["rows"] == len(pr)
    gp, gb = host(r["probe_rowid"]), host(r["build_rowid"])
    assert np.all(np.diff(gp) >= 0)  # probe-row order
    assert sorted(zip(gp.tolist(), gb.tolist())) == sorted(zip(pr.tolist(), br.tolist()))
    for c, (v, nl) in zip(bpay, r["build"]):
        hv, hn = host(v), host(nl)
        ok = gb >= 0
        assert np.array_equal(hv[ok], c[gb[ok]])
        assert np.all(hn[~ok])
    for c, (v, _) in zip(ppay, r["probe"]):
        assert np.array_equal(host(v), c[gp])
    t.free()
    return r


@pytest.mark.parametrize("n", EDGE_SIZES)
def test_join_edge_sizes(ctx, n):
    g = np.random.default_rng(n + 3)
    nb = max(1, n // 3)
    bkey = g.permutation(np.arange(1, nb + 1, dtype=np.int64))
    pkey = g.integers(0, 2 * nb + 2, n, dtype=np.int64)
    _check_join(ctx, bkey, pkey, bpay=[g.integers(0, 1 << 62, nb, dtype=np.int64), g.random(nb)])


def test_join_config_shape_small(ctx):
    (bkey, bpay), (fk, ppay) = workloads.join_tables(15_000, 600_000, seed_idx=21)
    _check_join(ctx, bkey, fk, bpay=bpay, ppay=[ppay])


def test_join_duplicates_semi_outer_nulls(ctx):
    g = np.random.default_rng(22)
    bkey = g.integers(-50, 50, 5000, dtype=np.int64)  # heavy duplicates
    pkey = g.integers(-80, 80, 40_000, dtype=np.int64)
    pay = g.integers(0, 1000, 5000, dtype=np.int64)
    for jt in (abi.INNER_JOIN, abi.LEFT_SEMI_JOIN, abi.LEFT_OUTER_JOIN):
        _check_join(ctx, bkey, pkey, jt, bpay=[pay] if jt != abi.LEFT_SEMI_JOIN else ())
    i64 = np.iinfo(np.int64)
    bkey2 = np.array([i64.min, 5, i64.max - 1, 7, i64.min], dtype=np.int64)
    pkey2 = np.array([i64.min, 7, 8, i64.max - 1, i64.min, 5], dtype=np.int64)
    _check_join(ctx, bkey2, pkey2)


def test_join_null_keys_never_match(ctx):
    g = np.random.default_rng(23)
    bkey = np.arange(1000, dtype=np.int64)
    bnull = g.random(1000) < 0.2
    pkey = g.integers(0, 1000, 20_000, dtype=np.int64)
    pnull = g.random(20_000) < 0.2
    pr, br = oracle.hash_join((bkey, bnull), (pkey, pnull))
    t = ctx.join_build((dev(bkey), dev(bnull.astype(np.uint8))))
    r = ctx.join_probe(t, (dev(pkey), dev(pnull.astype(np.uint8))))
    assert r["rows"] == len(pr)
    assert sorted(zip(host(r["probe_rowid"]).tolist(), host(r["build_rowid"]).tolist())) == \
        sorted(zip(pr.tolist(), br.tolist()))


def test_join_ghive_semi_outer_chain(ctx):
    with open(os.path.join(os.path.dirname(__file__), "golden", "ghive_join.json")) as f:
        case = json.load(f)["cases"][0]
    tabs = [np.array(t, dtype=np.int64) for t in case["tables"]]
    jt_map = {"LEFT_SEMI_JOIN": abi.LEFT_SEMI_JOIN, "LEFT_OUTER_JOIN": abi.LEFT_OUTER_JOIN}
    tuples = [(i,) for i in range(len(tabs[0]))]
    for name, left, right in case["join_types"]:
        rows = np.array([t[0] for t in tuples], dtype=np.int64)
        t = ctx.join_build(dev(tabs[right]))
        r = ctx.join_probe(t, dev(tabs[0][rows]), jt_map[name])
        pr, br = host(r["probe_rowid"]), host(r["build_rowid"])
        if jt_map[name] == abi.LEFT_SEMI_JOIN:
            tuples = [tuples[p] for p in pr]
        else:
            tuples = [tuples[p] + (int(b),) for p, b in zip(pr, br)]
        t.free()
    exp = case["expected_offsets"]
    w = len(tuples[0])
    assert sorted(tuples) == sorted(tuple(exp[i:i + w]) for i in range(0, len(exp), w))


# ------------------------------------------------------------------- sort
def _check_sort(ctx, keys, orders=None, null_orders=None, payload=(), rowid=True):
    perm = oracle.sort_perm([oracle_col(k) for k in keys], orders, null_orders)
    ok, op, rid = ctx.sort([devcol(k) for k in keys], orders, null_orders,
                           payload=[dev(p) for p in payload], rowid=rowid)
    if rowid:
        assert np.array_equal(host(rid), perm)
    for k, (v, nl) in zip(keys, ok):
        vals, isnull = (k if isinstance(k, tuple) else (k, None))
        hv = host(v)
        if isnull is not None:
            assert np.array_equal(host(nl), isnull[perm])
            m = ~isnull[perm]
            assert np.array_equal(hv[m].view(np.uint8) if hv.dtype == np.float64 else hv[m],
                                  vals[perm][m].view(np.uint8) if hv.dtype == np.float64 else vals[perm][m])
        else:
            assert np.array_equal(hv.view(np.uint8) if hv.dtype == np.float64 else hv,
                                  vals[perm].view(np.uint8) if hv.dtype == np.float64 else vals[perm])
    for p, (v, _) in zip(payload, op):
        assert np.array_equal(host(v), p[perm])


@pytest.mark.parametrize("n", EDGE_SIZES[1:])
def test_sort_edge_sizes(ctx, n):
    d, k, rowid = workloads.sort_table(n, seed_idx=30 + n % 11)
    _check_sort(ctx, [d, k], payload=[rowid], rowid=False)
    _check_sort(ctx, [d, k], rowid=True)


def test_sort_config_shape_and_zipf(ctx):
    for z in (False, True):
        d, k, rowid = workloads.sort_table(300_000, zipf=z, seed_idx=31)
        _check_sort(ctx, [d, k], payload=[rowid], rowid=False)


def test_sort_desc_nulls_doubles(ctx):
    g = np.random.default_rng(33)
    n = 60_000
    a = g.integers(-3, 3, n, dtype=np.int32)
    an = g.random(n) < 0.1
    x = g.choice(np.array([-np.inf, -1.5, -0.0, 0.0, 2.5, np.inf, 1e-300]), n)
    xn = g.random(n) < 0.1
    for orders in ([abi.ASC, abi.DESC], [abi.DESC, abi.ASC]):
        for nulls in ([abi.NULLS_DEFAULT] * 2, [abi.NULLS_LAST, abi.NULLS_FIRST]):
            _check_sort(ctx, [(a, an), (x, xn)], orders, nulls)
    i64 = np.iinfo(np.int64)
    big = g.choice(np.array([i64.min, i64.max, 0, -1, 1], dtype=np.int64), n)
    _check_sort(ctx, [big], [abi.DESC])


def test_sort_all_equal_and_keys_wider_than_64_bits(ctx):
    n = 10_000
    same = np.full(n, 42, dtype=np.int64)
    _check_sort(ctx, [same], payload=[np.arange(n, dtype=np.int32)], rowid=False)
    _check_sort(ctx, [same], rowid=True)
    g = np.random.default_rng(34)
    i64 = np.iinfo(np.int64)
    wide = [g.integers(-3, 3, n, dtype=np.int64),
            g.integers(i64.min, i64.max, n, dtype=np.int64),
            g.integers(i64.min, i64.max, n, dtype=np.int64)]
    isnull = g.random(n) < 0.05
    # three segments: a full-range key with NULLs needs 65 bits on its own
    _check_sort(ctx, [wide[0], (wide[1], isnull), wide[2]], [abi.ASC, abi.DESC, abi.ASC],
                payload=[np.arange(n, dtype=np.int32), g.random(n)])
    _check_sort(ctx, wide[1:], rowid=False, payload=[g.integers(0, 9, n, dtype=np.int64)])


# ------------------------------------------------------- host entry points
def test_host_entry_points_match_device(ctx):
    cols = workloads.fact_table(100_000, seed_idx=40)
    gk, ga, g = ctx.filter_groupby_host(workloads.fact_predicate(), cols, [0], workloads.AGGS_FACT,
                                        capacity=1000, max_groups=1000)
    ok, oa = oracle.filter_groupby(workloads.fact_predicate(), cols, [0], workloads.AGGS_FACT)
    assert g == 1000
    got = _norm_rows(gk, ga)
    exp = _norm_rows(ok, oa)
    for a, b in zip(got, exp):
        assert a[:3] == b[:3] and a[5:] == b[5:]
        assert abs(a[3] - b[3]) <= REL_TOL * abs(b[3])
    outs, k = ctx.filter_host(workloads.fact_predicate(), cols)
    sel = oracle.filter_rows(workloads.fact_predicate(), cols)
    assert k == len(sel) and np.array_equal(outs[3][0], cols[3][sel])
    (bkey, bpay), (fk, ppay) = workloads.join_tables(10_000, 200_000, seed_idx=41)
    r = ctx.hash_join_host(bkey, fk, build_payload=bpay, probe_payload=[ppay])
    pr, br = oracle.hash_join(bkey, fk)
    assert r["rows"] == len(pr)
    assert np.array_equal(r["probe_rowid"], pr) and np.array_equal(r["build_rowid"], br)
    assert np.array_equal(r["build"][0][0], bpay[0][br])
    d, k2, rowid = workloads.sort_table(100_000, seed_idx=42)
    okk, opp, _ = ctx.sort_host([d, k2], payload=[rowid])
    perm = oracle.sort_perm([d, k2])
    assert np.array_equal(opp[0][0], rowid[perm]) and np.array_equal(okk[1][0], k2[perm])


def _pin(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()


def _pinned_outs(types, cap):
    import torch
    from ghive_b200.ops import _Outs
    o = _Outs(types, cap, None)
    keep = []
    for j, t in enumerate(types):
        buf = torch.from_numpy(np.empty(max(1, cap), dtype=abi.NP_DTYPE[t])).pin_memory()
        nb = torch.empty(max(1, cap), dtype=torch.uint8).pin_memory()
        o.cols[j] = (buf.numpy(), nb.numpy())
        o.arr[j].data, o.arr[j].is_null = buf.data_ptr(), nb.data_ptr()
        keep += [buf, nb]
    o._pinned = keep
    return o


def test_filter_host_pinned_chunks(ctx):
    """Pinned host columns of 3.3M rows take the chunked host path (chunks
    copied in, filtered and copied out on three streams): the same rows in
    the same order as the oracle, a BYTEMAP input's NULLs carried, an
    output capacity below the row count refused with the full count, and
    pageable columns (one copy in, one out) giving the same rows."""
    from ghive_b200._lib import GhbError
    g = np.random.default_rng(43)
    n = 3_300_001
    a = g.integers(0, 2526, n, dtype=np.int32)
    b = g.integers(-(1 << 40), 1 << 40, n, dtype=np.int64)
    bnull = g.random(n) < 0.1
    c = g.random(n)
    pred = abi.Pred.or_(abi.Pred.leaf(abi.FILTER_LT, 0, a=700), abi.Pred.leaf(abi.FILTER_GT, 2, a=0.9))
    sel = oracle.filter_rows(pred, [a, (b, bnull), c])
    types = [abi.INT, abi.LONG, abi.DOUBLE]
    for cols in ([_pin(a), (_pin(b), _pin(bnull.astype(np.uint8))), _pin(c)], [a, (b, bnull), c]):
        outs = _pinned_outs(types, n)
        got, k = ctx.filter_host(pred, cols, outs=outs)
        assert k == len(sel)
        assert np.array_equal(got[0][0], a[sel]) and np.array_equal(got[1][0], b[sel])
        assert np.array_equal(got[2][0].view(np.uint8), c[sel].view(np.uint8))
        assert np.array_equal(got[1][1], bnull[sel]) and not got[0][1].any()
    cap = len(sel) // 2
    with pytest.raises(GhbError) as e:
        ctx.filter_host(pred, [_pin(a), (_pin(b), _pin(bnull.astype(np.uint8))), _pin(c)], capacity=cap,
                        outs=_pinned_outs(types, cap))
    assert e.value.code == abi.ERR_CAPACITY
    outs, k = ctx.filter_host(pred, [a, (b, bnull), c], proj=[2])
    assert k == len(sel) and np.array_equal(outs[0][0].view(np.uint8), c[sel].view(np.uint8))


@pytest.mark.parametrize("max_groups", [8, 1000])
def test_groupby_narrow_shared_accumulators(ctx, max_groups):
    """The specialised fold keeps COUNT as u32, integer SUM as a u32 pair with
    carry, INT MIN/MAX as u32 images and INT keys as u32 images in shared
    memory: extremes of every form, carries out of the low word, all-NULL
    groups, with and without warp combining (few / many groups), and the
    keyless warp reduction."""
    g = np.random.default_rng(31)
    n = 200_000
    i32, i64 = np.iinfo(np.int32), np.iinfo(np.int64)
    kv = np.array([i32.min, i32.min + 1, -1, 0, 1, i32.max - 1, i32.max], dtype=np.int32)
    k = kv[g.integers(0, len(kv), n)] if max_groups == 8 else \
        np.concatenate([kv, g.integers(i32.min, i32.max, n - len(kv), dtype=np.int32) % 997 - 498]).astype(np.int32)
    iv = g.choice(np.array([i32.min, i32.max, -1, 0, 1, 12345], dtype=np.int32), n)
    ivn = g.random(n) < 0.2
    ivn[k == 1] = True  # an all-NULL group for the INT aggregates
    lv = g.choice(np.array([0xFFFFFFFF, 0x100000000, -1, -0xFFFFFFFF, i64.max, i64.min, 7], dtype=np.int64), n)
    dv = g.random(n) * 1000 - 300
    aggs = [(abi.CNT, -1), (abi.CNT, 1), (abi.SUM, 1), (abi.MIN, 1), (abi.MAX, 1), (abi.AVG, 1),
            (abi.SUM, 2), (abi.MIN, 2), (abi.MAX, 2), (abi.SUM, 3), (abi.AVG, 3)]
    cols = [k, (iv, ivn), lv, dv]
    _check_groupby(ctx, None, cols, [0], aggs, max_groups=max_groups)
    _check_groupby(ctx, abi.Pred.leaf(abi.FILTER_GT, 3, a=0.0), cols, [0], aggs, max_groups=max_groups)
    _check_groupby(ctx, abi.Pred.leaf(abi.FILTER_GT, 3, a=0.0), cols, [], aggs)
    # INT values without NULLs: an extreme that is the only value of its group
    only = np.array([i32.min] * 50 + [i32.max] * 50, dtype=np.int32)
    kk = np.array([5] * 50 + [6] * 50, dtype=np.int32)
    _check_groupby(ctx, None, [kk, only], [0], [(abi.MIN, 1), (abi.MAX, 1), (abi.SUM, 1)],
                   max_groups=max_groups)
    _check_groupby(ctx, None, [kk[:50], only[:50]], [], [(abi.MIN, 1), (abi.MAX, 1)])
    _check_groupby(ctx, None, [kk[50:], only[50:]], [], [(abi.MIN, 1), (abi.MAX, 1)])


@pytest.mark.parametrize("dense", [True, False])
def test_join_direct_and_hashed_tables(ctx, dense):
    """Dense build keys (a range at most twice the rows) get a direct table
    (slot = key - min); sparse keys the hashed one.  Both with duplicates,
    every join type, INT and LONG keys, probe keys outside the range."""
    g = np.random.default_rng(24 + int(dense))
    n, m = 50_000, 200_000
    if dense:
        bkey = g.permutation(np.arange(-1000, -1000 + n, dtype=np.int64))
        pkey = g.integers(-3000, n + 2000, m, dtype=np.int64)
    else:
        bkey = g.integers(-(1 << 62), 1 << 62, n, dtype=np.int64)
        hit = bkey[g.integers(0, n, m)]
        pkey = np.where(g.random(m) < 0.7, hit, g.integers(-(1 << 62), 1 << 62, m, dtype=np.int64))
    bkey[:500] = bkey[500:1000]  # keys twice in the build
    pay = [g.integers(0, 1 << 40, n, dtype=np.int64), g.random(n)]
    for jt in (abi.INNER_JOIN, abi.LEFT_SEMI_JOIN, abi.LEFT_OUTER_JOIN):
        _check_join(ctx, bkey, pkey, jt, bpay=pay if jt != abi.LEFT_SEMI_JOIN else ())
    t = ctx.join_build(dev(bkey))
    rows, dup, slots = t.info()
    assert rows == n and dup == 2
    if dense:
        assert slots == int(bkey.max() - bkey.min() + 1)
    else:
        assert slots & (slots - 1) == 0
    t.free()
    if dense:  # INT keys
        _check_join(ctx, bkey.astype(np.int32), pkey.astype(np.int32), bpay=pay)


def test_join_many_chunks(ctx):
    """A probe of more than 4096 1024-row chunks: the chunk offsets come from
    the multi-CTA look-back scan.  Pairs compared as sorted arrays."""
    g = np.random.default_rng(26)
    nb, m = 100_000, 6_000_000
    bkey = g.permutation(np.arange(1, nb + 1, dtype=np.int64))
    bkey[:1000] = bkey[1000:2000]  # some keys twice
    pkey = g.integers(0, nb + 5000, m, dtype=np.int64)
    pr, br = oracle.hash_join(bkey, pkey, abi.INNER_JOIN)
    t = ctx.join_build(dev(bkey))
    r = ctx.join_probe(t, dev(pkey), abi.INNER_JOIN)
    assert r["rows"] == len(pr)
    gp, gb = host(r["probe_rowid"]).astype(np.int64), host(r["build_rowid"]).astype(np.int64)
    assert np.all(np.diff(gp) >= 0)
    o1, o2 = np.lexsort((gb, gp)), np.lexsort((br, pr))
    assert np.array_equal(gp[o1], pr[o2]) and np.array_equal(gb[o1], br[o2])
    t.free()


# --------------------------------------------------- several GROUP BY keys
@pytest.mark.parametrize("nkeys", [2, 3])
def test_groupby_several_keys_fact_shape(ctx, nkeys):
    """GROUP BY (k, d % 7[, qty]) over the fact table: the keys of a row are
    packed into one int64 value on the device and unpacked into the key
    output columns; results equal the oracle's Hive group-by."""
    k, qty, price, d = workloads.fact_table(600_000, seed_idx=60, groups=200)
    dow = (d % 7).astype(np.int32)
    cols = [k, qty, price, d, dow]
    keys = [0, 4] if nkeys == 2 else [0, 4, 1]
    g = 200 * 7 * (50 if nkeys == 3 else 1)
    got = _check_groupby(ctx, workloads.fact_predicate(), cols, keys, workloads.AGGS_FACT, max_groups=g)
    assert got > 1000


def test_groupby_several_keys_nulls_types_and_extremes(ctx):
    g = np.random.default_rng(61)
    n = 120_000
    i32, i64 = np.iinfo(np.int32), np.iinfo(np.int64)
    a = g.choice(np.array([i32.min, -1, 0, 7, i32.max - 1], dtype=np.int32), n)   # INT, full range
    an = g.random(n) < 0.1
    b = g.integers(-3, 3, n, dtype=np.int64)                                       # LONG, small
    bn = g.random(n) < 0.1
    c = np.round(g.integers(0, 5, n) * 0.25 - 0.5, 2)                              # DOUBLE, few values
    v = g.integers(-1000, 1000, n, dtype=np.int64)
    aggs = [(abi.CNT, -1), (abi.SUM, 3), (abi.MIN, 3), (abi.MAX, 3), (abi.AVG, 3)]
    cols = [(a, an), (b, bn), c, v]
    _check_groupby(ctx, None, cols, [0, 1, 2], aggs, max_groups=5 * 7 * 5)
    _check_groupby(ctx, abi.Pred.leaf(abi.FILTER_GT, 3, a=0), cols, [2, 0], aggs, max_groups=64)
    # a key column that is all NULL, and one constant column
    allnull = np.ones(n, dtype=bool)
    _check_groupby(ctx, None, [(b, allnull), np.full(n, 5, dtype=np.int64), v], [0, 1],
                   [(abi.SUM, 2)], max_groups=4)
    # empty input
    _check_groupby(ctx, None, [b[:0], c[:0], v[:0]], [0, 1], [(abi.SUM, 2)], max_groups=4)


def test_groupby_several_keys_too_wide_to_pack(ctx):
    """Key tuples whose ranges need more than 63 bits (two full-range LONG
    keys, a DOUBLE key of both signs beside them) are grouped by the row of
    each tuple's first occurrence instead of a packed key."""
    g = np.random.default_rng(62)
    n = 60_000
    i64 = np.iinfo(np.int64)
    a = g.integers(i64.min, i64.max, 300, dtype=np.int64)[g.integers(0, 300, n)]
    b = g.integers(i64.min, i64.max, 7, dtype=np.int64)[g.integers(0, 7, n)]
    bn = g.random(n) < 0.1
    c = g.normal(0, 1e6, 5)[g.integers(0, 5, n)]
    v = g.integers(-1000, 1000, n, dtype=np.int64)
    aggs = [(abi.CNT, -1), (abi.SUM, 3), (abi.MIN, 3)]
    _check_groupby(ctx, None, [a, (b, bn), c, v], [0, 1], aggs, max_groups=300 * 8)
    _check_groupby(ctx, abi.Pred.leaf(abi.FILTER_GT, 3, a=0), [a, (b, bn), c, v], [2, 0, 1], aggs,
                   max_groups=300 * 8 * 5)


def test_groupby_several_keys_host_entry_point(ctx):
    k, qty, price, d = workloads.fact_table(200_000, seed_idx=63, groups=50)
    cols = [k, qty, price, d, (d % 3).astype(np.int32)]
    gk, ga, g = ctx.filter_groupby_host(workloads.fact_predicate(), cols, [0, 4], workloads.AGGS_FACT,
                                        capacity=256, max_groups=150)
    ok, oa = oracle.filter_groupby(workloads.fact_predicate(), cols, [0, 4], workloads.AGGS_FACT)
    assert g == len(ok[0][0]) == 150
    got, exp = _norm_rows(gk, ga), _norm_rows(ok, oa)
    for a_, b_ in zip(got, exp):
        assert a_[:4] == b_[:4] and a_[6:] == b_[6:]
        assert abs(a_[4] - b_[4]) <= REL_TOL * abs(b_[4])
        assert abs(a_[5] - b_[5]) <= REL_TOL * abs(b_[5])


# --------------------------------------- host-buffer join in pipelined chunks
@pytest.mark.parametrize("jt", [abi.INNER_JOIN, abi.LEFT_OUTER_JOIN])
def test_host_join_in_chunks(ctx, jt):
    """ghb_hash_join_host probes in 8M-row chunks whose copies in and out
    overlap the kernels: a 17M-row probe (three chunks, the last partial)
    with duplicated build keys, a probe payload and both row-id outputs
    equals the oracle's pairs, in probe-row order."""
    g = np.random.default_rng(80 + jt)
    nb, m = 100_000, 17_000_000
    bkey = g.permutation(np.arange(1, nb + 1, dtype=np.int64))
    bkey[:500] = bkey[500:1000]                       # keys twice in the build
    pkey = g.integers(0, nb + 20_000, m, dtype=np.int64)
    bpay = [g.integers(0, 1 << 40, nb, dtype=np.int64), g.random(nb)]
    ppay = g.integers(-1000, 1000, m, dtype=np.int64).astype(np.int32)
    r = ctx.hash_join_host(bkey, pkey, jt, build_payload=bpay, probe_payload=[ppay],
                           capacity=m + m // 50)
    pr, br = oracle.hash_join(bkey, pkey, jt)
    assert r["rows"] == len(pr)
    gp, gb = r["probe_rowid"].astype(np.int64), r["build_rowid"].astype(np.int64)
    assert np.all(np.diff(gp) >= 0)
    o1, o2 = np.lexsort((gb, gp)), np.lexsort((br, pr))
    gp, gb, pr, br = gp[o1], gb[o1], pr[o2].astype(np.int64), br[o2].astype(np.int64)
    assert np.array_equal(gp, pr) and np.array_equal(gb, br)
    hit = gb >= 0
    (v0, n0), (v1, n1) = r["build"]
    assert np.array_equal(v0[o1][hit], bpay[0][gb[hit]]) and np.all(n0[o1][~hit])
    assert np.array_equal(v1[o1][hit].view(np.uint64), bpay[1][gb[hit]].view(np.uint64))
    assert np.array_equal(r["probe"][0][0][o1], ppay[gp])


def test_host_join_in_chunks_short_output(ctx):
    from ghive_b200._lib import GhbError
    (bkey, bpay), (fk, _) = workloads.join_tables(50_000, 9_000_000, seed_idx=81)
    with pytest.raises(GhbError) as e:
        ctx.hash_join_host(bkey, fk, build_payload=bpay, capacity=1_000_000)
    assert e.value.code == abi.ERR_CAPACITY
    r = ctx.hash_join_host(bkey, fk, build_payload=bpay, capacity=9_000_000)
    pr, br = oracle.hash_join(bkey, fk)
    assert r["rows"] == len(pr) and np.array_equal(r["probe_rowid"], pr)
    assert np.array_equal(r["build"][0][0], bpay[0][br])


# ---------------------------------------------------------------- strings
def _strings(values):
    """("string", utf-8 bytes, int32 [start,end) pairs) of a list of str/None
    (None: NULL as (-1, -1), GTable.java:240-257)."""
    chars, idx, pos = bytearray(), [], 0
    for v in values:
        if v is None:
            idx += [-1, -1]
            continue
        b = v.encode()
        idx += [pos, pos + len(b)]
        chars += b
        pos += len(b)
    return ("string", bytes(chars) or b"\0", np.array(idx, dtype=np.int32))


def _dev_strings(s):
    import torch
    return ("string", torch.frombuffer(bytearray(s[1]), dtype=torch.uint8).cuda(), dev(s[2]))


def _decode(col_str, pairs):
    b = col_str[1]
    p = pairs.reshape(-1, 2)
    return [None if s < 0 else b[s:e].decode() for s, e in p]


def _words(g, n, nulls=0.1):
    pool = ["", "a", "ab", "abc", "b", "MFGR#12", "MFGR#1221", "MFGR#1238", "zz", "été", "Z", "abd"]
    return [None if g.random() < nulls else pool[g.integers(0, len(pool))] for _ in range(n)]


def test_filter_string_predicates_every_mode_and_projection(ctx):
    g = np.random.default_rng(95)
    n = 40_000
    words = _words(g, n)
    s = _strings(words)
    v = g.integers(-100, 100, n, dtype=np.int64)
    ds = _dev_strings(s)
    for mode in range(abi.FILTER_NOT_NULL + 1):
        for a, b in (("ab", "b"), ("MFGR#12", "MFGR#1238"), ("", "zz"), ("é", "été~")):
            p = abi.Pred.leaf(mode, 0, a=a, b=b)
            sel = oracle.filter_rows(p, [s, v])
            outs, k = ctx.filter(p, [ds, dev(v)], proj=[1, 0])
            assert k == len(sel), (mode, a, b)
            assert np.array_equal(host(outs[0][0]), v[sel])
            assert _decode(s, host(outs[1][0])) == [words[i] for i in sel]
    # a STRING leaf inside a tree with a numeric one, and column vs column
    t = _strings(_words(g, n, 0.05))
    p = abi.Pred.and_(abi.Pred.leaf(abi.FILTER_GE, 0, a="abc"), abi.Pred.leaf(abi.FILTER_LT, 1, a=50))
    sel = oracle.filter_rows(p, [s, v])
    _, k = ctx.filter(p, [ds, dev(v)])
    assert k == len(sel)
    p2 = abi.Pred.leaf(abi.FILTER_LT, 0, col2=2)
    sel = oracle.filter_rows(p2, [s, v, t])
    _, k = ctx.filter(p2, [ds, dev(v), _dev_strings(t)])
    assert k == len(sel)


@pytest.mark.parametrize("with_pred", [False, True])
def test_groupby_string_keys(ctx, with_pred):
    """GROUP BY a STRING key, and (INT, STRING) keys: each STRING key becomes
    the row of its value's first occurrence on the device; the output holds
    [start,end) pairs into the key column's bytes."""
    g = np.random.default_rng(96 + with_pred)
    n = 150_000
    words = _words(g, n)
    s = _strings(words)
    year = g.integers(1992, 1999, n, dtype=np.int32)
    rev = g.integers(1, 10_000_000, n) / 100.0
    qty = g.integers(1, 51, n, dtype=np.int64)
    pred = abi.Pred.leaf(abi.FILTER_GT, 3, a=10) if with_pred else None
    aggs = [(abi.CNT, -1), (abi.SUM, 3), (abi.SUM, 2), (abi.AVG, 2), (abi.MAX, 1)]
    ds = _dev_strings(s)
    for keys in ([0], [1, 0]):
        exp = oracle.groupby_string_key([s, year, rev, qty], keys, aggs) if not with_pred else None
        if with_pred:
            m = qty > 10
            exp = oracle.groupby_string_key([_strings([w for w, k in zip(words, m) if k]), year[m], rev[m],
                                             qty[m]], keys, aggs)
        gk, ga, ng = ctx.filter_groupby(pred, [ds, dev(year), dev(rev), dev(qty)], keys, aggs,
                                        capacity=256, max_groups=200)
        assert ng == len(exp)
        kcols = []
        for j, k in enumerate(keys):
            if k == 0:
                kcols.append(_decode(s, host(gk[j][0])[:2 * ng]))
            else:
                vals, nl = host(gk[j][0]), host(gk[j][1])
                kcols.append([None if nl[i] else int(vals[i]) for i in range(ng)])
        rows = []
        for i in range(ng):
            r = [kc[i] for kc in kcols]
            for v, nl in ga:
                r.append(None if host(nl)[i] else host(v)[i].item())
            rows.append(tuple(r))
        key = lambda r: tuple((x is not None, x if x is not None else "") for x in r[:len(keys)])  # noqa: E731
        got, want = sorted(rows, key=key), sorted(exp, key=key)
        for a, b in zip(got, want):
            assert a[:len(keys) + 2] == b[:len(keys) + 2] and a[-1] == b[-1], (a, b)
            for x, y in zip(a[len(keys) + 2:-1], b[len(keys) + 2:-1]):
                assert abs(x - y) <= REL_TOL * abs(y)


def test_groupby_ghive_golden_string_keys(ctx):
    """GHive's shouldSuccess (one STRING key) and multipleKeysTest (INT and
    STRING keys) through the GPU: Table::toString rows as the test expects."""
    with open(os.path.join(os.path.dirname(__file__), "golden", "ghive_groupby.json")) as f:
        cases = json.load(f)["cases"]
    ran = 0
    for case in cases:
        if not any(case["columns"][k][0] == "string" for k in case["keys"]):
            continue
        cols, hcols = [], []
        for c in case["columns"]:
            if c[0] == "string":
                chars = c[1].encode()
                hc = ("string", chars, np.array(c[2], dtype=np.int32))
                hcols.append(hc)
                cols.append(_dev_strings(hc))
            else:
                a = np.array(c[1], dtype={"long": np.int64, "double": np.float64, "int": np.int32}[c[0]])
                hcols.append(a)
                cols.append(dev(a))
        aggs = [(abi.AGG_NAMES[t.lower()], c) for t, c in case["aggs"]]
        gk, ga, g = ctx.filter_groupby(None, cols, case["keys"], aggs, capacity=64, max_groups=32)
        out = []
        for j, k in enumerate(case["keys"]):
            if case["columns"][k][0] == "string":
                out.append(_decode(hcols[k], host(gk[j][0])[:2 * g]))
            else:
                out.append([str(x) for x in host(gk[j][0])[:g]])
        for (v, _), t in zip(ga, case["expected_types"][len(case["keys"]):]):
            out.append([("%f" % x) if t == abi.DOUBLE else str(x) for x in host(v)[:g]])
        rows = sorted(tuple(col[i] for col in out) for i in range(g))
        assert rows == sorted(tuple(r) for r in case["expected_rows"]), case["test"]
        ran += 1
    assert ran == 2


@pytest.mark.parametrize("full", [True, False])
@pytest.mark.parametrize("key_int", [False, True])
def test_join_lean_pass_on_direct_tables(ctx, full, key_int):
    """The lean write pass (INNER, unique build keys, inline payloads, no
    build row ids) on a direct table reads each probe key again instead of a
    slot array: with every key of the range present (a full table, no table
    load in the count pass) and with holes in the range; NULL probe keys and
    keys outside the range match nothing."""
    import torch
    from ghive_b200.ops import _Outs
    g = np.random.default_rng(97 + 2 * full + key_int)
    nb, m = 40_000, 700_000
    dt = np.int32 if key_int else np.int64
    if full:
        bkey = g.permutation(np.arange(-500, nb - 500)).astype(dt)
    else:
        bkey = g.choice(np.arange(-500, int(1.3 * nb) - 500), nb, replace=False).astype(dt)
    pay = [g.integers(0, 1 << 40, nb, dtype=np.int64), g.random(nb)]
    pkey = g.integers(-2000, int(1.4 * nb), m).astype(dt)
    pnull = g.random(m) < 0.03
    pr, br = oracle.hash_join(bkey, (pkey, pnull))
    t = ctx.join_build(dev(bkey), build_payload=[dev(c) for c in pay])
    ob = _Outs([abi.LONG, abi.DOUBLE], m, "cuda:0", with_nulls=False)
    op = _Outs([], m, "cuda:0")
    prow = torch.empty(m, dtype=torch.int32, device="cuda:0")
    d_rows = torch.zeros(1, dtype=torch.int64, device="cuda:0")
    ctx.join_probe(t, (dev(pkey), dev(pnull.astype(np.uint8))), abi.INNER_JOIN, capacity=m, rowids=False,
                   outs=(ob, op, prow, None, d_rows))
    k = int(d_rows.item())
    assert k == len(pr)
    assert np.array_equal(host(prow[:k]), pr)
    assert np.array_equal(host(ob.cols[0][0][:k]), pay[0][br])
    assert np.array_equal(host(ob.cols[1][0][:k]).view(np.uint64), pay[1][br].view(np.uint64))
    _, _, slots = t.info()
    assert slots == int(bkey.max()) - int(bkey.min()) + 1   # a direct table
    t.free()


def test_sort_string_keys(ctx):
    """ORDER BY a STRING key (Hive's unsigned byte order, then length; NULLs
    first for ASC) and a STRING key behind an INT key, ASC and DESC: the sort
    runs on each string's 8-byte parts and length, and the STRING outputs are
    [start,end) pairs gathered by row id."""
    g = np.random.default_rng(98)
    n = 90_000
    pool = ["", "a", "a\x00", "ab", "abc", "abcdefgh", "abcdefghi", "abcdefgh\x01", "MFGR#1221",
            "MFGR#12", "zz", "été", "Z", "b" * 23]
    words = [None if g.random() < 0.07 else pool[g.integers(0, len(pool))] for _ in range(n)]
    s = _strings(words)
    yr = g.integers(1992, 1995, n, dtype=np.int32)
    rid = np.arange(n, dtype=np.int32)
    ds = _dev_strings(s)
    for keys, hkeys, orders in (([ds], [s], [abi.ASC]), ([ds], [s], [abi.DESC]),
                                ([dev(yr), ds], [yr, s], [abi.DESC, abi.ASC])):
        perm = oracle.sort_perm(hkeys, orders)
        ok, op, _ = ctx.sort(keys, orders, payload=[dev(rid)])
        assert np.array_equal(host(op[0][0]), perm), orders
        got = _decode(s, host(ok[-1][0]))
        assert got == [words[i] for i in perm]
