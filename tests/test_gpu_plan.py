"""A vertex's operator chain on device-resident intermediates, fed the way
GHive's JNI entry point is fed (a GTables object) and answered the way it
answers (GPUResult's arrays grouped by type, plus sequence).

Each chain's result equals the oracle's Hive operators applied one after the
other: bit-exact for keys, counts, integer sums, MIN/MAX and row order;
DOUBLE SUM/AVG within REL_TOL of the oracle's sequential sums.
"""
import numpy as np
import pytest

from ghive_b200 import abi, workloads
from ghive_b200.gtables import GTables, op_filter, op_groupby, op_join, op_sort, run_plan
from oracle import oracle

pytestmark = pytest.mark.gpu

REL_TOL = 1e-12


@pytest.fixture(scope="module")
def ctx():
    from ghive_b200.ops import Context
    c = Context(0)
    yield c
    c.close()


def _sequence(types):
    base = {0: 0, 1: types.count(0), 2: types.count(0) + types.count(1)}
    seen = {0: 0, 1: 0, 2: 0}
    out = []
    for t in types:
        out.append(base[t] + seen[t])
        seen[t] += 1
    return out


def _assert_cols(got, exp, types):
    for j, ((gv, gn), (ev, en)) in enumerate(zip(got, exp)):
        assert np.array_equal(gn, en), j
        if types[j] == abi.DOUBLE:
            e, g = ev[~en], gv[~gn]
            assert np.all(np.abs(g - e) <= REL_TOL * np.maximum(np.abs(e), 1e-300)), j
        else:
            assert np.array_equal(gv[~gn], ev[~en]), j


def test_filter_groupby_sort_chain(ctx):
    """TableScan -> Filter (d < 1263) -> GroupBy k -> Sink ORDER BY k DESC."""
    cols = workloads.fact_table(2_000_000, seed_idx=90, groups=700)
    gt = GTables([("Map 1", 0, cols)])
    pred = workloads.fact_predicate()
    aggs = workloads.AGGS_FACT
    r = run_plan(ctx, gt, 0, [op_filter(pred), op_groupby([0], aggs, max_groups=700),
                              op_sort([0], orders=[abi.DESC])])
    ok, oa = oracle.filter_groupby(pred, cols, [0], aggs)
    exp = [(c[0][::-1], c[1][::-1]) for c in ok + oa]   # the oracle orders groups by key ASC
    assert r["rows"] == 700
    types = [abi.INT, abi.LONG, abi.LONG, abi.DOUBLE, abi.DOUBLE, abi.INT, abi.INT]
    assert r["types"] == types
    _assert_cols(r["columns"], exp, types)
    assert r["sequence"] == _sequence(types)
    assert len(r["longCols"]) == 2 and len(r["doubleCols"]) == 2 and len(r["intCols"]) == 3


def test_join_groupby_chain_with_two_input_tables(ctx):
    """A map-join vertex: the fact table (input 0) probes a dimension table
    (input 1, key + attribute), then GROUP BY the attribute, ORDER BY it."""
    g = np.random.default_rng(91)
    nd, nf = 5_000, 1_500_000
    dkey = g.permutation(np.arange(1, nd + 1, dtype=np.int64))
    dattr = g.integers(0, 40, nd, dtype=np.int32)
    fk = g.integers(1, nd + 500, nf, dtype=np.int64)
    qty = g.integers(1, 51, nf, dtype=np.int64)
    price = g.integers(90000, 10500001, nf) / 100.0
    gt = GTables([("Map 1", 0, [fk, qty, price]), ("Map 2", 1, [dkey, dattr])])
    aggs = [(abi.CNT, -1), (abi.SUM, 1), (abi.AVG, 2)]
    r = run_plan(ctx, gt, 0, [op_join(0, 1, 0, build_keep=[1]),          # -> fk, qty, price, attr
                              op_groupby([3], aggs, max_groups=64), op_sort([0])])
    pr, br = oracle.hash_join(dkey, fk)
    joined = [fk[pr], qty[pr], price[pr], dattr[br]]
    ok, oa = oracle.filter_groupby(None, joined, [3], aggs)
    types = [abi.INT, abi.LONG, abi.LONG, abi.DOUBLE]
    assert r["rows"] == len(ok[0][0]) == 40
    _assert_cols(r["columns"], ok + oa, types)
    assert r["sequence"] == _sequence(types)


def test_semi_join_filter_projection_chain(ctx):
    g = np.random.default_rng(92)
    keys = np.arange(0, 2000, 3, dtype=np.int64)
    fk = g.integers(0, 2000, 300_000, dtype=np.int64)
    v = g.integers(-50, 50, 300_000, dtype=np.int64)
    gt = GTables([("Map 1", 0, [fk, v]), ("Map 2", 0, [keys])])
    r = run_plan(ctx, gt, 0, [op_join(0, 1, 0, join_type=abi.LEFT_SEMI_JOIN),
                              op_filter(abi.Pred.leaf(abi.FILTER_GT, 1, a=0), proj=[1, 0])])
    m = np.isin(fk, keys) & (v > 0)
    assert r["rows"] == int(m.sum())
    assert np.array_equal(r["columns"][0][0], v[m]) and np.array_equal(r["columns"][1][0], fk[m])


def test_missing_input_table_is_refused(ctx):
    from ghive_b200._lib import GhbError
    gt = GTables([("Map 1", 0, [np.arange(10, dtype=np.int64)]), (None, 0, [np.arange(3, dtype=np.int64)])])
    with pytest.raises(GhbError) as e:
        run_plan(ctx, gt, 0, [op_join(0, 1, 0)])
    assert e.value.code == abi.ERR_INVALID
    r = run_plan(ctx, gt, 0, [op_sort([0], orders=[abi.DESC])])
    assert np.array_equal(r["columns"][0][0], np.arange(10)[::-1])


def test_three_table_chain_with_two_column_keys(ctx):
    """An N-way map-join chain (SortMergeJoinPredicate.cu:257-454 joins each
    further table to the tuples so far): lineorder probes a (year, month)
    calendar on two key columns, then a supplier table on one, then GROUP BY
    the calendar's quarter and the supplier's region."""
    g = np.random.default_rng(93)
    n = 400_000
    year = g.integers(1992, 1999, n, dtype=np.int32)
    month = g.integers(1, 13, n, dtype=np.int32)
    supp = g.integers(0, 2_200, n, dtype=np.int64)
    rev = g.integers(1, 100_000, n, dtype=np.int64)
    cy = np.repeat(np.arange(1992, 1998, dtype=np.int32), 12)        # 1998 missing: no match
    cm = np.tile(np.arange(1, 13, dtype=np.int32), 6)
    cq = ((cm - 1) // 3 + 1).astype(np.int32)
    skey = np.arange(0, 2_000, dtype=np.int64)                        # keys >= 2000 missing
    sreg = g.integers(0, 5, 2_000, dtype=np.int32)
    gt = GTables([("Map 1", 0, [year, month, supp, rev]), ("Map 2", 2, [cy, cm, cq]),
                  ("Map 3", 1, [skey, sreg])])
    aggs = [(abi.CNT, -1), (abi.SUM, 3)]
    r = run_plan(ctx, gt, 0, [op_join([0, 1], 1, [0, 1], build_keep=[2]),
                              op_join(2, 2, 0, build_keep=[1]),            # + quarter (4), region (5)
                              op_groupby([4, 5], aggs, max_groups=64), op_sort([0, 1])])
    cal = {(y, m): q for y, m, q in zip(cy, cm, cq)}
    reg = dict(zip(skey.tolist(), sreg.tolist()))
    exp = {}
    for y, m, s, v in zip(year.tolist(), month.tolist(), supp.tolist(), rev.tolist()):
        if (y, m) in cal and s in reg:
            k = (int(cal[(y, m)]), reg[s])
            c, t = exp.get(k, (0, 0))
            exp[k] = (c + 1, t + v)
    keys = sorted(exp)
    assert r["rows"] == len(keys)
    (q, _), (rg, _), (cnt, _), (sm, _) = r["columns"]
    assert list(zip(q.tolist(), rg.tolist())) == keys
    assert cnt.tolist() == [exp[k][0] for k in keys] and sm.tolist() == [exp[k][1] for k in keys]


def _strings(vals):
    """A GTables string column from a list of bytes (None = NULL): the bytes
    packed in row order and int32 [start,end) pairs, -1,-1 for NULL."""
    blob, pairs, at = bytearray(), [], 0
    for v in vals:
        if v is None:
            pairs += [-1, -1]
            continue
        blob += v
        pairs += [at, at + len(v)]
        at += len(v)
    return ("string", bytes(blob), np.array(pairs, dtype=np.int32))


def test_string_columns_through_filter_join_groupby_sort(ctx):
    """STRING columns on the whole chain: a predicate on a STRING column, a
    join on a STRING key keeping a STRING attribute of the build side, then
    GROUP BY (attribute, city) and ORDER BY both; the strings come back
    packed with their pairs the way GPUResult's String[][] is filled."""
    g = np.random.default_rng(94)
    n = 200_000
    cities = [b"AMSTERDAM", b"BERLIN", b"CAIRO", b"CALGARY", b"DELHI", b"", b"\xc3\xa9VORA"]
    cats = [b"MFGR#%d" % i for i in range(1, 41)]
    city = [None if x < 0 else cities[x] for x in g.integers(-1, len(cities), n).tolist()]
    # category keys: NULLs, the 40 categories, and some no dimension row has
    cat = [None if x < 0 else (cats[x] if x < len(cats) else b"NOPE%d" % x)
           for x in g.integers(-1, len(cats) + 5, n).tolist()]
    rev = g.integers(1, 1000, n, dtype=np.int64)
    dcat = cats[:35]                                        # 5 categories have no dimension row
    brand = [b"BRAND-%d" % (i % 7) if i % 11 else None for i in range(35)]
    w = np.arange(35, dtype=np.int32) * 3 - 20
    gt = GTables([("Map 1", 0, [_strings(city), _strings(cat), rev]),
                  ("Map 2", 1, [_strings(dcat), _strings(brand), w])])
    pred = abi.Pred.leaf(abi.FILTER_GE, 0, a="C")           # city >= 'C' (bytes, unsigned)
    aggs = [(abi.CNT, -1), (abi.SUM, 2), (abi.SUM, 4)]
    r = run_plan(ctx, gt, 0, [op_filter(pred), op_join(1, 1, 0, build_keep=[1, 2]),   # city cat rev brand w
                              op_groupby([3, 0], aggs, max_groups=4096), op_sort([0, 1])])
    dim = {c: (b, int(x)) for c, b, x in zip(dcat, brand, w.tolist())}
    exp = {}
    for c, k, v in zip(city, cat, rev.tolist()):
        if c is None or c < b"C" or k is None or k not in dim:
            continue
        b, x = dim[k]
        key = (b, c)
        e = exp.get(key, [0, 0, 0])
        e[0] += 1
        e[1] += v
        e[2] += x
        exp[key] = e
    # Hive's order: NULLs first ascending, then bytes unsigned, shorter first on a tie
    keys = sorted(exp, key=lambda t: tuple((0, b"") if x is None else (1, x) for x in t))
    assert r["rows"] == len(keys)
    assert r["types"] == [abi.STRING, abi.STRING, abi.LONG, abi.LONG, abi.LONG]
    (gb, gbn), (gc, _), (cnt, _), (s1, _), (s2, _) = r["columns"]
    assert list(zip(gb, gc)) == keys
    assert gbn.tolist() == [k[0] is None for k in keys]
    assert cnt.tolist() == [exp[k][0] for k in keys]
    assert s1.tolist() == [exp[k][1] for k in keys] and s2.tolist() == [exp[k][2] for k in keys]
    assert r["sequence"] == [3, 4, 0, 1, 2] and len(r["stringCols"]) == 2


def test_string_join_keys_of_two_columns_and_outer_misses(ctx):
    """A LEFT OUTER join on (STRING, INT) keys: a probe row without a match
    keeps its columns and gets NULL build columns, a STRING one included."""
    g = np.random.default_rng(95)
    n = 50_000
    names = [b"n%03d" % i for i in range(60)]
    pk1 = [names[x] if x >= 0 else None for x in g.integers(-1, 60, n).tolist()]
    pk2 = g.integers(0, 4, n, dtype=np.int32)
    bk1 = names[:50] * 3
    bk2 = np.repeat(np.arange(3, dtype=np.int32), 50)
    battr = [b"attr-" + x + b"-%d" % y for x, y in zip(bk1, bk2.tolist())]
    gt = GTables([("Map 1", 0, [_strings(pk1), pk2]), ("Map 2", 2, [_strings(bk1), bk2, _strings(battr)])])
    r = run_plan(ctx, gt, 0, [op_join([0, 1], 1, [0, 1], build_keep=[2], join_type=abi.LEFT_OUTER_JOIN),
                              op_sort([0, 1])])
    look = {(a, b): c for a, b, c in zip(bk1, bk2.tolist(), battr)}
    rows = [(a, b, None if a is None else look.get((a, b))) for a, b in zip(pk1, pk2.tolist())]
    rows.sort(key=lambda t: ((0, b"") if t[0] is None else (1, t[0]), t[1]))   # stable, like the sort
    assert r["rows"] == n
    (s, _), (i, _), (a, an) = r["columns"]
    assert list(zip(s, i.tolist(), a)) == rows
    assert an.tolist() == [t[2] is None for t in rows]


def test_plans_over_empty_tables_and_empty_intermediates(ctx):
    """Edge cases the chain must carry: an input table of no rows, a build
    table of no rows, a filter that passes nothing before a GROUP BY (no
    groups) and a global aggregate over nothing (one row: COUNT 0, SUM NULL),
    and a STRING column of only NULLs through a join and a sort."""
    e64, e32 = np.array([], dtype=np.int64), np.array([], dtype=np.int32)
    gt = GTables([("Map 1", 0, [e64, e32]), ("Map 2", 0, [np.arange(5, dtype=np.int64)])])
    r = run_plan(ctx, gt, 0, [op_join(0, 1, 0), op_sort([1])])
    assert r["rows"] == 0 and r["types"] == [abi.INT, abi.LONG]      # the sort key first
    keys = np.arange(100, dtype=np.int64)
    gt = GTables([("Map 1", 0, [keys, np.ones(100, dtype=np.int32)]), ("Map 2", 0, [e64, e32])])
    r = run_plan(ctx, gt, 0, [op_join(0, 1, 0, build_keep=[1], join_type=abi.LEFT_OUTER_JOIN)])
    assert r["rows"] == 100 and r["columns"][2][1].all()            # every build column NULL
    r = run_plan(ctx, gt, 0, [op_join(0, 1, 0)])
    assert r["rows"] == 0
    never = abi.Pred.leaf(abi.FILTER_LT, 0, a=-1)
    r = run_plan(ctx, gt, 0, [op_filter(never), op_groupby([1], [(abi.CNT, -1), (abi.SUM, 0)])])
    assert r["rows"] == 0
    r = run_plan(ctx, gt, 0, [op_filter(never), op_groupby([], [(abi.CNT, -1), (abi.SUM, 0)])])
    assert r["rows"] == 1 and r["columns"][0][0][0] == 0 and r["columns"][1][1][0]
    nulls = _strings([None] * 50)
    gt = GTables([("Map 1", 0, [nulls, np.arange(50, dtype=np.int64)]), ("Map 2", 0, [_strings([b"a", None])])])
    r = run_plan(ctx, gt, 0, [op_join(0, 1, 0, join_type=abi.LEFT_OUTER_JOIN), op_sort([1], orders=[abi.DESC])])
    assert r["rows"] == 50 and all(v is None for v in r["columns"][1][0])
    assert r["columns"][0][0].tolist() == list(range(49, -1, -1))
