"""GPU tests of the operator server: each request's result is the same alone
and in a concurrent mix (and the same as the plain operator call), admission
respects the HBM budget, errors stay with their request.

Bit-exact for keys, counts, integer sums, MIN/MAX, filter rows, join pairs
(as sorted multisets) and sort order; DOUBLE SUM/AVG within REL_TOL.
"""
import threading
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

from ghive_b200 import abi, workloads

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


def _host(res):
    """(columns as numpy (values, nulls)), rowid, rowid2 of a served result."""
    cols = [(v.cpu().numpy().copy(), None if nl is None else nl.cpu().numpy().copy()) for v, nl in res.cols]
    rid = None if res.rowid is None else res.rowid.cpu().numpy().copy()
    rid2 = None if res.rowid2 is None else res.rowid2.cpu().numpy().copy()
    return cols, rid, rid2, res.rows


def _groupby_canon(cols, nkeys):
    if nkeys:
        v, nl = cols[0]
        nl = np.zeros(len(v), bool) if nl is None else nl.astype(bool)
        order = np.lexsort((np.where(nl, 0, v), ~nl))
    else:
        order = slice(None)
    return [(v[order], None if nl is None else nl.astype(bool)[order]) for v, nl in cols]


def _same_cols(a, b, tol_cols=()):
    assert len(a) == len(b)
    for j, ((av, an), (bv, bn)) in enumerate(zip(a, b)):
        an = np.zeros(len(av), bool) if an is None else an.astype(bool)
        bn = np.zeros(len(bv), bool) if bn is None else bn.astype(bool)
        assert np.array_equal(an, bn), j
        x, y = av[~an], bv[~bn]
        if j in tol_cols:
            assert np.all(np.abs(x - y) <= REL_TOL * np.maximum(np.abs(y), 1e-300)), j
        else:
            assert np.array_equal(x, y), j


class Mix:
    """A seeded mix of requests over device-resident inputs."""

    def __init__(self, srv, n_req=28, seed=41):
        g = workloads.rng(seed)
        self.fact = [dev(c) for c in workloads.fact_table(2_000_000, seed_idx=seed, groups=3000)]
        (bkey, bpay), (fk, _) = workloads.join_tables(200_000, 3_000_000, seed_idx=seed)
        self.bkey, self.bpay = dev(bkey), [dev(c) for c in bpay]
        self.fk = dev(fk)
        bkey2 = g.permutation(np.arange(1, 50_001, dtype=np.int64))
        self.bkey2, self.bpay2 = dev(bkey2), [dev(g.integers(0, 1 << 40, 50_000, dtype=np.int64))]
        d, k, rowid = workloads.sort_table(2_000_000, seed_idx=seed)
        self.sort = [dev(d), dev(k), dev(rowid)]
        self.tables = [srv.add_join_table(self.bkey, self.bpay), srv.add_join_table(self.bkey2, self.bpay2)]
        self.reqs = []
        for i in range(n_req):
            kind = ["groupby", "join", "sort", "filter"][i % 4]
            n = int(np.exp(g.uniform(np.log(1_000), np.log(2_000_000))))
            off = int(g.integers(0, 2_000_000 - n + 1))
            self.reqs.append((kind, n, off, int(g.integers(100, 2400))))

    def submit(self, srv, i):
        kind, n, off, cut = self.reqs[i]
        if kind == "groupby":
            cols = [c[off:off + n] for c in self.fact]
            return srv.submit_groupby(workloads.fact_predicate(cut), cols, [0], workloads.AGGS_FACT, 3000)
        if kind == "filter":
            cols = [c[off:off + n] for c in self.fact]
            return srv.submit_filter(workloads.fact_predicate(cut), cols, proj=[0, 2])
        if kind == "join":
            m = min(n, 3_000_000 - off)
            return srv.submit_join(self.tables[(i // 4) % 2], self.fk[off:off + m])
        return srv.submit_sort([c[off:off + n] for c in self.sort[:2]], payload=[self.sort[2][off:off + n]])

    def plain(self, ctx, i):
        """The same request through the plain operator API."""
        kind, n, off, cut = self.reqs[i]
        if kind == "groupby":
            cols = [c[off:off + n] for c in self.fact]
            k, a, g = ctx.filter_groupby(workloads.fact_predicate(cut), cols, [0], workloads.AGGS_FACT,
                                         capacity=3000, max_groups=3000)
            return [(v.cpu().numpy(), nl.cpu().numpy()) for v, nl in k + a], None, g
        if kind == "filter":
            cols = [c[off:off + n] for c in self.fact]
            outs, k = ctx.filter(workloads.fact_predicate(cut), cols, proj=[0, 2])
            return [(v.cpu().numpy(), None) for v, nl in outs], None, k
        if kind == "join":
            m = min(n, 3_000_000 - off)
            key, pay = (self.bkey, self.bpay) if (i // 4) % 2 == 0 else (self.bkey2, self.bpay2)
            t = ctx.join_build(key, build_payload=pay)
            r = ctx.join_probe(t, self.fk[off:off + m], abi.INNER_JOIN, capacity=m)
            t.free()
            return r
        d, kk, rid = (c[off:off + n] for c in self.sort)
        outs = ctx.sort([d, kk], payload=[rid])
        return outs


def _check(mix, ctx, i, served):
    kind = mix.reqs[i][0]
    cols, rid, _, rows = served
    if kind == "groupby":
        exp, _, g = mix.plain(ctx, i)
        assert rows == g
        _same_cols(_groupby_canon(cols, 1), _groupby_canon(exp, 1), tol_cols=(3, 4))
    elif kind == "filter":
        exp, _, k = mix.plain(ctx, i)
        assert rows == k
        _same_cols([(v, None) for v, _ in cols], exp)
    elif kind == "join":
        r = mix.plain(ctx, i)
        prow = r["probe_rowid"].cpu().numpy() if isinstance(r, dict) else None
        if prow is None:
            return
        exp = sorted(zip(prow.tolist(), *[c[0].cpu().numpy().tolist() for c in r["build"]]))
        got = sorted(zip(rid.tolist(), *[c[0].tolist() for c in cols]))
        assert rows == len(exp) and got == exp
    else:
        outs = mix.plain(ctx, i)
        keys, pay = outs[0], outs[1]
        exp = [(v.cpu().numpy(), None) for v, _ in keys + pay]
        _same_cols([(v, None) for v, _ in cols], exp)


def test_served_results_same_alone_and_in_the_mix(ctx):
    from ghive_b200.serve import Server
    with Server(0, slots=4) as srv:
        mix = Mix(srv)
        # alone: one request at a time through the server
        alone = []
        for i in range(len(mix.reqs)):
            t = mix.submit(srv, i)
            alone.append(_host(srv.wait(t)))
            srv.release(t)
        # in the mix: every request submitted at once from 8 threads
        mixed = [None] * len(mix.reqs)

        def run(i):
            t = mix.submit(srv, i)
            res = srv.wait(t)
            mixed[i] = (_host(res), res.admit_ns, res.done_ns)
            srv.release(t)

        with ThreadPoolExecutor(8) as ex:
            list(ex.map(run, range(len(mix.reqs))))
        spans = sorted((a, d) for _, a, d in mixed)
        overlap = any(spans[k + 1][0] < spans[k][1] for k in range(len(spans) - 1))
        assert overlap, "no two requests ran at the same time"
        for i in range(len(mix.reqs)):
            a, m = alone[i], mixed[i][0]
            assert a[3] == m[3], i
            kind = mix.reqs[i][0]
            if kind == "groupby":
                _same_cols(_groupby_canon(a[0], 1), _groupby_canon(m[0], 1), tol_cols=(3, 4))
            elif kind == "join":
                assert sorted(zip(a[1].tolist(), *[c[0].tolist() for c in a[0]])) == \
                    sorted(zip(m[1].tolist(), *[c[0].tolist() for c in m[0]]))
            else:
                _same_cols(a[0], m[0])
            _check(mix, ctx, i, m)
        assert srv.stats()["bytes_admitted"] == 0


def test_admission_budget_serialises_large_requests():
    from ghive_b200.serve import Server
    d, k, rowid = workloads.sort_table(1_000_000, seed_idx=42)
    cols = [dev(d), dev(k), dev(rowid)]
    # each sort needs ~40 MB of outputs and scratch: a 50 MB budget admits one at a time
    with Server(0, slots=4, hbm_budget=50 << 20) as srv:
        ts = [srv.submit_sort(cols[:2], payload=[cols[2]]) for _ in range(6)]
        res = [srv.wait(t) for t in ts]
        spans = sorted((r.admit_ns, r.done_ns) for r in res)
        for (a0, d0), (a1, d1) in zip(spans, spans[1:]):
            assert a1 >= d0, "two requests over the budget overlapped"
        first = [(v.cpu().numpy().copy()) for v, _ in res[0].cols]
        for r in res[1:]:
            for x, (v, _) in zip(first, r.cols):
                assert np.array_equal(x, v.cpu().numpy())
        for t in ts:
            srv.release(t)


def test_errors_stay_with_their_request():
    from ghive_b200._lib import GhbError
    from ghive_b200.serve import Server
    cols = [dev(c) for c in workloads.fact_table(100_000, seed_idx=43, groups=1000)]
    with Server(0, slots=2) as srv:
        bad = srv.submit_groupby(None, cols, [0], workloads.AGGS_FACT, max_groups=10)  # 1000 groups
        good = srv.submit_groupby(None, cols, [0], workloads.AGGS_FACT, max_groups=1000)
        with pytest.raises(GhbError) as e:
            srv.wait(bad)
        assert e.value.code == abi.ERR_CAPACITY
        r = srv.wait(good)
        assert r.status == 0 and r.rows == 1000
        srv.release(bad)
        srv.release(good)
        again = srv.submit_groupby(None, cols, [0], workloads.AGGS_FACT, max_groups=1000)
        assert srv.wait(again).rows == 1000
        srv.release(again)


def test_destroy_with_requests_in_flight():
    from ghive_b200.serve import Server
    d, k, rowid = workloads.sort_table(500_000, seed_idx=44)
    cols = [dev(d), dev(k), dev(rowid)]
    srv = Server(0, slots=2)
    for _ in range(10):
        srv.submit_sort(cols[:2], payload=[cols[2]])
    done = threading.Event()

    def close():
        srv.close()
        done.set()

    th = threading.Thread(target=close)
    th.start()
    th.join(timeout=60)
    assert done.is_set()
