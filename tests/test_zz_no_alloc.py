"""The allocation-free group-by entry point against the allocating one.

ghb_filter_groupby_noalloc serves callers that cannot call cudaMalloc (a task
whose device memory is all reserved by another allocator, or code that must
not risk the device-wide synchronisation an allocation may imply).  It keeps
its hash table in a fixed file-scope device array instead of a context.  This
test calls it through the C ABI twice in a row (the second call must not see
the first call's table) and compares each result with ghb_filter_groupby on
the same inputs: keys, counts, integer sums and MIN/MAX bit-exact, double
SUM/AVG within REL_TOL.  It also checks the size limit is refused up front.
The file name sorts last so a stop-at-first-failure run has run every other
test before this one.
"""
import ctypes as C

import numpy as np
import pytest

from ghive_b200 import abi, workloads

pytestmark = pytest.mark.gpu

REL_TOL = 1e-12


def _rows(keys, aggs):
    n = len(keys[0][0])
    rows = [tuple(v[i].item() if not nl[i] else None for v, nl in keys + aggs) for i in range(n)]
    return sorted(rows, key=lambda r: r[0])


def _noalloc(cols, keys, aggs, capacity, max_groups):
    import torch

    from ghive_b200._lib import lib
    from ghive_b200.ops import _Cols, _Outs
    cs = _Cols(cols)
    types = [cs[k].type for k in keys]
    types += [abi.agg_out_type(t, cs[c].type if c >= 0 else abi.LONG) for t, c in aggs]
    outs = _Outs(types, capacity, "cuda:0")
    ka = (C.c_int32 * max(1, len(keys)))(*keys)
    ag = (abi.AggDesc * len(aggs))()
    for i, (t, c) in enumerate(aggs):
        ag[i].type, ag[i].col = t, c
    cfg = abi.GroupByCfg()
    cfg.max_groups = max_groups
    d_groups = torch.zeros(1, dtype=torch.int64, device="cuda:0")
    pred = workloads.fact_predicate().as_struct()
    st = lib().ghb_filter_groupby_noalloc(C.addressof(pred), cs.ptr, cs.n, ka, len(keys), ag,
                                          len(aggs), outs.ptr, capacity, d_groups.data_ptr(),
                                          C.byref(cfg), torch.cuda.current_stream().cuda_stream)
    g = int(d_groups.item())
    res = outs.rows(min(g, capacity))
    return st, res[:len(keys)], res[len(keys):], g


def _host(res):
    return [(v.cpu().numpy(), nl.cpu().numpy()) for v, nl in res]


def test_noalloc_matches_allocating_entry_point_twice():
    import torch

    from ghive_b200.ops import Context
    torch.cuda.set_device(0)
    for call, seed in enumerate((50, 51)):
        cols = workloads.fact_table(400_000, seed_idx=seed, groups=1000 if call == 0 else 300)
        dcols = [torch.from_numpy(c).cuda() for c in cols]
        st, nk, na, ng = _noalloc(dcols, [0], workloads.AGGS_FACT, capacity=1024, max_groups=1000)
        assert st == abi.OK
        with Context(0) as ctx:
            rk, ra, rg = ctx.filter_groupby(workloads.fact_predicate(), dcols, [0],
                                            workloads.AGGS_FACT, capacity=1024, max_groups=1000)
        assert ng == rg == (1000 if call == 0 else 300)
        got = _rows(_host(nk), _host(na))
        ref = _rows(_host(rk), _host(ra))
        types = [abi.LONG, abi.LONG, abi.DOUBLE, abi.DOUBLE, abi.INT, abi.INT]
        for a, b in zip(got, ref):
            assert a[0] == b[0]
            for x, y, t in zip(a[1:], b[1:], types):
                if t == abi.DOUBLE:
                    assert abs(x - y) <= REL_TOL * abs(y)
                else:
                    assert x == y


def test_noalloc_refuses_a_table_beyond_its_array():
    import torch
    # 200,000 groups need a 2^19-slot table (~29 MB), beyond the 8 MiB array
    cols = [torch.from_numpy(c).cuda() for c in workloads.fact_table(200_000, seed_idx=52)]
    st, _, _, _ = _noalloc(cols, [0], workloads.AGGS_FACT, capacity=200_000, max_groups=200_000)
    assert st == abi.ERR_CAPACITY
