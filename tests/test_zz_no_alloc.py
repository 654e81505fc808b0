"""The allocation-free group-by entry point against the oracle and against the
allocating one.

ghb_filter_groupby_noalloc serves callers that cannot call cudaMalloc (a task
whose device memory is all reserved by another allocator, or code that must
not risk the device-wide synchronisation an allocation may imply).  It keeps
its hash table in a fixed file-scope device array instead of a context.  This
test calls it through the C ABI twice in a row (the second call must not see
the first call's table) and compares each result with the CPU oracle and with
ghb_filter_groupby on the same inputs: keys, counts, integer sums and MIN/MAX
bit-exact, double SUM/AVG within REL_TOL.  The second call must leave the
device's free memory unchanged (the first call on a device is its set-up and
may load code).  It also checks the size limit is refused up front.  The file
name sorts last so a stop-at-first-failure run has run every other test
before this one.
"""
import ctypes as C

import numpy as np
import pytest

from ghive_b200 import abi, workloads
from oracle import oracle

pytestmark = pytest.mark.gpu

REL_TOL = 1e-12
TYPES = [abi.LONG, abi.LONG, abi.DOUBLE, abi.DOUBLE, abi.INT, abi.INT]


def _rows(keys, aggs):
    n = len(keys[0][0])
    rows = [tuple(v[i].item() if not nl[i] else None for v, nl in keys + aggs) for i in range(n)]
    return sorted(rows, key=lambda r: r[0])


class _NoallocCall:
    """Arguments of one ghb_filter_groupby_noalloc call, prepared (and their
    device buffers allocated) before the call, so the call itself is the
    only thing that runs between two readings of the device's free memory."""

    def __init__(self, cols, keys, aggs, capacity, max_groups):
        import torch

        from ghive_b200.ops import _Cols, _Outs
        self.cs = _Cols(cols)
        types = [self.cs[k].type for k in keys]
        types += [abi.agg_out_type(t, self.cs[c].type if c >= 0 else abi.LONG) for t, c in aggs]
        self.outs = _Outs(types, capacity, "cuda:0")
        self.ka = (C.c_int32 * max(1, len(keys)))(*keys)
        self.ag = (abi.AggDesc * len(aggs))()
        for i, (t, c) in enumerate(aggs):
            self.ag[i].type, self.ag[i].col = t, c
        self.cfg = abi.GroupByCfg()
        self.cfg.max_groups = max_groups
        self.d_groups = torch.zeros(1, dtype=torch.int64, device="cuda:0")
        self.pred = workloads.fact_predicate().as_struct()
        self.nkeys, self.naggs, self.capacity = len(keys), len(aggs), capacity
        self.stream = torch.cuda.current_stream().cuda_stream

    def __call__(self):
        from ghive_b200._lib import lib
        return lib().ghb_filter_groupby_noalloc(
            C.addressof(self.pred), self.cs.ptr, self.cs.n, self.ka, self.nkeys, self.ag,
            self.naggs, self.outs.ptr, self.capacity, self.d_groups.data_ptr(),
            C.byref(self.cfg), self.stream)

    def result(self):
        g = int(self.d_groups.item())
        res = [(v.cpu().numpy(), nl.cpu().numpy()) for v, nl in self.outs.rows(min(g, self.capacity))]
        return res[:self.nkeys], res[self.nkeys:], g


def _assert_rows_match(got, ref):
    assert len(got) == len(ref)
    for a, b in zip(got, ref):
        assert a[0] == b[0]
        for x, y, t in zip(a[1:], b[1:], TYPES):
            if t == abi.DOUBLE:
                assert abs(x - y) <= REL_TOL * abs(y), (a[0], x, y)
            else:
                assert x == y, (a[0], x, y)


def test_noalloc_matches_oracle_and_allocating_entry_point_twice():
    import torch

    from ghive_b200.ops import Context
    torch.cuda.set_device(0)
    for call, seed in enumerate((50, 51)):
        groups = 1000 if call == 0 else 300
        cols = workloads.fact_table(400_000, seed_idx=seed, groups=groups)
        dcols = [torch.from_numpy(c).cuda() for c in cols]
        fn = _NoallocCall(dcols, [0], workloads.AGGS_FACT, capacity=1024, max_groups=1000)
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info(0)[0]
        st = fn()
        torch.cuda.synchronize()
        free_after = torch.cuda.mem_get_info(0)[0]
        assert st == abi.OK
        if call == 1:  # after the set-up call, a call allocates nothing
            assert free_after == free_before, (free_before, free_after)
        nk, na, ng = fn.result()
        assert ng == groups
        got = _rows(nk, na)
        ok, oa = oracle.filter_groupby(workloads.fact_predicate(), cols, [0], workloads.AGGS_FACT)
        _assert_rows_match(got, _rows(ok, oa))
        with Context(0) as ctx:
            rk, ra, rg = ctx.filter_groupby(workloads.fact_predicate(), dcols, [0],
                                            workloads.AGGS_FACT, capacity=1024, max_groups=1000)
        assert rg == groups
        _assert_rows_match(got, _rows([(v.cpu().numpy(), nl.cpu().numpy()) for v, nl in rk],
                                      [(v.cpu().numpy(), nl.cpu().numpy()) for v, nl in ra]))


def test_noalloc_refuses_a_table_beyond_its_array():
    import torch
    # 200,000 groups need a 2^19-slot table (~29 MB), beyond the 8 MiB array
    cols = [torch.from_numpy(c).cuda() for c in workloads.fact_table(200_000, seed_idx=52)]
    fn = _NoallocCall(cols, [0], workloads.AGGS_FACT, capacity=200_000, max_groups=200_000)
    assert fn() == abi.ERR_CAPACITY
