"""Multi-rank host logic on CPU: world_size-2 gloo process groups.

Each rank runs the oracle on its shard (the device kernels' results equal the
oracle's, as the GPU tests show), the ranks exchange their partial results
with a collective, and the merged result must equal the oracle over all rows:
bit-exact for keys, counts, integer sums, MIN/MAX and join pairs, DOUBLE
SUM/AVG within REL_TOL.
"""
import os
import socket

import numpy as np
import pytest

from ghive_b200 import abi, shard, workloads

REL_TOL = 1e-12
WORLD = 2


def _port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _oracle_local_groupby(pred, cols, keys, aggs):
    """One rank's group-by over its columns (torch CPU tensors or (values,
    isnull) pairs): the CPU oracle here, the device operator on a GPU."""
    import torch

    from oracle import oracle

    def np_col(c):
        return (c[0].numpy(), c[1].numpy().astype(bool)) if isinstance(c, tuple) else c.numpy()
    k, v = oracle.filter_groupby(pred, [np_col(c) for c in cols], keys, aggs)
    key = (torch.from_numpy(k[0][0]), torch.from_numpy(k[0][1])) if keys else None
    return key, [(torch.from_numpy(a), torch.from_numpy(b)) for a, b in v]


def _groupby_rank(rank, world, port, q):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        cols = workloads.fact_table(200_003, seed_idx=51, groups=700)
        lo, hi = shard.shard_range(len(cols[0]), rank, world)
        mine = [torch.from_numpy(c[lo:hi]) for c in cols]
        key, vals = shard.groupby_sharded(mine, 0, workloads.AGGS_FACT, _oracle_local_groupby,
                                          pred=workloads.fact_predicate())
        _, gvals = shard.groupby_sharded(mine, None, [(abi.SUM, 1), (abi.MIN, 3), (abi.AVG, 2)],
                                         _oracle_local_groupby)
        res = ((key[0].numpy(), key[1].numpy()), [(v.numpy(), n.numpy()) for v, n in vals],
               [(v.numpy(), n.numpy()) for v, n in gvals])
        gathered = [None] * world
        dist.all_gather_object(gathered, res)
        if rank == 0:
            q.put(gathered)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _join_rank(rank, world, port, q):
    import torch.distributed as dist

    from oracle import oracle
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        (bkey, bpay), (fk, _) = workloads.join_tables(50_000, 300_001, seed_idx=52)
        lo, hi = shard.shard_range(len(fk), rank, world)
        prow, outs = oracle.hash_join_mt(2, bkey, fk[lo:hi], bpay)
        gathered = [None] * world
        dist.all_gather_object(gathered, (np.asarray(prow) + lo, [np.asarray(o) for o in outs]))
        if rank == 0:
            q.put(gathered)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _sort_table(n):
    g = np.random.default_rng(53)
    d = g.integers(0, 40, n, dtype=np.int32)
    dn = g.random(n) < 0.05
    k = g.integers(-1000, 1000, n, dtype=np.int64)
    x = np.round(g.normal(0, 10, n), 1)
    return d, dn, k, x


def _np_local_sort(keys, payload, orders, null_orders):
    """The stable local sort of one rank's received rows: the CPU oracle here
    (the ranks are CPU processes); on a GPU it is the device sort."""
    import torch

    from oracle import oracle

    def np_col(c):
        return (c[0].numpy(), c[1].numpy().astype(bool)) if isinstance(c, tuple) else c.numpy()

    perm = oracle.sort_perm([np_col(c) for c in keys], orders, null_orders)
    pt = torch.from_numpy(perm)

    def take(c):
        return (c[0][pt], c[1][pt]) if isinstance(c, tuple) else c[pt]
    return [take(c) for c in keys], [take(c) for c in payload]


def _sort_rank(rank, world, port, q):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        d, dn, k, x = _sort_table(100_003)
        lo, hi = shard.shard_range(len(d), rank, world)
        rid = np.arange(lo, hi, dtype=np.int64)
        keys = [(torch.from_numpy(d[lo:hi]), torch.from_numpy(dn[lo:hi].astype(np.uint8))),
                torch.from_numpy(x[lo:hi])]
        pay = [torch.from_numpy(k[lo:hi]), torch.from_numpy(rid)]
        out = {}
        for name, orders, nulls in (("asc", [abi.ASC, abi.DESC], None),
                                    ("desc", [abi.DESC, abi.ASC], [abi.NULLS_FIRST, abi.NULLS_DEFAULT])):
            ok, op = shard.sort_sharded(keys, pay, _np_local_sort, orders, nulls, sample_per_rank=500)
            out[name] = (ok[0][0].numpy(), ok[0][1].numpy(), ok[1].numpy(), op[1].numpy())
        gathered = [None] * world
        dist.all_gather_object(gathered, out)
        if rank == 0:
            q.put(gathered)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _spawn(fn):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _port()
    procs = [ctx.Process(target=fn, args=(r, WORLD, port, q)) for r in range(WORLD)]
    for p in procs:
        p.start()
    out = q.get(timeout=240)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    return out


def test_shard_ranges_cover_rows_once():
    for n in (0, 1, 7, 1000, 1001):
        for w in (1, 2, 3, 8):
            got = [shard.shard_range(n, r, w) for r in range(w)]
            assert got[0][0] == 0 and got[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(got, got[1:]))
            assert max(h - l for l, h in got) - min(h - l for l, h in got) <= 1


def _check_cols(got, exp):
    for j, ((gv, gn), (xv, xn)) in enumerate(zip(got, exp)):
        assert np.array_equal(gn, xn), j
        if xv.dtype.kind == "f":
            assert np.all(np.abs(gv[~gn] - xv[~xn]) <= REL_TOL * np.abs(xv[~xn])), j
        else:
            assert np.array_equal(gv[~gn].astype(xv.dtype), xv[~xn]), j


def test_sharded_groupby_merges_to_the_whole():
    """Two ranks aggregate their halves, exchange the partial rows by the
    hash of their key and merge them: the union of the ranks' groups is the
    oracle's result over all rows, each group on exactly one rank; the global
    aggregate's one row is on rank 0."""
    from oracle import oracle
    gathered = _spawn(_groupby_rank)
    kv = np.concatenate([g[0][0] for g in gathered])
    kn = np.concatenate([g[0][1] for g in gathered])
    vals = [(np.concatenate([g[1][j][0] for g in gathered]), np.concatenate([g[1][j][1] for g in gathered]))
            for j in range(len(workloads.AGGS_FACT))]
    assert all(len(g[0][0]) > 0 for g in gathered)    # both ranks own groups
    order = np.lexsort((np.where(kn, 0, kv), ~kn))
    cols = workloads.fact_table(200_003, seed_idx=51, groups=700)
    ek, ev = oracle.filter_groupby(workloads.fact_predicate(), cols, [0], workloads.AGGS_FACT)
    assert np.array_equal(kv[order], ek[0][0]) and np.array_equal(kn[order], ek[0][1])
    _check_cols([(v[order], n[order]) for v, n in vals], ev)
    gaggs = [(abi.SUM, 1), (abi.MIN, 3), (abi.AVG, 2)]
    _, gv = oracle.filter_groupby(None, cols, [], gaggs)
    assert len(gathered[0][2][0][0]) == 1 and len(gathered[1][2][0][0]) == 0
    _check_cols(gathered[0][2], gv)


def test_sharded_join_probe_unions_to_the_whole():
    from oracle import oracle
    gathered = _spawn(_join_rank)
    (bkey, bpay), (fk, _) = workloads.join_tables(50_000, 300_001, seed_idx=52)
    prow, outs = oracle.hash_join_mt(2, bkey, fk, bpay)
    got = sorted(zip(np.concatenate([g[0] for g in gathered]).tolist(),
                     *[np.concatenate([g[1][j] for g in gathered]).tolist() for j in range(len(bpay))]))
    exp = sorted(zip(np.asarray(prow).tolist(), *[np.asarray(o).tolist() for o in outs]))
    assert got == exp


def test_sharded_sort_is_the_global_stable_order():
    """Sample sort over two ranks: the ranks' outputs, concatenated in rank
    order, are the oracle's stable order of all rows (row ids compared, so
    ties keep the input order across ranks too), ASC and DESC, NULLs."""
    from oracle import oracle
    gathered = _spawn(_sort_rank)
    d, dn, k, x = _sort_table(100_003)
    for name, orders, nulls in (("asc", [abi.ASC, abi.DESC], None),
                                ("desc", [abi.DESC, abi.ASC], [abi.NULLS_FIRST, abi.NULLS_DEFAULT])):
        perm = oracle.sort_perm([(d, dn), x], orders, nulls)
        rid = np.concatenate([g[name][3] for g in gathered])
        assert np.array_equal(rid, perm), name
        assert all(len(g[name][3]) > 0 for g in gathered)   # both ranks got rows
        got_x = np.concatenate([g[name][2] for g in gathered])
        assert np.array_equal(got_x.view(np.uint64), x[perm].view(np.uint64))


def test_order_image_is_monotone():
    import torch
    g = np.random.default_rng(4)
    v = np.concatenate([g.normal(0, 1e3, 2000), [0.0, np.inf, -np.inf, 1e-300, -1e-300]])
    img = shard.order_image(torch.from_numpy(v), None, False, True).numpy()
    o = np.argsort(v, kind="stable")
    assert np.all(np.diff(img[o]) >= 0)
    z = shard.order_image(torch.tensor([-0.0, 0.0], dtype=torch.float64), None, False, True).numpy()
    assert z[0] < z[1]   # IEEE total order: -0.0 before +0.0
    iv = g.integers(-(1 << 62), 1 << 62, 3000, dtype=np.int64)
    img = shard.order_image(torch.from_numpy(iv), None, True, False).numpy()
    o = np.argsort(-iv, kind="stable")
    assert np.all(np.diff(img[o]) >= 0)


if __name__ == "__main__":
    pytest.main([__file__, "-q"])
