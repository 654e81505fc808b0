"""The sharded group-by's device path on one GPU: the rank's partial
aggregates (AVG as SUM + COUNT) computed by the device group-by and merged by
a second device group-by over the partial rows, against the oracle over the
same rows (one rank: no exchange)."""
import numpy as np
import pytest

from ghive_b200 import abi, shard, workloads

pytestmark = pytest.mark.gpu

REL_TOL = 1e-12


def test_groupby_sharded_on_the_device():
    import torch

    from ghive_b200.ops import Context
    from oracle import oracle
    ctx = Context(0)
    dev = torch.device("cuda", 0)

    def local(pred, cols, keys, aggs):
        k, v, _ = ctx.filter_groupby(pred, cols, keys, aggs)
        return (k[0] if keys else None), v

    try:
        cols = workloads.fact_table(2_000_000, seed_idx=72, groups=5000)
        dcols = [torch.from_numpy(c).to(dev) for c in cols]
        key, vals = shard.groupby_sharded(dcols, 0, workloads.AGGS_FACT, local, pred=workloads.fact_predicate())
        _, gvals = shard.groupby_sharded(dcols, None, [(abi.SUM, 1), (abi.AVG, 2), (abi.MAX, 3)], local)
    finally:
        ctx.close()
    kv, kn = key[0].cpu().numpy(), key[1].cpu().numpy()
    order = np.lexsort((np.where(kn, 0, kv), ~kn))
    ek, ev = oracle.filter_groupby(workloads.fact_predicate(), cols, [0], workloads.AGGS_FACT)
    assert np.array_equal(kv[order], ek[0][0])
    _, gv = oracle.filter_groupby(None, cols, [], [(abi.SUM, 1), (abi.AVG, 2), (abi.MAX, 3)])
    for got, exp, o in ((vals, ev, order), (gvals, gv, np.arange(1))):
        for j, ((v, n), (xv, xn)) in enumerate(zip(got, exp)):
            v, n = v.cpu().numpy()[o], n.cpu().numpy()[o]
            assert np.array_equal(n, xn), j
            if xv.dtype.kind == "f":
                assert np.all(np.abs(v[~n] - xv[~xn]) <= REL_TOL * np.abs(xv[~xn])), j
            else:
                assert np.array_equal(v[~n].astype(xv.dtype), xv[~xn]), j
