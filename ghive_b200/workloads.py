"""Seeded synthetic inputs with the shapes of the benchmark workloads.

There is no dataset in this project: the fact-table, join and sort workloads
are generated with numpy's PCG64 from a seed (base seed 20261203 + workload
index), with the column types, ranges and distributions the workloads name.
"""
import numpy as np

from . import abi

SEED = 20261203

AGGS_FACT = [(abi.CNT, -1), (abi.SUM, 1), (abi.SUM, 2), (abi.AVG, 2), (abi.MIN, 3), (abi.MAX, 3)]


def rng(idx, salt=0):
    return np.random.Generator(np.random.PCG64(SEED + idx + 1000 * salt))


def fact_table(n=6_000_000, seed_idx=0, groups=1000, days=2526):
    """Filter + group-by fact table: k int32 U[0,groups), qty int64 U[1,50],
    price double U_int[90000,10500000]/100 (two decimals), d int32 U[0,days)."""
    g = rng(seed_idx)
    k = g.integers(0, groups, n, dtype=np.int32)
    qty = g.integers(1, 51, n, dtype=np.int64)
    price = g.integers(90000, 10500001, n, dtype=np.int64) / 100.0
    d = g.integers(0, days, n, dtype=np.int32)
    return [k, qty, price, d]


def fact_predicate(cut=1263):
    """d < cut on column 3 (about 50% of rows for cut = 1263)."""
    return abi.Pred.leaf(abi.FILTER_LT, 3, a=cut)


def join_tables(n_build=1_500_000, n_probe=60_000_000, miss=0.05, seed_idx=1):
    """Build: unique int64 keys = a permutation of [1, n_build], payload int64
    U[0,2^62), payload double U[0,1).  Probe: int64 foreign key uniform over the
    build keys, a `miss` fraction replaced by keys in (n_build, 2*n_build] that
    match nothing, plus an int32 payload."""
    g = rng(seed_idx)
    bkey = g.permutation(np.arange(1, n_build + 1, dtype=np.int64))
    bpay_l = g.integers(0, 1 << 62, n_build, dtype=np.int64)
    bpay_d = g.random(n_build)
    fk = g.integers(1, n_build + 1, n_probe, dtype=np.int64)
    m = g.random(n_probe) < miss
    fk[m] = g.integers(n_build + 1, 2 * n_build + 1, int(m.sum()), dtype=np.int64)
    ppay = g.integers(0, 1 << 31, n_probe, dtype=np.int64).astype(np.int32)
    return (bkey, [bpay_l, bpay_d]), (fk, ppay)


def zipf_ranks(g, n, distinct, theta):
    """Ranks in [0, distinct) with P(r) proportional to 1/(r+1)^theta (theta >= 0)."""
    if theta <= 0.0:
        return g.integers(0, distinct, n, dtype=np.int64)
    w = 1.0 / np.power(np.arange(1, distinct + 1, dtype=np.float64), theta)
    cdf = np.cumsum(w)
    cdf /= cdf[-1]
    return np.minimum(np.searchsorted(cdf, g.random(n), side="right"), distinct - 1).astype(np.int64)


def sort_table(n=60_000_000, zipf=False, seed_idx=2, days=2526):
    """d int32 U[0,days), k int64 U[0,2^40) (or Zipf(0.99) over 10^6 distinct
    values, each rank mapped to a fixed distinct value in [0,2^40)), rowid int32."""
    g = rng(seed_idx, 1 if zipf else 0)
    d = g.integers(0, days, n, dtype=np.int32)
    if zipf:
        vals = np.unique(g.integers(0, 1 << 40, 1_200_000, dtype=np.int64))[:1_000_000]
        g.shuffle(vals)
        k = vals[zipf_ranks(g, n, len(vals), 0.99)]
    else:
        k = g.integers(0, 1 << 40, n, dtype=np.int64)
    rowid = np.arange(n, dtype=np.int32)
    return d, k, rowid


def batched_instances(count=512, seed_idx=3, min_rows=1_000, max_rows=10_000_000,
                      scale=1.0):
    """Independent filter + group-by instances: rows log-U[min_rows,max_rows]
    (times scale), groups log-U[10,10^6], int64 keys Zipf(theta U[0,1.2]) over
    the groups, qty/price as the fact table, d int32 U[0,2526) with predicate
    d < round(s*2526), s U[0.01,0.9].  Yields dicts per instance."""
    g = rng(seed_idx)
    for i in range(count):
        rows = int(np.exp(g.uniform(np.log(min_rows), np.log(max_rows))) * scale)
        rows = max(rows, 1)
        groups = int(np.exp(g.uniform(np.log(10), np.log(1_000_000))))
        theta = g.uniform(0.0, 1.2)
        sel = g.uniform(0.01, 0.9)
        ig = rng(seed_idx, 10 + i)
        keys = zipf_ranks(ig, rows, groups, theta)
        qty = ig.integers(1, 51, rows, dtype=np.int64)
        price = ig.integers(90000, 10500001, rows, dtype=np.int64) / 100.0
        d = ig.integers(0, 2526, rows, dtype=np.int32)
        yield {"rows": rows, "groups": groups, "theta": theta, "cut": int(round(sel * 2526)),
               "cols": [keys, qty, price, d]}
