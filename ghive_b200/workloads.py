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


def join_tables(n_build=1_500_000, n_probe=60_000_000, miss=0.05, seed_idx=1, sparse=False):
    """Build: unique int64 keys = a permutation of [1, n_build], payload int64
    U[0,2^62), payload double U[0,1).  Probe: int64 foreign key uniform over the
    build keys, a `miss` fraction replaced by keys in (n_build, 2*n_build] that
    match nothing, plus an int32 payload.  sparse=True passes every key (build
    and probe) through mix64_np, a bijection: the same matches, but keys spread
    over the whole int64 range (a natural key instead of a surrogate one)."""
    g = rng(seed_idx)
    bkey = g.permutation(np.arange(1, n_build + 1, dtype=np.int64))
    bpay_l = g.integers(0, 1 << 62, n_build, dtype=np.int64)
    bpay_d = g.random(n_build)
    fk = g.integers(1, n_build + 1, n_probe, dtype=np.int64)
    m = g.random(n_probe) < miss
    fk[m] = g.integers(n_build + 1, 2 * n_build + 1, int(m.sum()), dtype=np.int64)
    ppay = g.integers(0, 1 << 31, n_probe, dtype=np.int64).astype(np.int32)
    if sparse:
        bkey, fk = mix64_np(bkey), mix64_np(fk)
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


_MIX1, _MIX2 = 0xBF58476D1CE4E5B9, 0x94D049BB133111EB


def mix64_np(x):
    """splitmix64's finalizer, a bijection on 64-bit words: spreads group
    ranks over the int64 range so keys are not small consecutive integers."""
    x = np.asarray(x).astype(np.uint64)
    x ^= x >> np.uint64(30)
    x *= np.uint64(_MIX1)
    x ^= x >> np.uint64(27)
    x *= np.uint64(_MIX2)
    x ^= x >> np.uint64(31)
    return x.view(np.int64)


def mix64_torch(x):
    """mix64_np on an int64 tensor (wrapping multiplies, logical shifts)."""
    def srl(v, k):
        return (v >> k) & ((1 << (64 - k)) - 1)

    def signed(c):
        return c - (1 << 64) if c >= 1 << 63 else c

    x = x ^ srl(x, 30)
    x = x * signed(_MIX1)
    x = x ^ srl(x, 27)
    x = x * signed(_MIX2)
    return x ^ srl(x, 31)


def batched_specs(count=512, seed_idx=3, min_rows=1_000, max_rows=10_000_000, scale=1.0):
    """Per instance: rows log-U[min_rows,max_rows] (times scale), groups
    log-U[10,10^6], Zipf theta U[0,1.2], selectivity s U[0.01,0.9] and the
    predicate cut d < round(s*2526)."""
    g = rng(seed_idx)
    out = []
    for _ in range(count):
        rows = max(int(np.exp(g.uniform(np.log(min_rows), np.log(max_rows))) * scale), 1)
        groups = int(np.exp(g.uniform(np.log(10), np.log(1_000_000))))
        theta = g.uniform(0.0, 1.2)
        sel = g.uniform(0.01, 0.9)
        out.append({"rows": rows, "groups": groups, "theta": theta, "cut": int(round(sel * 2526))})
    return out


def batched_instances(count=512, seed_idx=3, min_rows=1_000, max_rows=10_000_000,
                      scale=1.0):
    """Independent filter + group-by instances (host columns): int64 keys
    Zipf(theta) over the instance's groups, qty/price as the fact table, d
    int32 U[0,2526) filtered by d < cut.  Yields the spec dicts with "cols"."""
    for i, s in enumerate(batched_specs(count, seed_idx, min_rows, max_rows, scale)):
        ig = rng(seed_idx, 10 + i)
        rows = s["rows"]
        keys = mix64_np(zipf_ranks(ig, rows, s["groups"], s["theta"]))
        qty = ig.integers(1, 51, rows, dtype=np.int64)
        price = ig.integers(90000, 10500001, rows, dtype=np.int64) / 100.0
        d = ig.integers(0, 2526, rows, dtype=np.int32)
        yield dict(s, cols=[keys, qty, price, d])


def batched_instances_device(specs, device, seed_idx=3):
    """The same instances generated on the device with torch's generator
    (same distributions, a different random stream): for batches too large
    to build on the host."""
    import torch
    out = []
    for i, s in enumerate(specs):
        gen = torch.Generator(device=device)
        gen.manual_seed(SEED + seed_idx * 1000 + i)
        rows, G, theta = s["rows"], s["groups"], s["theta"]
        if theta <= 0.0:
            ranks = torch.randint(0, G, (rows,), generator=gen, device=device, dtype=torch.int64)
        else:
            w = torch.arange(1, G + 1, device=device, dtype=torch.float64).pow(-theta)
            cdf = torch.cumsum(w, 0)
            cdf /= cdf[-1].clone()
            u = torch.rand(rows, generator=gen, device=device, dtype=torch.float64)
            ranks = torch.clamp(torch.searchsorted(cdf, u, right=True), max=G - 1)
        keys = mix64_torch(ranks)
        qty = torch.randint(1, 51, (rows,), generator=gen, device=device, dtype=torch.int64)
        price = torch.randint(90000, 10500001, (rows,), generator=gen, device=device,
                              dtype=torch.int64).to(torch.float64) / 100.0
        d = torch.randint(0, 2526, (rows,), generator=gen, device=device, dtype=torch.int32)
        out.append(dict(s, cols=[keys, qty, price, d]))
    return out


SERVED_MIX = (("groupby", 0.4), ("join", 0.3), ("sort", 0.2), ("filter", 0.1))


def served_specs(count, seed_idx=4, min_rows=10_000, max_rows=100_000_000, tables=8):
    """Requests of the served mixed stream: operator by SERVED_MIX, rows
    log-U[min_rows,max_rows], an offset into the resident column pools, a
    predicate cut (d < cut) and a build table id for probes."""
    g = rng(seed_idx)
    names = [m for m, _ in SERVED_MIX]
    p = np.array([w for _, w in SERVED_MIX])
    out = []
    for _ in range(count):
        op = names[int(g.choice(len(names), p=p))]
        rows = int(np.exp(g.uniform(np.log(min_rows), np.log(max_rows))))
        out.append({"op": op, "rows": rows, "offset": int(g.integers(0, max_rows - rows + 1)),
                    "cut": int(g.integers(126, 2400)), "table": int(g.integers(0, tables))})
    return out


def batched_predicate(cut):
    """d < cut on column 3 of a batched instance."""
    return abi.Pred.leaf(abi.FILTER_LT, 3, a=cut)
