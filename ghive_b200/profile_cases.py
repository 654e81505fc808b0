"""Small, fixed cases of each operator's kernels, for ncu captures.

    python -m ghive_b200.profile_cases <case> [reps]

Each case builds its inputs on cuda:0 and runs the operator `reps` times
(default 2), so that a capture can skip the first (cold) launch:

  groupby   filter d < 1263 + GROUP BY k over the 6M-row fact table
            (COUNT(*), SUM(qty), SUM(price), AVG(price), MIN(d), MAX(d))
  gbaggs    the same table, one call per aggregate list (COUNT(*); + SUM(qty);
            + SUM(price); + MIN(d), MAX(d); COUNT(*) without the predicate)
  gbcnt     the same table, COUNT(*) only
  batch     64 batched filter + group-by instances (rows log-U[1e3, 2e6])
  join      1.5M-key build, 20M-row probe with int64 + double build payloads
  sort      ORDER BY (d int32, k int64) with an int32 row id, 20M rows
"""
import sys

import torch

from ghive_b200 import abi, workloads
from ghive_b200.ops import Context, _Outs


def main(argv):
    case = argv[1]
    reps = int(argv[2]) if len(argv) > 2 else 2
    ctx = Context(0)
    dev = torch.device("cuda", 0)
    if case == "join":
        (bkey, bpay), (fk, _) = workloads.join_tables(1_500_000, 20_000_000, seed_idx=1)
        db = torch.from_numpy(bkey).to(dev)
        dp = [torch.from_numpy(c).to(dev) for c in bpay]
        df = torch.from_numpy(fk).to(dev)
        cap = 20_000_000
        ob = _Outs([abi.LONG, abi.DOUBLE], cap, dev, with_nulls=False)
        opp = _Outs([], cap, dev)
        prow = torch.empty(cap, dtype=torch.int32, device=dev)
        d_rows = torch.zeros(1, dtype=torch.int64, device=dev)
        t = ctx.join_build(db, build_payload=dp)
        for _ in range(reps):
            ctx.join_probe(t, df, abi.INNER_JOIN, capacity=cap, rowids=False, sync=True,
                           outs=(ob, opp, prow, None, d_rows))
        print("rows", int(d_rows.item()))
    elif case in ("groupby", "gbaggs", "gbcnt"):
        cols = [torch.from_numpy(c).to(dev) for c in workloads.fact_table(6_000_000, seed_idx=0)]
        pred = workloads.fact_predicate()
        lists = {"groupby": [("fact", pred, workloads.AGGS_FACT)],
                 "gbcnt": [("cnt", pred, [(abi.CNT, -1)])],
                 "gbaggs": [("cnt", pred, [(abi.CNT, -1)]),
                            ("cnt+sum_i", pred, [(abi.CNT, -1), (abi.SUM, 1)]),
                            ("cnt+sum_f", pred, [(abi.CNT, -1), (abi.SUM, 2)]),
                            ("cnt+min+max", pred, [(abi.CNT, -1), (abi.MIN, 3), (abi.MAX, 3)]),
                            ("cnt_nopred", None, [(abi.CNT, -1)])]}[case]
        for name, pr, aggs in lists:
            for _ in range(reps):
                _, _, g = ctx.filter_groupby(pr, cols, [0], aggs, capacity=1000, max_groups=1000)
            print(name, "groups", g)
    elif case == "sort":
        d, k, r = workloads.sort_table(20_000_000, seed_idx=2)
        dd, dk, dr = (torch.from_numpy(x).to(dev) for x in (d, k, r))
        for _ in range(reps):
            ctx.sort([dd, dk], payload=[dr])
        ctx.sync()
        print("sorted")
    elif case == "batch":
        specs = workloads.batched_specs(64, seed_idx=3, max_rows=2_000_000)
        inst = workloads.batched_instances_device(specs, dev)
        entries = [(workloads.batched_predicate(s["cut"]), it["cols"],
                    max(1, min(s["groups"], s["rows"])) + 8, s["groups"]) for s, it in zip(specs, inst)]
        b = ctx.batch_groupby(entries, [0], workloads.AGGS_FACT, autotune=False, use_graph=False)
        for _ in range(reps):
            b.launch()
        ctx.sync()
        print("rows", sum(s["rows"] for s in specs))
    else:
        raise SystemExit("unknown case %r; see the module docstring" % case)


if __name__ == "__main__":
    main(sys.argv)
