"""Host side of running the operators on several GPUs (one rank per GPU).

Every operator shards without a data-path exchange on this path:
  filter, group-by  each rank takes a contiguous row range (shard_range);
                    group-by ranks compute mergeable partial aggregates
                    (AVG travels as SUM + COUNT) and the partials are merged
                    on one rank (merge_groupby), the all-gather form that suits
                    small group counts;
  join              the build side is replicated, each rank probes its probe
                    row range; probe row ids are offset by the range start.
"""
import numpy as np

from . import abi


def shard_range(n, rank, world):
    """Rows [lo, hi) of `rank` when n rows are split as evenly as possible."""
    base, extra = divmod(n, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def partial_aggs(aggs):
    """The per-rank aggregates for `aggs` and, per original aggregate, the
    indices of its partials: AVG(c) becomes SUM(c) and COUNT(c)."""
    part, where = [], []
    for t, c in aggs:
        if t == abi.AVG:
            where.append((len(part), len(part) + 1))
            part += [(abi.SUM, c), (abi.CNT, c)]
        else:
            where.append((len(part),))
            part.append((t, c))
    return part, where


def merge_groupby(parts, aggs, has_key=True):
    """Merges per-rank partial group-by results.

    parts: per rank (key, vals), key = (values, isnull) or None, vals = list of
    (values, isnull) for partial_aggs(aggs)[0].  Returns (key, vals) for
    `aggs`, groups ordered by key (NULL first)."""
    _, where = partial_aggs(aggs)
    if has_key:
        kv = np.concatenate([p[0][0] for p in parts])
        kn = np.concatenate([np.asarray(p[0][1], bool) for p in parts])
        ukey = np.where(kn, 0, kv)
        # NULL keys form their own group, ordered first
        order = np.lexsort((ukey, ~kn))
        kv, kn, ukey = kv[order], kn[order], ukey[order]
        new = np.ones(len(kv), bool)
        new[1:] = (ukey[1:] != ukey[:-1]) | (kn[1:] != kn[:-1])
        gid = np.cumsum(new) - 1
        ng = int(gid[-1]) + 1 if len(gid) else 0
        key = (kv[new], kn[new])
    else:
        order = np.arange(len(parts))
        gid = np.zeros(len(parts), np.int64)
        ng = 1
        key = None

    def col(j):
        v = np.concatenate([p[1][j][0] for p in parts])[order]
        n = np.concatenate([np.asarray(p[1][j][1], bool) for p in parts])[order]
        return v, n

    out = []
    for (t, c), w in zip(aggs, where):
        v, n = col(w[0])
        if t in (abi.SUM, abi.CNT, abi.AVG):
            s = np.zeros(ng, dtype=v.dtype)
            seen = np.zeros(ng, bool)
            if v.dtype.kind == "f":
                np.add.at(s, gid[~n], v[~n])
            else:
                # int64 sums wrap like Hive's
                np.add.at(s.view(np.uint64), gid[~n], v[~n].view(np.uint64))
            np.logical_or.at(seen, gid[~n], True)
            if t == abi.AVG:
                cv, cn = col(w[1])
                cnt = np.zeros(ng, np.int64)
                np.add.at(cnt, gid[~cn], cv[~cn])
                avg = np.where(cnt > 0, s / np.maximum(cnt, 1), 0.0)
                out.append((avg, cnt == 0))
            elif t == abi.CNT:
                out.append((s, np.zeros(ng, bool)))
            else:
                out.append((s, ~seen))
        else:
            fill = np.inf if v.dtype.kind == "f" else np.iinfo(v.dtype).max
            if t == abi.MAX:
                fill = -np.inf if v.dtype.kind == "f" else np.iinfo(v.dtype).min
            r = np.full(ng, fill, dtype=v.dtype)
            (np.minimum if t == abi.MIN else np.maximum).at(r, gid[~n], v[~n])
            seen = np.zeros(ng, bool)
            np.logical_or.at(seen, gid[~n], True)
            out.append((r, ~seen))
    return key, out
