"""Host side of running the operators on several GPUs (one rank per GPU).

  filter, group-by  each rank takes a contiguous row range (shard_range);
                    group-by ranks compute mergeable partial aggregates
                    (AVG travels as SUM + COUNT) and the partials are merged
                    on one rank (merge_groupby), the all-gather form that suits
                    small group counts;
  join              the build side is replicated, each rank probes its probe
                    row range; probe row ids are offset by the range start;
  sort              sample sort (sort_sharded): splitters from an all-gathered
                    sample of every rank's leading key, each rank's rows
                    range-partitioned by them, one all-to-all per column
                    (NCCL over NVLink between GPUs), then the stable local sort.
"""
import numpy as np

from . import abi

I64_MIN, I64_MAX = -(1 << 63), (1 << 63) - 1


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


# ------------------------------------------------------------ sample sort
def order_image(values, isnull, desc, nulls_first):
    """int64 values whose signed order is the ORDER BY order of one key column
    (BinarySortable order: integers by value, doubles by IEEE total order;
    DESC reversed; NULLs first or last).  Monotone but not one-to-one: rows
    that tie here are told apart by the local sort."""
    import torch
    if values.dtype == torch.float64:
        b = values.view(torch.int64)
        # IEEE total order as a signed int64: negative doubles' bits reversed
        img = torch.where(b < 0, b ^ I64_MAX, b)
    else:
        img = values.to(torch.int64)
    if desc:
        img = ~img
    if isnull is not None:
        img = torch.where(isnull.bool(), torch.full_like(img, I64_MIN if nulls_first else I64_MAX), img)
    return img


def choose_splitters(samples, world):
    """world - 1 splitters from the all-gathered sorted sample."""
    import torch
    s, _ = torch.sort(samples)
    if s.numel() == 0:
        return s[:0]
    idx = torch.tensor([(i * s.numel()) // world for i in range(1, world)], dtype=torch.int64,
                       device=s.device)
    return s[idx]


def sort_sharded(keys, payload, local_sort, orders=None, null_orders=None, group=None,
                 sample_per_rank=4096):
    """Stable ORDER BY over the rows of all ranks, each rank holding a shard.

    keys / payload: this rank's columns, each a tensor or (values, isnull)
    pair (a CUDA tensor under NCCL, a CPU tensor under gloo).  local_sort(keys,
    payload, orders, null_orders) sorts one rank's received rows and returns
    (keys, payload) in the same column forms (the device sort, Context.sort,
    on a GPU).  The result on rank r is the r-th range of the global order;
    rows with equal keys keep the order of (rank, row) of the input, because
    equal leading keys always go to one rank and the all-to-all delivers the
    source ranks in order.  Returns this rank's sorted (keys, payload)."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    nk = len(keys)
    orders = orders or [abi.ASC] * nk
    null_orders = null_orders or [abi.NULLS_DEFAULT] * nk

    def split(c):
        return (c[0], c[1]) if isinstance(c, tuple) else (c, None)

    v0, n0 = split(keys[0])
    desc = orders[0] == abi.DESC
    nf = null_orders[0] == abi.NULLS_FIRST or (null_orders[0] == abi.NULLS_DEFAULT and not desc)
    img = order_image(v0, n0, desc, nf)
    n = img.numel()
    dev = img.device
    # splitters from an evenly spaced sample of every rank's leading key
    m = min(sample_per_rank, n)
    pick = (torch.arange(m, device=dev, dtype=torch.int64) * n) // max(m, 1)
    local = img[pick] if m else img[:0]
    counts = [torch.zeros(1, dtype=torch.int64, device=dev) for _ in range(world)]
    dist.all_gather(counts, torch.tensor([m], dtype=torch.int64, device=dev), group=group)
    sizes = [int(c.item()) for c in counts]
    mx = max(sizes)
    padded = torch.full((mx,), I64_MAX, dtype=torch.int64, device=dev)
    padded[:m] = local
    gathered = [torch.empty(mx, dtype=torch.int64, device=dev) for _ in range(world)]
    dist.all_gather(gathered, padded, group=group)
    samples = torch.cat([g[:sz] for g, sz in zip(gathered, sizes)])
    splitters = choose_splitters(samples, world)
    # destination rank of each row; rows keep their order within a destination
    dest = torch.searchsorted(splitters, img, right=True) if world > 1 else \
        torch.zeros(n, dtype=torch.int64, device=dev)
    order = torch.argsort(dest, stable=True)
    send = torch.bincount(dest, minlength=world).to(torch.int64)
    recv = torch.empty_like(send)
    dist.all_to_all_single(recv, send, group=group)
    send_l, recv_l = send.tolist(), recv.tolist()

    def exchange(t):
        t = t[order].contiguous()
        out = torch.empty((sum(recv_l),) + tuple(t.shape[1:]), dtype=t.dtype, device=dev)
        dist.all_to_all_single(out, t, recv_l, send_l, group=group)
        return out

    def move(c):
        v, nl = split(c)
        v2 = exchange(v)
        if nl is None:
            return v2
        return (v2, exchange(nl.to(torch.uint8)))

    return local_sort([move(c) for c in keys], [move(c) for c in payload], orders, null_orders)
