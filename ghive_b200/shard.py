"""Host side of running the operators on several GPUs (one rank per GPU).

  filter, group-by  each rank takes a contiguous row range (shard_range);
                    group-by ranks compute mergeable partial aggregates on
                    the device (AVG travels as SUM + COUNT), exchange them by
                    the hash of their key (one all-to-all per column) and
                    merge them with the device group-by (groupby_sharded);
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
    indices of its partials: AVG(c) becomes SUM(c) and COUNT(c).  A partial
    two aggregates need (SUM(c) for both SUM(c) and AVG(c)) is computed once."""
    part, where = [], []

    def index(a):
        if a not in part:
            part.append(a)
        return part.index(a)
    for t, c in aggs:
        if t == abi.AVG:
            where.append((index((abi.SUM, c)), index((abi.CNT, c))))
        else:
            where.append((index((t, c)),))
    return part, where


def merge_aggs(aggs, first=1):
    """The aggregates that merge partial_aggs(aggs)[0]'s columns: partial j,
    column first + j of a table (key, partial 0, partial 1, ...), is summed
    (SUM, COUNT) or reduced by MIN / MAX."""
    part, _ = partial_aggs(aggs)
    return [(abi.SUM if t in (abi.SUM, abi.CNT) else t, first + j) for j, (t, _c) in enumerate(part)]


def groupby_sharded(cols, key_col, aggs, local_groupby, pred=None, group=None):
    """Filter + GROUP BY over row-sharded columns, one rank per GPU.

    Each rank aggregates its own rows into partial aggregates (local_groupby,
    the device operator; AVG travels as SUM + COUNT), sends each partial row
    to the rank that owns its key (the key's 64-bit mix modulo the world size;
    NULL keys to rank 0) with one all-to-all per column, and merges what it
    receives with a second local_groupby over the partial rows (SUM of sums
    and counts, MIN of minima, MAX of maxima).  AVG is the merged SUM over the
    merged COUNT.  The ranks end up with disjoint sets of groups.

    local_groupby(pred, cols, keys, aggs) -> ((key values, key isnull),
    [(values, isnull) per aggregate]) with torch tensors on this rank's
    device (isnull a bool tensor, or None when no row is NULL).
    key_col None is a global aggregate: every rank's partial row goes to rank
    0, which returns the one result row (the others return none).  The key
    is a fixed-width column (a STRING key's [start,end) pairs point into
    its own rank's bytes and do not travel).
    Returns (key or None, [(values, isnull) per aggregate of `aggs`])."""
    import torch
    import torch.distributed as dist

    from .workloads import mix64_torch

    part, where = partial_aggs(aggs)
    keyed = key_col is not None
    key, vals = local_groupby(pred, cols, [key_col] if keyed else [], part)
    first = vals[0][0] if vals else key[0]
    dev = first.device
    g = len(first)

    def nulls(nl):
        return torch.zeros(g, dtype=torch.bool, device=dev) if nl is None else nl.to(torch.bool)

    columns = ([(key[0], nulls(key[1]))] if keyed else []) + [(v, nulls(n)) for v, n in vals]
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    if world > 1:
        if keyed:
            kv = key[0]
            bits = kv.view(torch.int64) if kv.element_size() == 8 else kv.to(torch.int64)
            owner = torch.remainder(mix64_torch(bits), world)
            owner = torch.where(columns[0][1], torch.zeros_like(owner), owner)
        else:   # a global aggregate: every partial row goes to rank 0
            owner = torch.zeros(g, dtype=torch.int64, device=dev)
        order = torch.argsort(owner, stable=True)
        send = torch.bincount(owner, minlength=world)
        recv = torch.empty_like(send)
        dist.all_to_all_single(recv, send, group=group)
        send_l, recv_l = send.tolist(), recv.tolist()
        moved = []
        for v, n in columns:
            pair = []
            for t in (v[order].contiguous(), n[order].to(torch.uint8).contiguous()):
                out = torch.empty(sum(recv_l), dtype=t.dtype, device=dev)
                dist.all_to_all_single(out, t, recv_l, send_l, group=group)
                pair.append(out)
            moved.append((pair[0], pair[1].to(torch.bool)))
        columns = moved
    # the owner's merge: GROUP BY the key over the partial rows (a COUNT
    # partial is never NULL: it goes without a NULL map, so its merge needs
    # no non-NULL count)
    off = 1 if keyed else 0
    for j, (t, _c) in enumerate(part):
        if t == abi.CNT:
            columns[off + j] = columns[off + j][0]
    mkey, mvals = local_groupby(None, columns, [0] if keyed else [], merge_aggs(aggs, off))
    ng = len(mvals[0][0]) if mvals else len(mkey[0])
    out = []
    for (t, _c), w in zip(aggs, where):
        v, n = mvals[w[0]]
        n = torch.zeros(ng, dtype=torch.bool, device=v.device) if n is None else n.to(torch.bool)
        if t == abi.AVG:
            cnt, _ = mvals[w[1]]
            empty = cnt == 0
            avg = torch.where(empty, torch.zeros_like(v, dtype=torch.float64),
                              v.to(torch.float64) / torch.clamp(cnt, min=1).to(torch.float64))
            out.append((avg, empty))
        elif t == abi.CNT:
            out.append((v, torch.zeros(ng, dtype=torch.bool, device=v.device)))
        else:
            out.append((v, n))
    if not keyed and world > 1 and dist.get_rank(group) != 0:
        return None, [(v[:0], n[:0]) for v, n in out]   # rank 0 holds the one row
    return (mkey if keyed else None), out


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
