"""Python face of the operators: a thin layer over the C ABI.

Mirrors the operator vocabulary of GHive (FilterPredicate / GroupByPredicate /
BaseJoinPredicate / Sink sort, gpu_impl/inc/Operator/*.hpp) for the tests,
the benchmark and Python callers.  Device columns are torch tensors on a CUDA
device (torch is used only for device memory and streams); host columns are
numpy arrays.  A column is a tensor/array, or a (values, isnull) pair with
isnull in Hive's isNull[] layout (one byte per row, nonzero = NULL), or a
Sentinel(values) wrapper for GHive's in-band NULL sentinels.
"""
import ctypes as C

import numpy as np

from . import abi
from ._lib import GhbError, lib

try:
    import torch
except ImportError:  # host-only use
    torch = None

_TORCH_TYPE = {}
if torch is not None:
    _TORCH_TYPE = {torch.int64: abi.LONG, torch.float64: abi.DOUBLE, torch.int32: abi.INT}
    _TYPE_TORCH = {abi.LONG: torch.int64, abi.DOUBLE: torch.float64, abi.INT: torch.int32}


class Sentinel:
    """A column whose NULLs are GHive's in-band sentinels (Table.hpp:29-52)."""

    def __init__(self, values):
        self.values = values


def _split(c):
    if isinstance(c, tuple) and len(c) == 3 and isinstance(c[0], str) and c[0] == "string":
        return c, None, abi.NULLS_NONE
    if isinstance(c, Sentinel):
        return c.values, None, abi.NULLS_SENTINEL
    if isinstance(c, tuple):
        return c[0], c[1], abi.NULLS_BYTEMAP
    return c, None, abi.NULLS_NONE


def _ptr(x):
    if x is None:
        return None
    if torch is not None and isinstance(x, torch.Tensor):
        return x.data_ptr()
    return x.ctypes.data


def _dtype_code(x):
    if torch is not None and isinstance(x, torch.Tensor):
        return _TORCH_TYPE[x.dtype]
    return abi.TYPE_OF_DTYPE[np.dtype(x.dtype)]


class _Cols:
    """ghb_column descriptors for a list of columns (keeps the arrays alive)."""

    def __init__(self, cols):
        self.keep = []
        descs = []
        for c in cols:
            v, isnull, mode = _split(c)
            if isinstance(v, tuple):   # ("string", utf-8 bytes, int32 [start,end) pairs)
                _, chars, idx = v
                d = abi.Column()
                d.type, d.null_mode = abi.STRING, abi.NULLS_NONE
                d.data, d.aux, d.n = _ptr(chars), _ptr(idx), len(idx) // 2
                self.keep += [chars, idx]
                descs.append(d)
                continue
            if torch is not None and isinstance(v, torch.Tensor):
                v = v.contiguous()
                if isnull is not None:
                    isnull = isnull.to(torch.uint8).contiguous()
            else:
                v = np.ascontiguousarray(v)
                if isnull is not None:
                    isnull = np.ascontiguousarray(isnull, dtype=np.uint8)
            d = abi.Column()
            d.type, d.null_mode = _dtype_code(v), mode
            d.data, d.is_null, d.n = _ptr(v), _ptr(isnull), len(v)
            self.keep += [v, isnull]
            descs.append(d)
        self.n = len(descs)
        self.arr = (abi.Column * max(1, self.n))(*descs)

    def __getitem__(self, i):
        return self.arr[i]

    @property
    def ptr(self):
        return C.addressof(self.arr)


class _Outs:
    """Output columns allocated on the device (torch) or host (numpy)."""

    def __init__(self, types, cap, device=None, with_nulls=True):
        self.cols = []
        descs = []
        for t in types:
            n = max(1, cap)
            if t == abi.STRING:   # [start,end) pairs into the input column's bytes
                data = torch.empty(2 * n, dtype=torch.int32, device=device) if device is not None else \
                    np.empty(2 * n, dtype=np.int32)
                nul = (torch.empty(n, dtype=torch.uint8, device=device) if device is not None else
                       np.empty(n, dtype=np.uint8)) if with_nulls else None
                o = abi.OutColumn()
                o.type, o.data, o.is_null = t, _ptr(data), _ptr(nul)
                descs.append(o)
                self.cols.append((data, nul))
                continue
            if device is not None:
                data = torch.empty(n, dtype=_TYPE_TORCH[t], device=device)
                nul = torch.empty(n, dtype=torch.uint8, device=device) if with_nulls else None
            else:
                data = np.empty(n, dtype=abi.NP_DTYPE[t])
                nul = np.empty(n, dtype=np.uint8) if with_nulls else None
            o = abi.OutColumn()
            o.type, o.data, o.is_null = t, _ptr(data), _ptr(nul)
            descs.append(o)
            self.cols.append((data, nul))
        self.arr = (abi.OutColumn * max(1, len(descs)))(*descs)

    @property
    def ptr(self):
        return C.addressof(self.arr)

    def rows(self, k):
        out = []
        for (d, nl), o in zip(self.cols, self.arr):
            d = d[:2 * k] if o.type == abi.STRING else d[:k]
            out.append((d, None if nl is None else nl[:k].bool() if torch is not None and
                        isinstance(nl, torch.Tensor) else nl[:k].astype(bool)))
        return out


def _pred(pred):
    if pred is None:
        return None, None
    s = pred.as_struct()
    return C.addressof(s), s


def _stream(stream):
    if stream is None:
        if torch is not None and torch.cuda.is_available():
            return torch.cuda.current_stream().cuda_stream
        return None
    return stream if isinstance(stream, int) else stream.cuda_stream


class JoinTable:
    """A device-resident build side (ghb_join_table)."""

    def __init__(self, ctx, handle, build_rows, keep):
        self.ctx, self.handle, self.build_rows, self._keep = ctx, handle, build_rows, keep

    def info(self):
        rows, dup, slots = C.c_int64(), C.c_int64(), C.c_int64()
        self.ctx._check(lib().ghb_join_table_info(self.ctx.h, self.handle, C.byref(rows),
                                                  C.byref(dup), C.byref(slots)))
        return rows.value, dup.value, slots.value

    def free(self):
        if self.handle:
            lib().ghb_join_table_free(self.ctx.h, self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class GroupByBatch:
    """A captured batch of filter + group-by instances (ghb_batch).

    outs[i] holds instance i's output columns and groups[i] its group count
    after launch() and a sync; results(i) slices them."""

    def __init__(self, ctx, handle, outs, groups, nkeys, keep):
        self.ctx, self.handle, self.outs, self.groups = ctx, handle, outs, groups
        self.nkeys, self._keep = nkeys, keep

    def launch(self, stream=None):
        self.ctx._check(lib().ghb_batch_launch(self.handle, _stream(stream)))

    def describe(self):
        import json
        buf = C.create_string_buffer(1 << 16)
        self.ctx._check(lib().ghb_batch_describe(self.handle, buf, len(buf)))
        return json.loads(buf.value.decode())

    def results(self, i, counts=None):
        g = int(self.groups[i]) if counts is None else int(counts[i])
        res = self.outs[i].rows(min(g, len(self.outs[i].cols[0][0])))
        return res[:self.nkeys], res[self.nkeys:], g

    def free(self):
        if self.handle:
            lib().ghb_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Context:
    """One ghb_ctx: device scratch, error state and kernel-launch counter."""

    def __init__(self, device=0, arena_bytes=0):
        h = C.c_void_p()
        st = lib().ghb_ctx_create(device, arena_bytes, C.byref(h))
        if st:
            raise GhbError(st, "ghb_ctx_create(device=%d) failed" % device)
        self.h = h
        self.device = device
        self.torch_device = "cuda:%d" % device

    def close(self):
        if self.h:
            lib().ghb_ctx_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, st):
        if st:
            raise GhbError(st, lib().ghb_last_error(self.h).decode())

    @property
    def launches(self):
        return lib().ghb_kernel_launches(self.h)

    def sync(self, stream=None):
        self._check(lib().ghb_sync(self.h, _stream(stream)))

    def set_spin_limit(self, polls):
        """Bound of this context's look-back waits (polls <= 0: the default)."""
        self._check(lib().ghb_ctx_set_spin_limit(self.h, int(polls)))

    def set_log(self, path, level=1, peak_gbs=0.0):
        """One JSON line per operator call of this context appended to `path`
        (level 2 also times each call on the device and synchronises it);
        path None closes the log."""
        self._check(lib().ghb_ctx_set_log(self.h, None if path is None else str(path).encode(), int(level),
                                          float(peak_gbs)))

    # ------------------------------------------------------------ device ops
    def filter(self, pred, cols, proj=None, capacity=None, stream=None, sync=True, with_nulls=True,
               outs=None):
        """FilterPredicate::process + FilterOperator::clean_data on device columns.
        with_nulls=False leaves out the outputs' NULL maps; outs reuses output
        columns made earlier (an _Outs of the projected types).

        Returns ([(values, isnull)] per projected column, row count tensor or int)."""
        cs = _Cols(cols)
        n = cs[0].n if cs.n else 0
        proj = list(range(cs.n)) if proj is None else list(proj)
        cap = n if capacity is None else capacity
        if outs is None:
            outs = _Outs([cs[j].type for j in proj], cap, self.torch_device, with_nulls=with_nulls)
        pa = (C.c_int32 * max(1, len(proj)))(*proj)
        d_rows = torch.zeros(1, dtype=torch.int64, device=self.torch_device)
        pp, keep = _pred(pred)
        self._check(lib().ghb_filter(self.h, pp, cs.ptr, cs.n, pa, len(proj), outs.ptr, cap,
                                     d_rows.data_ptr(), _stream(stream)))
        if not sync:
            return outs, d_rows
        self.sync(stream)
        k = int(d_rows.item())
        return outs.rows(min(k, cap)), k

    def filter_groupby(self, pred, cols, keys, aggs, capacity=None, max_groups=None, cfg=None,
                       stream=None, sync=True):
        """GroupByPredicate::gpu_execute fused with the filter.  aggs: [(type, col)]."""
        cs = _Cols(cols)
        n = cs[0].n if cs.n else 0
        types = [cs[k].type for k in keys]
        types += [abi.agg_out_type(t, cs[c].type if c >= 0 else abi.LONG) for t, c in aggs]
        cap = capacity if capacity is not None else (max_groups or max(n, 1))
        outs = _Outs(types, cap, self.torch_device)
        ka = (C.c_int32 * max(1, len(keys)))(*keys)
        ag = (abi.AggDesc * max(1, len(aggs)))()
        for i, (t, c) in enumerate(aggs):
            ag[i].type, ag[i].col = t, c
        if cfg is None:
            cfg = abi.GroupByCfg()
        if max_groups:
            cfg.max_groups = max_groups
        d_groups = torch.empty(1, dtype=torch.int64, device=self.torch_device)  # the finalize writes it
        pp, keep = _pred(pred)
        self._check(lib().ghb_filter_groupby(self.h, pp, cs.ptr, cs.n, ka, len(keys), ag, len(aggs),
                                             outs.ptr, cap, d_groups.data_ptr(), C.byref(cfg),
                                             _stream(stream)))
        if not sync:
            return outs, d_groups
        self.sync(stream)
        g = int(d_groups.item())
        res = outs.rows(min(g, cap))
        return res[:len(keys)], res[len(keys):], g

    def batch_groupby(self, instances, keys, aggs, autotune=True, block_threads=0, smem_slots=0,
                      load_factor=0.0, use_graph=True, stream=None):
        """Many filter + group-by instances of one signature in one captured launch.

        instances: [(pred, cols, capacity, max_groups)], cols device columns of
        the same types in every instance.  Returns a GroupByBatch; call
        launch() (and sync) to run it, as often as wanted."""
        nin = len(instances)
        arr = (abi.GroupByInstance * max(1, nin))()
        keep, outs = [], []
        ncols = None
        for i, (pred, cols, cap, mg) in enumerate(instances):
            cs = _Cols(cols)
            ncols = cs.n if ncols is None else ncols
            if cs.n != ncols:
                raise ValueError("instance %d has %d columns, instance 0 has %d" % (i, cs.n, ncols))
            types = [cs[k].type for k in keys]
            types += [abi.agg_out_type(t, cs[c].type if c >= 0 else abi.LONG) for t, c in aggs]
            o = _Outs(types, cap, self.torch_device)
            pp, pk = _pred(pred)
            arr[i].cols, arr[i].pred, arr[i].out = cs.ptr, pp, o.ptr
            arr[i].out_capacity, arr[i].max_groups = cap, mg or 0
            keep += [cs, pk, o]
            outs.append(o)
        ka = (C.c_int32 * max(1, len(keys)))(*keys)
        ag = (abi.AggDesc * max(1, len(aggs)))()
        for i, (t, c) in enumerate(aggs):
            ag[i].type, ag[i].col = t, c
        cfg = abi.BatchCfg()
        cfg.autotune, cfg.block_threads, cfg.smem_slots = int(autotune), block_threads, smem_slots
        cfg.load_factor, cfg.use_graph = load_factor, int(use_graph)
        groups = torch.zeros(max(1, nin), dtype=torch.int64, device=self.torch_device)
        h = C.c_void_p()
        self._check(lib().ghb_batch_groupby_create(self.h, arr, nin, ncols or 0, ka, len(keys), ag,
                                                   len(aggs), groups.data_ptr(), C.byref(cfg),
                                                   _stream(stream), C.byref(h)))
        return GroupByBatch(self, h.value, outs, groups, len(keys), keep + [arr, ka, ag])

    def join_build(self, key, build_payload=(), load_factor=0.0, l2_persist=False, stream=None):
        """Builds the device hash table; it keeps the build payload columns
        (the first two inline in its slots), which must outlive the table."""
        cs, bp = _Cols([key]), _Cols(build_payload)
        cfg = abi.JoinCfg()
        cfg.load_factor, cfg.l2_persist = load_factor, 1 if l2_persist else 0
        h = C.c_void_p()
        self._check(lib().ghb_join_build(self.h, cs.ptr, bp.ptr, bp.n, C.byref(cfg), C.byref(h),
                                         _stream(stream)))
        t = JoinTable(self, h, cs[0].n, (cs, bp))
        t.payload_types = [bp[j].type for j in range(bp.n)]
        return t

    def join_probe(self, table, probe_key, join_type=abi.INNER_JOIN, probe_payload=(),
                   capacity=None, rowids=True, stream=None, sync=True, outs=None):
        pk = _Cols([probe_key])
        ppl = _Cols(probe_payload)
        n = pk[0].n
        if capacity is None:
            _, dup, _ = table.info()
            capacity = max(1, n * max(1, dup))
        if outs is None:
            ob = _Outs(table.payload_types, capacity, self.torch_device)
            op = _Outs([ppl[j].type for j in range(ppl.n)], capacity, self.torch_device)
            prow = torch.empty(capacity, dtype=torch.int32, device=self.torch_device) if rowids else None
            brow = torch.empty(capacity, dtype=torch.int32, device=self.torch_device) if rowids else None
            d_rows = torch.zeros(1, dtype=torch.int64, device=self.torch_device)
            outs = (ob, op, prow, brow, d_rows)
        ob, op, prow, brow, d_rows = outs
        self._check(lib().ghb_join_probe(self.h, table.handle, pk.ptr, join_type, ob.ptr,
                                         ppl.ptr, ppl.n, op.ptr, _ptr(prow), _ptr(brow),
                                         capacity, d_rows.data_ptr(), _stream(stream)))
        if not sync:
            return outs
        self.sync(stream)
        k = int(d_rows.item())
        m = min(k, capacity)
        return {"rows": k, "probe_rowid": None if prow is None else prow[:m],
                "build_rowid": None if brow is None else brow[:m],
                "build": ob.rows(m), "probe": op.rows(m)}

    def sort(self, keys, orders=None, null_orders=None, payload=(), rowid=False, stream=None,
             sync=True, with_nulls=True, outs=None):
        """ORDER BY on device columns.  with_nulls=False leaves out the
        outputs' NULL maps (NULLs then carry their sentinels); outs = (key
        outputs, payload outputs) reuses output columns made earlier."""
        ks, ps = _Cols(keys), _Cols(payload)
        n = ks[0].n
        if outs is not None:
            ok, op = outs
        else:
            ok = _Outs([ks[j].type for j in range(ks.n)], n, self.torch_device, with_nulls=with_nulls)
            op = _Outs([ps[j].type for j in range(ps.n)], n, self.torch_device, with_nulls=with_nulls)
        rid = torch.empty(max(1, n), dtype=torch.int32, device=self.torch_device) if rowid else None
        o = (C.c_int32 * ks.n)(*(orders or [abi.ASC] * ks.n))
        no = (C.c_int32 * ks.n)(*(null_orders or [abi.NULLS_DEFAULT] * ks.n))
        self._check(lib().ghb_sort(self.h, ks.ptr, o, no, ks.n, ps.ptr, ps.n, ok.ptr, op.ptr,
                                   _ptr(rid), None, _stream(stream)))
        if sync:
            self.sync(stream)
        return ok.rows(n), op.rows(n), (None if rid is None else rid[:n])

    # -------------------------------------------------------------- host ops
    def filter_host(self, pred, cols, proj=None, capacity=None, outs=None):
        cs = _Cols(cols)
        n = cs[0].n if cs.n else 0
        proj = list(range(cs.n)) if proj is None else list(proj)
        cap = n if capacity is None else capacity
        outs = outs or _Outs([cs[j].type for j in proj], cap)
        pa = (C.c_int32 * max(1, len(proj)))(*proj)
        rows = C.c_int64()
        pp, keep = _pred(pred)
        self._check(lib().ghb_filter_host(self.h, pp, cs.ptr, cs.n, pa, len(proj), outs.ptr, cap,
                                          C.byref(rows)))
        return outs.rows(min(rows.value, cap)), rows.value

    def filter_groupby_host(self, pred, cols, keys, aggs, capacity, max_groups=None, outs=None):
        cs = _Cols(cols)
        types = [cs[k].type for k in keys]
        types += [abi.agg_out_type(t, cs[c].type if c >= 0 else abi.LONG) for t, c in aggs]
        outs = outs or _Outs(types, capacity)
        ka = (C.c_int32 * max(1, len(keys)))(*keys)
        ag = (abi.AggDesc * max(1, len(aggs)))()
        for i, (t, c) in enumerate(aggs):
            ag[i].type, ag[i].col = t, c
        cfg = abi.GroupByCfg()
        if max_groups:
            cfg.max_groups = max_groups
        g = C.c_int64()
        pp, keep = _pred(pred)
        self._check(lib().ghb_filter_groupby_host(self.h, pp, cs.ptr, cs.n, ka, len(keys), ag,
                                                  len(aggs), outs.ptr, capacity, C.byref(g),
                                                  C.byref(cfg)))
        res = outs.rows(min(g.value, capacity))
        return res[:len(keys)], res[len(keys):], g.value

    def hash_join_host(self, build_key, probe_key, join_type=abi.INNER_JOIN, build_payload=(),
                       probe_payload=(), capacity=None, rowids=True, load_factor=0.5, outs=None):
        bk, pk = _Cols([build_key]), _Cols([probe_key])
        bp, ppl = _Cols(build_payload), _Cols(probe_payload)
        cap = capacity or max(1, pk[0].n)
        if outs is None:
            ob = _Outs([bp[j].type for j in range(bp.n)], cap)
            op = _Outs([ppl[j].type for j in range(ppl.n)], cap)
            prow = np.empty(cap, dtype=np.int32) if rowids else None
            brow = np.empty(cap, dtype=np.int32) if rowids else None
            outs = (ob, op, prow, brow)
        ob, op, prow, brow = outs
        cfg = abi.JoinCfg()
        cfg.load_factor = load_factor
        rows = C.c_int64()
        self._check(lib().ghb_hash_join_host(self.h, bk.ptr, pk.ptr, join_type, bp.ptr, bp.n, ob.ptr,
                                             ppl.ptr, ppl.n, op.ptr, _ptr(prow), _ptr(brow), cap,
                                             C.byref(rows), C.byref(cfg)))
        m = min(rows.value, cap)
        return {"rows": rows.value, "probe_rowid": None if prow is None else prow[:m],
                "build_rowid": None if brow is None else brow[:m],
                "build": ob.rows(m), "probe": op.rows(m)}

    def sort_host(self, keys, orders=None, null_orders=None, payload=(), rowid=False, outs=None):
        ks, ps = _Cols(keys), _Cols(payload)
        n = ks[0].n
        if outs is None:
            ok = _Outs([ks[j].type for j in range(ks.n)], n)
            op = _Outs([ps[j].type for j in range(ps.n)], n)
            rid = np.empty(max(1, n), dtype=np.int32) if rowid else None
            outs = (ok, op, rid)
        ok, op, rid = outs
        o = (C.c_int32 * ks.n)(*(orders or [abi.ASC] * ks.n))
        no = (C.c_int32 * ks.n)(*(null_orders or [abi.NULLS_DEFAULT] * ks.n))
        self._check(lib().ghb_sort_host(self.h, ks.ptr, o, no, ks.n, ps.ptr, ps.n, ok.ptr, op.ptr,
                                        _ptr(rid), None))
        return ok.rows(n), op.rows(n), (None if rid is None else rid[:n])
