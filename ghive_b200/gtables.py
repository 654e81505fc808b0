"""GHive's JNI input (GTables) and a vertex's operator chain, from Python.

A Tez task hands GHive a GTables object (ghive/GTables.java:13-31): per
input table the column types, row count, key count and vertex name, and the
columns as direct ByteBuffers concatenated by type over the tables.  The JNI
shim reads those fields into a ghb_gtables; this module builds the same
struct from numpy columns (the tests and Python callers), and runs a chain
of operators on it through ghb_run_plan, returning the result the way
GPUResult holds it (arrays grouped by type plus `sequence`).
"""
import ctypes as C

import numpy as np

from . import abi
from ._lib import GhbError, lib

GT_TYPE = {np.dtype(np.int64): 0, np.dtype(np.float64): 1, np.dtype(np.int32): 2}


class GTables:
    """tables: [(vertex_name or None, key_cnt, [column, ...])] where a column
    is a numpy int64 / float64 / int32 array (NULLs as GHive's sentinels) or
    ("string", utf8_bytes, int32 [start, end) pairs)."""

    def __init__(self, tables):
        self.keep = []
        types, ncols, rows, keys, names = [], [], [], [], []
        bufs = {0: [], 1: [], 2: [], 3: []}
        idx_bufs = []
        for name, key_cnt, cols in tables:
            tt, n = [], None
            for c in cols:
                if isinstance(c, tuple) and c[0] == "string":
                    chars = np.frombuffer(c[1], dtype=np.uint8).copy()
                    pairs = np.ascontiguousarray(c[2], dtype=np.int32)
                    self.keep += [chars, pairs]
                    bufs[3].append(chars.ctypes.data)
                    idx_bufs.append(pairs.ctypes.data)
                    tt.append(3)
                    n = len(pairs) // 2
                else:
                    a = np.ascontiguousarray(c)
                    self.keep.append(a)
                    t = GT_TYPE[a.dtype]
                    bufs[t].append(a.ctypes.data)
                    tt.append(t)
                    n = len(a)
            arr = (C.c_int32 * max(1, len(tt)))(*tt)
            self.keep.append(arr)
            types.append(C.cast(arr, C.c_void_p).value)
            ncols.append(len(tt))
            rows.append(n or 0)
            keys.append(key_cnt)
            names.append(None if name is None else name.encode())
        g = abi.GTables()
        nt = len(tables)
        self._ncols = (C.c_int32 * max(1, nt))(*ncols)
        self._types = (C.c_void_p * max(1, nt))(*types)
        self._rows = (C.c_int32 * max(1, nt))(*rows)
        self._keys = (C.c_int32 * max(1, nt))(*keys)
        self._names = (C.c_char_p * max(1, nt))(*names)
        self._bufs = {t: (C.c_void_p * max(1, len(v)))(*v) for t, v in bufs.items()}
        self._idx = (C.c_void_p * max(1, len(idx_bufs)))(*idx_bufs)
        g.ntables = nt
        g.ncols, g.types = C.addressof(self._ncols), C.addressof(self._types)
        g.row_cnt, g.key_cnt = C.addressof(self._rows), C.addressof(self._keys)
        g.vertex_name = C.addressof(self._names)
        g.nlong, g.long_cols = len(bufs[0]), C.addressof(self._bufs[0])
        g.ndouble, g.double_cols = len(bufs[1]), C.addressof(self._bufs[1])
        g.nint, g.int_cols = len(bufs[2]), C.addressof(self._bufs[2])
        g.nstring, g.string_cols = len(bufs[3]), C.addressof(self._bufs[3])
        g.string_idx_cols = C.addressof(self._idx)
        self.struct = g

    @property
    def ptr(self):
        return C.addressof(self.struct)

    def table(self, t, cap=abi.MAX_RESULT_COLS):
        """Column descriptors of input table t (ghb_gtables_table)."""
        cols = (abi.Column * cap)()
        n, rows = C.c_int32(), C.c_int64()
        st = lib().ghb_gtables_table(self.ptr, t, cols, cap, C.byref(n), C.byref(rows))
        if st:
            raise GhbError(st, "ghb_gtables_table(%d) failed" % t)
        return [cols[i] for i in range(n.value)], rows.value


def op_filter(pred, proj=None):
    return {"op": abi.OP_FILTER, "pred": pred, "idx": proj}


def op_groupby(keys, aggs, max_groups=0):
    return {"op": abi.OP_GROUPBY, "idx": list(keys), "aggs": list(aggs), "max_groups": max_groups}


def op_join(probe_key, build_table, build_key, build_keep=(), join_type=abi.INNER_JOIN):
    """probe_key / build_key: one column index each, or equally long lists
    (a key of several columns)."""
    pk = list(probe_key) if isinstance(probe_key, (list, tuple)) else [probe_key]
    bk = list(build_key) if isinstance(build_key, (list, tuple)) else [build_key]
    if len(pk) != len(bk):
        raise ValueError("probe and build keys differ in length")
    return {"op": abi.OP_JOIN_PROBE, "idx": pk + bk, "build_table": build_table,
            "build_keep": list(build_keep), "join_type": join_type}


def op_sort(keys, orders=None, null_orders=None):
    return {"op": abi.OP_SORT, "idx": list(keys), "orders": orders, "null_orders": null_orders}


def _ops_array(ops):
    keep = []
    arr = (abi.PlanOp * max(1, len(ops)))()
    for i, o in enumerate(ops):
        a = arr[i]
        a.op = o["op"]
        a.join_type = o.get("join_type", abi.INNER_JOIN)
        if o.get("pred") is not None:
            s = o["pred"].as_struct()
            keep.append(s)
            a.pred = C.addressof(s)
        if o.get("idx") is not None:
            ia = (C.c_int32 * max(1, len(o["idx"])))(*o["idx"])
            keep.append(ia)
            a.idx, a.nidx = C.addressof(ia), len(o["idx"])
        if o.get("aggs"):
            ag = (abi.AggDesc * len(o["aggs"]))()
            for j, (t, c) in enumerate(o["aggs"]):
                ag[j].type, ag[j].col = t, c
            keep.append(ag)
            a.aggs, a.naggs = C.addressof(ag), len(o["aggs"])
        a.max_groups = o.get("max_groups", 0)
        for name in ("orders", "null_orders"):
            if o.get(name) is not None:
                oa = (C.c_int32 * len(o[name]))(*o[name])
                keep.append(oa)
                setattr(a, name, C.addressof(oa))
        a.build_table = o.get("build_table", 0)
        bk = o.get("build_keep") or []
        if bk:
            ba = (C.c_int32 * len(bk))(*bk)
            keep.append(ba)
            a.build_keep, a.nbuild_keep = C.addressof(ba), len(bk)
    return arr, keep


def run_plan(ctx, gtables, input_table, ops):
    """Runs the chain on the device; returns a dict shaped like GPUResult:
    long/double/int column lists, row count and sequence, plus `columns`
    (the result columns in order, as (values, isnull) pairs; a STRING
    column's values are a list of bytes, None for NULL)."""
    arr, keep = _ops_array(ops)
    res = abi.PlanResult()
    st = lib().ghb_run_plan(ctx.h, gtables.ptr, input_table, arr, len(ops), C.byref(res))
    if st:
        raise GhbError(st, lib().ghb_last_error(ctx.h).decode())
    try:
        cols = []
        n = res.rows
        for i in range(res.ncols):
            t = res.types[i]
            if t == abi.STRING:   # pairs into the column's packed bytes -> bytes per row, None = NULL
                pairs = np.ctypeslib.as_array(C.cast(res.data[i], C.POINTER(C.c_int32)),
                                              shape=(2 * max(n, 1),))[:2 * n].reshape(-1, 2)
                nb = res.str_nbytes[i]
                blob = C.string_at(res.str_bytes[i], nb) if nb > 0 else b""
                vals = [None if a < 0 else blob[a:b] for a, b in pairs.tolist()]
                cols.append((vals, np.array([v is None for v in vals], dtype=bool)))
                continue
            dt = abi.NP_DTYPE[t]
            vals = np.ctypeslib.as_array(C.cast(res.data[i], C.POINTER(np.ctypeslib.as_ctypes_type(dt))),
                                         shape=(max(n, 1),))[:n].copy()
            if res.is_null[i]:
                nl = np.ctypeslib.as_array(C.cast(res.is_null[i], C.POINTER(C.c_uint8)),
                                           shape=(max(n, 1),))[:n].astype(bool)
            else:
                nl = np.zeros(n, dtype=bool)
            cols.append((vals, nl))
        by_type = {0: [], 1: [], 2: [], 3: []}
        for i in range(res.ncols):
            by_type[res.types[i]].append(cols[i][0])
        return {"columns": cols, "rows": n, "sequence": [res.sequence[i] for i in range(res.ncols)],
                "longCols": by_type[0], "doubleCols": by_type[1], "intCols": by_type[2],
                "stringCols": by_type[3], "types": [res.types[i] for i in range(res.ncols)]}
    finally:
        lib().ghb_plan_result_free(C.byref(res))
