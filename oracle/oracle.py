"""Python face of the CPU oracle (oracle/hive_oracle.cpp).

TEST INFRASTRUCTURE: the parity checker and the timed CPU baseline.  Only the
tests, the smoke check and bench.py's CPU legs import this module; the
product package never does.

Columns are numpy arrays; a NULL-able column is passed as (values, isnull)
with isnull a bool/uint8 array in Hive's isNull[] layout.
"""
import ctypes as C
import os
import subprocess

import numpy as np

from ghive_b200 import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "lib", "libhive_oracle.so")
_lib = None


def build():
    """Compiles the oracle with its Makefile (g++)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        P, I32, I64 = C.c_void_p, C.c_int32, C.c_int64
        L.hive_filter.restype = I64
        L.hive_filter.argtypes = [P, P, I32, I64, P]
        L.hive_filter_groupby.restype = I64
        L.hive_filter_groupby.argtypes = [P, P, I32, I64, P, I32, P, I32, P, I64, P]
        L.hive_groupby_string_key.restype = I64
        L.hive_groupby_string_key.argtypes = [P, I32, I64, P, I32, P, I32, P, I64, P, P, I64]
        L.hive_hash_join.restype = I64
        L.hive_hash_join.argtypes = [P, P, I32, C.c_float, P, P, I64]
        L.hive_hashmap_lookup.restype = I64
        L.hive_hashmap_lookup.argtypes = [P, I64, C.c_float, I64, P, I64, P]
        L.hive_sort_perm.restype = None
        L.hive_sort_perm.argtypes = [P, P, P, I32, I64, P]
        L.hive_long_hash_code.restype = I64
        L.hive_long_hash_code.argtypes = [I64]
        L.hive_filter_groupby_mt.restype = I64
        L.hive_filter_groupby_mt.argtypes = [I32, P, P, I32, I64, P, I32, P, I32, P, I64]
        L.hive_hash_join_mt.restype = I64
        L.hive_hash_join_mt.argtypes = [I32, P, P, I32, P, I32, P, P, I64]
        L.hive_sort_perm_mt.restype = None
        L.hive_sort_perm_mt.argtypes = [I32, P, P, P, I32, I64, P]
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data


class Cols:
    """Holds numpy columns and their ghb_column descriptors alive together."""

    def __init__(self, columns, null_mode=None):
        self.keep = []
        descs = []
        for c in columns:
            d = abi.Column()
            if isinstance(c, tuple) and isinstance(c[0], str) and c[0] == "string":
                _, chars, idx = c
                chars = np.ascontiguousarray(np.frombuffer(chars, dtype=np.uint8))
                idx = np.ascontiguousarray(idx, dtype=np.int32)
                d.type, d.null_mode = abi.STRING, abi.NULLS_SENTINEL
                d.data, d.aux, d.n = _ptr(chars), _ptr(idx), len(idx) // 2
                self.keep += [chars, idx]
            else:
                vals, isnull = (c if isinstance(c, tuple) else (c, None))
                vals = np.ascontiguousarray(vals)
                d.type = abi.TYPE_OF_DTYPE[vals.dtype]
                d.data, d.n = _ptr(vals), len(vals)
                if isnull is not None:
                    isnull = np.ascontiguousarray(isnull, dtype=np.uint8)
                    d.null_mode, d.is_null = abi.NULLS_BYTEMAP, _ptr(isnull)
                    self.keep.append(isnull)
                else:
                    d.null_mode = abi.NULLS_NONE if null_mode is None else null_mode
                self.keep.append(vals)
            descs.append(d)
        self.arr = (abi.Column * max(1, len(descs)))(*descs)
        self.n = len(descs)

    def __getitem__(self, i):
        return self.arr[i]

    @property
    def ptr(self):
        return C.addressof(self.arr)


def _pred_ptr(pred):
    if pred is None:
        return None, None
    s = pred.as_struct()
    return C.addressof(s), s


def filter_rows(pred, columns, n=None):
    """Selected row indices (int64, ascending) of the rows passing pred."""
    cols = Cols(columns)
    n = cols[0].n if n is None else n
    out = np.empty(max(n, 1), dtype=np.int64)
    pp, keep = _pred_ptr(pred)
    k = lib().hive_filter(pp, cols.ptr, cols.n, n, out.ctypes.data)
    return out[:k]


def _out_cols(types, cap):
    outs, keep = [], []
    for t in types:
        o = abi.OutColumn()
        o.type = t
        data = np.empty(max(cap, 1), dtype=abi.NP_DTYPE[t])
        nul = np.empty(max(cap, 1), dtype=np.uint8)
        o.data, o.is_null = data.ctypes.data, nul.ctypes.data
        outs.append(o)
        keep.append((data, nul))
    arr = (abi.OutColumn * max(1, len(outs)))(*outs)
    return arr, keep


def _agg_arr(aggs):
    arr = (abi.AggDesc * max(1, len(aggs)))()
    for i, (t, c) in enumerate(aggs):
        arr[i].type, arr[i].col = t, c
    return arr


def filter_groupby(pred, columns, key_cols, aggs, cap=None, with_comp=False,
                   threads=0):
    """Hive hash group-by over the rows passing pred.

    Returns (keys, aggs[, comp]) where keys/aggs are lists of (values, isnull)
    numpy pairs, groups ordered by key (NULL first).  threads > 0 runs the
    multi-threaded CPU baseline instead of the sequential oracle.
    """
    cols = Cols(columns)
    n = cols[0].n if cols.n else 0
    types = [cols[k].type for k in key_cols]
    types += [abi.agg_out_type(t, cols[c].type if c >= 0 else abi.LONG) for t, c in aggs]
    cap = cap if cap is not None else max(n, 1)
    out, keep = _out_cols(types, cap)
    kc = (C.c_int32 * max(1, len(key_cols)))(*key_cols)
    ag = _agg_arr(aggs)
    comp = np.zeros(max(1, len(aggs) * cap), dtype=np.float64) if with_comp else None
    pp, pkeep = _pred_ptr(pred)
    if threads > 0:
        g = lib().hive_filter_groupby_mt(threads, pp, cols.ptr, cols.n, n, kc, len(key_cols),
                                         ag, len(aggs), out, cap)
    else:
        g = lib().hive_filter_groupby(pp, cols.ptr, cols.n, n, kc, len(key_cols), ag, len(aggs),
                                      out, cap, _ptr(comp))
    if g < 0:
        raise ValueError("group count %d exceeds capacity %d" % (-g, cap))
    res = [(d[:g].copy(), nl[:g].astype(bool)) for d, nl in keep]
    keys, vals = res[:len(key_cols)], res[len(key_cols):]
    if with_comp:
        c = [comp[i * cap:i * cap + g].copy() for i in range(len(aggs))]
        return keys, vals, c
    return keys, vals


def groupby_string_key(columns, key_cols, aggs):
    """Group-by with STRING key columns; keys come back as Python strings."""
    cols = Cols(columns)
    n = cols[0].n
    types = [abi.INT if cols[k].type == abi.STRING else cols[k].type for k in key_cols]
    types += [abi.agg_out_type(t, cols[c].type if c >= 0 else abi.LONG) for t, c in aggs]
    cap = max(n, 1)
    out, keep = _out_cols(types, cap)
    kc = (C.c_int32 * len(key_cols))(*key_cols)
    ag = _agg_arr(aggs)
    kidx = np.zeros(2 * cap * len(key_cols), dtype=np.int32)
    chars_cap = 1 << 16
    kchars = np.zeros(chars_cap, dtype=np.uint8)
    g = lib().hive_groupby_string_key(cols.ptr, cols.n, n, kc, len(key_cols), ag, len(aggs),
                                      out, cap, kidx.ctypes.data, kchars.ctypes.data, chars_cap)
    rows = []
    for r in range(g):
        row = []
        for j, k in enumerate(key_cols):
            if cols[k].type == abi.STRING:
                s, e = kidx[2 * (r * len(key_cols) + j)], kidx[2 * (r * len(key_cols) + j) + 1]
                row.append(None if s < 0 else bytes(kchars[s:e]).decode())
            else:
                d, nl = keep[j]
                row.append(None if nl[r] else d[r].item())
        for j in range(len(aggs)):
            d, nl = keep[len(key_cols) + j]
            row.append(None if nl[r] else d[r].item())
        rows.append(tuple(row))
    return rows


def hash_join(build_key, probe_key, join_type=abi.INNER_JOIN, load_factor=0.75):
    """(probe_rows, build_rows) int32 pairs in probe-row order."""
    bc, pc = Cols([build_key]), Cols([probe_key])
    n = pc[0].n
    cap = max(1, n)
    for _ in range(8):
        pr = np.empty(cap, dtype=np.int32)
        br = np.empty(cap, dtype=np.int32)
        k = lib().hive_hash_join(bc.ptr, pc.ptr, join_type, load_factor, pr.ctypes.data,
                                 br.ctypes.data, cap)
        if k >= 0:
            return pr[:k], br[:k]
        cap = -k
    raise RuntimeError("unreachable")


def hash_join_mt(threads, build_key, probe_key, build_payload, join_type=abi.INNER_JOIN,
                 cap=None):
    """Multi-threaded CPU baseline join with payload gather."""
    bc, pc, bp = Cols([build_key]), Cols([probe_key]), Cols(build_payload)
    n = pc[0].n
    cap = cap or n
    types = [bp[j].type for j in range(bp.n)]
    out, keep = _out_cols(types, cap)
    prow = np.empty(cap, dtype=np.int32)
    k = lib().hive_hash_join_mt(threads, bc.ptr, pc.ptr, join_type, bp.ptr, bp.n, out,
                                prow.ctypes.data, cap)
    if k < 0:
        raise ValueError("join output %d exceeds capacity %d" % (-k, cap))
    return prow[:k], [d[:k] for d, _ in keep]


def hashmap_lookup(keys, queries, load_factor=0.75, initial_capacity=8):
    keys = np.ascontiguousarray(keys, dtype=np.int64)
    queries = np.ascontiguousarray(queries, dtype=np.int64)
    found = np.zeros(max(1, len(queries)), dtype=np.int64)
    buckets = lib().hive_hashmap_lookup(keys.ctypes.data, len(keys), load_factor,
                                        initial_capacity, queries.ctypes.data, len(queries),
                                        found.ctypes.data)
    return found[:len(queries)], buckets


def sort_perm(keys, orders=None, null_orders=None, threads=0):
    """Stable permutation (int64) ordering rows by the key columns."""
    kc = Cols(keys)
    n = kc[0].n
    nk = kc.n
    o = (C.c_int32 * nk)(*(orders or [abi.ASC] * nk))
    no = (C.c_int32 * nk)(*(null_orders or [abi.NULLS_DEFAULT] * nk))
    perm = np.empty(max(1, n), dtype=np.int64)
    if threads > 0:
        lib().hive_sort_perm_mt(threads, kc.ptr, o, no, nk, n, perm.ctypes.data)
    else:
        lib().hive_sort_perm(kc.ptr, o, no, nk, n, perm.ctypes.data)
    return perm[:n]


def long_hash_code(key):
    return lib().hive_long_hash_code(int(key))
