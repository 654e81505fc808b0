"""Python face of the operator server (ghb_server_*): requests from many
threads, admitted by free slots and HBM budget, run concurrently on the GPU.

A request's input tensors must stay alive until it is done; wait() returns a
ServedResult whose device outputs (views on the server's memory) stay valid
until release().
"""
import ctypes as C

import torch

from . import abi
from ._lib import GhbError, lib
from .ops import _Cols, _pred

_NP = {abi.LONG: torch.int64, abi.DOUBLE: torch.float64, abi.INT: torch.int32}


class _DevView:
    """A device buffer as __cuda_array_interface__, for torch.as_tensor."""

    def __init__(self, ptr, n, dtype):
        typestr = {torch.int64: "<i8", torch.float64: "<f8", torch.int32: "<i4",
                   torch.uint8: "|u1"}[dtype]
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr,
                                         "data": (ptr, False), "version": 3, "strides": None}


def _view(ptr, n, dtype, device):
    if not ptr or n == 0:
        return torch.empty(0, dtype=dtype, device=device)
    return torch.as_tensor(_DevView(ptr, n, dtype), device=device)


class ServedResult:
    def __init__(self, res, device):
        self.status, self.rows = res.status, res.rows
        self.submit_ns, self.admit_ns, self.done_ns = res.submit_ns, res.admit_ns, res.done_ns
        self.launched_ns, self.slot = res.launched_ns, res.slot
        n = max(0, res.rows)
        self.cols = []
        for j in range(res.ncols):
            o = res.cols[j]
            v = _view(o.data, n, _NP[o.type], device)
            nl = _view(o.is_null, n, torch.uint8, device).bool() if o.is_null else None
            self.cols.append((v, nl))
        self.rowid = _view(res.rowid, n, torch.int32, device) if res.rowid else None
        self.rowid2 = _view(res.rowid2, n, torch.int32, device) if res.rowid2 else None

    @property
    def latency_ms(self):
        return (self.done_ns - self.submit_ns) / 1e6


class Server:
    def __init__(self, device=0, slots=8, hbm_budget=0):
        self.device = torch.device("cuda", device)
        cfg = abi.ServerCfg()
        cfg.slots, cfg.hbm_budget = slots, hbm_budget
        h = C.c_void_p()
        st = lib().ghb_server_create(device, C.byref(cfg), C.byref(h))
        if st:
            raise GhbError(st, "ghb_server_create failed")
        self.h = h.value
        self._tables = []   # keeps build columns alive

    def _check(self, st):
        if st:
            raise GhbError(st, (lib().ghb_server_last_error(self.h) or b"").decode())

    def close(self):
        if self.h:
            lib().ghb_server_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def add_join_table(self, key, payload=(), load_factor=0.0):
        ks, ps = _Cols([key]), _Cols(payload)
        tid = C.c_int32()
        self._check(lib().ghb_server_add_join_table(self.h, ks.ptr, ps.ptr if ps.n else None, ps.n,
                                                    load_factor, C.byref(tid)))
        self._tables.append((ks, ps))
        return tid.value

    def _submit(self, req, keep):
        t = C.c_uint64()
        self._check(lib().ghb_server_submit(self.h, C.byref(req), C.byref(t)))
        return t.value

    def submit_filter(self, pred, cols, proj=None):
        cs = _Cols(cols)
        pp, pk = _pred(pred)
        r = abi.Request()
        r.op, r.ncols, r.cols, r.pred = abi.OP_FILTER, cs.n, cs.ptr, pp
        pa = None
        if proj is not None:
            pa = (C.c_int32 * max(1, len(proj)))(*proj)
            r.idx, r.nidx = C.addressof(pa), len(proj)
        return self._submit(r, (cs, pk, pa))

    def submit_groupby(self, pred, cols, keys, aggs, max_groups):
        cs = _Cols(cols)
        pp, pk = _pred(pred)
        ka = (C.c_int32 * max(1, len(keys)))(*keys)
        ag = (abi.AggDesc * max(1, len(aggs)))()
        for i, (t, c) in enumerate(aggs):
            ag[i].type, ag[i].col = t, c
        r = abi.Request()
        r.op, r.ncols, r.cols, r.pred = abi.OP_GROUPBY, cs.n, cs.ptr, pp
        r.idx, r.nidx, r.aggs, r.naggs = C.addressof(ka), len(keys), C.addressof(ag), len(aggs)
        r.max_groups = max_groups
        return self._submit(r, (cs, pk, ka, ag))

    def submit_join(self, table, probe_key, join_type=abi.INNER_JOIN, build_rowid=False):
        cs = _Cols([probe_key])
        r = abi.Request()
        r.op, r.ncols, r.cols, r.table, r.join_type = abi.OP_JOIN_PROBE, 1, cs.ptr, table, join_type
        r.want_rowid = int(build_rowid)
        return self._submit(r, (cs,))

    def submit_sort(self, keys, payload=(), orders=None, null_orders=None, rowid=False):
        cs = _Cols(list(keys) + list(payload))
        r = abi.Request()
        r.op, r.ncols, r.cols, r.nkeys, r.want_rowid = abi.OP_SORT, cs.n, cs.ptr, len(keys), int(rowid)
        oa = na = None
        if orders is not None:
            oa = (C.c_int32 * len(keys))(*orders)
            r.orders = C.addressof(oa)
        if null_orders is not None:
            na = (C.c_int32 * len(keys))(*null_orders)
            r.null_orders = C.addressof(na)
        return self._submit(r, (cs, oa, na))

    def wait(self, ticket, check=True):
        res = abi.Result()
        st = lib().ghb_server_wait(self.h, ticket, C.byref(res))
        if st and check:
            self._check(st)
        return ServedResult(res, self.device)

    def release(self, ticket):
        self._check(lib().ghb_server_release(self.h, ticket))

    def stats(self):
        v = [C.c_int64() for _ in range(4)]
        self._check(lib().ghb_server_stats(self.h, *[C.byref(x) for x in v]))
        return dict(zip(("completed", "running", "queued", "bytes_admitted"), (x.value for x in v)))
