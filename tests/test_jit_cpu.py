"""The specialised group-by kernels compile (NVRTC, sm_100a) for a spread of
signatures, with no GPU: key types and NULL modes, predicate shapes (leaf,
AND/OR tree, column-vs-column, double literals, NOT NULL), every aggregate
kind, global aggregates, and the batched fold."""
import ctypes as C

import numpy as np
import pytest

from ghive_b200 import abi
from ghive_b200._lib import lib
from ghive_b200.ops import Sentinel, _Cols


def _source(pred, cols, keys, aggs, batch=False):
    cs = _Cols(cols)
    ka = (C.c_int32 * max(1, len(keys)))(*keys)
    ag = (abi.AggDesc * max(1, len(aggs)))()
    for i, (t, c) in enumerate(aggs):
        ag[i].type, ag[i].col = t, c
    ps = pred.as_struct() if pred is not None else None
    buf = C.create_string_buffer(1 << 16)
    st = lib().ghb_jit_groupby_source(C.addressof(ps) if ps is not None else None, cs.ptr, cs.n, ka,
                                      len(keys), ag, len(aggs), int(batch), buf, len(buf))
    assert st == 0
    return buf.value


def _compile(src):
    n = C.c_int64()
    log = C.create_string_buffer(1 << 16)
    st = lib().ghb_jit_compile_source(src, C.byref(n), log, len(log))
    assert st == 0, log.value.decode()
    assert n.value > 0
    return n.value


N = 64
k32 = np.arange(N, dtype=np.int32)
k64 = np.arange(N, dtype=np.int64)
f64 = np.linspace(0, 1, N)
nul = np.zeros(N, dtype=np.uint8)

CASES = {
    "fact": (abi.Pred.leaf(abi.FILTER_LT, 3, a=1263), [k32, k64, f64, k32], [0],
             [(abi.CNT, -1), (abi.SUM, 1), (abi.SUM, 2), (abi.AVG, 2), (abi.MIN, 3), (abi.MAX, 3)]),
    "tree_nullable_bytemap": (abi.Pred.or_(abi.Pred.and_(abi.Pred.leaf(abi.FILTER_GE, 1, a=3),
                                                         abi.Pred.leaf(abi.FILTER_RANGE, 2, a=0.1, b=0.7)),
                                           abi.Pred.leaf(abi.FILTER_NOT_NULL, 0)),
                              [(k64, nul), (k64, nul), (f64, nul)], [0],
                              [(abi.CNT, 0), (abi.SUM, 1), (abi.MAX, 2), (abi.MIN, 2), (abi.AVG, 1)]),
    "col_vs_col_sentinel_key": (abi.Pred.leaf(abi.FILTER_LT, 1, col2=2), [Sentinel(k64), k64, f64], [0],
                                [(abi.CNT, -1), (abi.SUM, 2)]),
    "global_aggregate": (None, [k64, f64], [], [(abi.CNT, -1), (abi.SUM, 0), (abi.AVG, 1), (abi.MIN, 0)]),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_specialised_fold_compiles(name):
    pred, cols, keys, aggs = CASES[name]
    src = _source(pred, cols, keys, aggs)
    assert b"SigFolder" in src and b"fold_kernel_body" in src
    _compile(src)


def test_batched_fold_compiles():
    pred, cols, keys, aggs = CASES["fact"]
    src = _source(pred, cols, keys, aggs, batch=True)
    assert b"batch_fold_body" in src
    _compile(src)


def test_literals_are_not_part_of_the_signature():
    _, cols, keys, aggs = CASES["fact"]
    a = _source(abi.Pred.leaf(abi.FILTER_LT, 3, a=10), cols, keys, aggs)
    b = _source(abi.Pred.leaf(abi.FILTER_LT, 3, a=2000), cols, keys, aggs)
    assert a == b
    c = _source(abi.Pred.leaf(abi.FILTER_GT, 3, a=10), cols, keys, aggs)
    assert c != a


def test_rows_and_warp_combine_are_in_the_signature():
    """The folder's rows per thread and warp-combine mode are template
    arguments: a single call fixes warp combining (0 or 1), a batch decides it
    per instance at run time (2), a global aggregate never uses it."""
    pred, cols, keys, aggs = CASES["fact"]
    single = _source(pred, cols, keys, aggs)
    batch = _source(pred, cols, keys, aggs, batch=True)
    glob = _source(pred, cols, [], aggs)

    def sig_args(src):
        head = src.split(b"SigFolder<", 1)[1].split(b",")
        return int(head[0]), int(head[1]), head[2].strip()

    rows, wagg, keyed = sig_args(single)
    assert 1 <= rows <= 4 and wagg in (0, 1) and keyed == b"true"
    _, wagg_b, _ = sig_args(batch)
    assert wagg_b == 2
    _, wagg_g, keyed_g = sig_args(glob)
    assert wagg_g == 0 and keyed_g == b"false"
    for s in (single, batch, glob):
        _compile(s)
