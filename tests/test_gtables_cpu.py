"""GHive's GTables input, read without a GPU.

A Tez task's GTables (ghive/GTables.java:13-31) carries each input table's
column types and the columns as direct buffers concatenated by type over the
tables in table order; GPUProcess takes each column from the next unused
buffer of its type (ghive_JNIInterface.cu:132-201).  ghb_gtables_table must
hand out exactly those buffers, with GHive's sentinel NULL convention, and
refuse a missing table or a short buffer list.
"""
import numpy as np
import pytest

from ghive_b200 import abi
from ghive_b200._lib import GhbError
from ghive_b200.gtables import GTables


def _tables():
    g = np.random.default_rng(5)
    t0 = [g.integers(0, 9, 10, dtype=np.int64), g.random(10), g.integers(0, 9, 10, dtype=np.int32),
          g.integers(0, 9, 10, dtype=np.int64)]
    t1 = [g.random(7), g.integers(0, 9, 7, dtype=np.int32),
          ("string", b"abcdefg", np.array([0, 1, 1, 3, 3, 3, 3, 4, -1, -1, 4, 6, 6, 7], dtype=np.int32))]
    t2 = [g.integers(0, 9, 4, dtype=np.int64), g.integers(0, 9, 4, dtype=np.int32)]
    return t0, t1, t2


def test_columns_come_from_the_next_buffer_of_their_type():
    t0, t1, t2 = _tables()
    gt = GTables([("Map 1", 1, t0), ("Map 2", 0, t1), ("Reducer 3", 2, t2)])
    for t, cols in enumerate((t0, t1, t2)):
        descs, rows = gt.table(t)
        assert len(descs) == len(cols)
        for d, c in zip(descs, cols):
            if isinstance(c, tuple):
                assert d.type == abi.STRING and d.n == len(c[2]) // 2
                assert d.aux == c[2].ctypes.data
            else:
                assert d.type == abi.TYPE_OF_DTYPE[c.dtype] and d.n == len(c) == rows
            assert d.null_mode == abi.NULLS_SENTINEL
        # the very buffers, in order (no copy)
        keep = [a for a in gt.keep if isinstance(a, np.ndarray)]
        for d, c in zip(descs, cols):
            arr = c[1] if isinstance(c, tuple) else c
            match = [a for a in keep if a.ctypes.data == d.data]
            assert match and (isinstance(c, tuple) or np.array_equal(match[0], arr))


def test_missing_table_and_short_buffer_lists_are_refused():
    t0, t1, t2 = _tables()
    gt = GTables([("Map 1", 1, t0), (None, 0, t1)])
    gt.table(0)
    with pytest.raises(GhbError) as e:
        gt.table(1)
    assert e.value.code == abi.ERR_INVALID
    with pytest.raises(GhbError):
        gt.table(2)
    # a table claims one LONG column more than there are buffers
    gt2 = GTables([("Map 1", 1, t2)])
    gt2.struct.nlong = 0
    with pytest.raises(GhbError):
        gt2.table(0)
