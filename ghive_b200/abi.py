"""ctypes mirror of include/ghive_b200.h (structs and constants only).

The values of the enums are GHive's own (ColumnType in
gpu_impl/inc/DataFlow/Column.hpp:5-11, PredicateMode in
gpu_impl/inc/Operator/FilterPredicate.hpp:17-58, AggregationType in
gpu_impl/inc/Operator/AggregationDesc.hpp:6-25, BaseJoinType in
gpu_impl/inc/Operator/BaseJoinPredicate.hpp:11-25), so a caller that speaks
GHive's vocabulary passes its numbers through unchanged.
"""
import ctypes as C

import numpy as np

# status codes
OK, ERR_INVALID, ERR_OOM, ERR_CUDA, ERR_TIMEOUT, ERR_CAPACITY, ERR_UNSUPPORTED = range(7)
STATUS_NAMES = {0: "OK", 1: "INVALID", 2: "OOM", 3: "CUDA", 4: "TIMEOUT",
                5: "CAPACITY", 6: "UNSUPPORTED"}

# column types (GHive ColumnType)
LONG, DOUBLE, INT, STRING = 0, 1, 2, 3
NP_DTYPE = {LONG: np.int64, DOUBLE: np.float64, INT: np.int32}
TYPE_OF_DTYPE = {np.dtype(np.int64): LONG, np.dtype(np.float64): DOUBLE,
                 np.dtype(np.int32): INT}

# NULL conventions
NULLS_NONE, NULLS_SENTINEL, NULLS_BYTEMAP = 0, 1, 2
SENTINEL = {LONG: np.iinfo(np.int64).max, INT: np.iinfo(np.int32).max, DOUBLE: np.nan}

# predicate modes (GHive PredicateMode)
(FILTER_EQ, FILTER_LE, FILTER_GE, FILTER_LT, FILTER_GT, FILTER_RANGE,
 FILTER_EQ_RANGE, FILTER_NOT_EQ, FILTER_NOT_RANGE, FILTER_NOT_EQ_RANGE,
 FILTER_NOT_NULL, FILTER_AND, FILTER_OR) = range(13)
MAX_PRED_NODES = 32

# aggregation types (GHive AggregationType)
SUM, MAX, MIN, AVG, CNT = 0, 1, 2, 3, 4
AGG_NAMES = {"sum": SUM, "max": MAX, "min": MIN, "avg": AVG, "count": CNT}

# join types (GHive BaseJoinType)
INNER_JOIN, LEFT_OUTER_JOIN, LEFT_SEMI_JOIN = 0, 1, 4

# sort
ASC, DESC = 0, 1
NULLS_DEFAULT, NULLS_FIRST, NULLS_LAST = 0, 1, 2


class Column(C.Structure):
    _fields_ = [("type", C.c_int32), ("null_mode", C.c_int32),
                ("data", C.c_void_p), ("is_null", C.c_void_p),
                ("aux", C.c_void_p), ("n", C.c_int64)]


class OutColumn(C.Structure):
    _fields_ = [("type", C.c_int32), ("reserved", C.c_int32),
                ("data", C.c_void_p), ("is_null", C.c_void_p)]


class PredNode(C.Structure):
    _fields_ = [("mode", C.c_int32), ("col", C.c_int32), ("col2", C.c_int32),
                ("lit_is_double", C.c_int32), ("child", C.c_int32 * 2),
                ("lit_i", C.c_int64 * 2), ("lit_d", C.c_double * 2),
                ("lit_s", C.c_void_p * 2), ("lit_s_len", C.c_int32 * 2)]


class Predicate(C.Structure):
    _fields_ = [("n_nodes", C.c_int32), ("root", C.c_int32),
                ("nodes", C.POINTER(PredNode))]


class AggDesc(C.Structure):
    _fields_ = [("type", C.c_int32), ("col", C.c_int32)]


class GroupByCfg(C.Structure):
    _fields_ = [("block_threads", C.c_int32), ("smem_slots", C.c_int32),
                ("global_slots_log2", C.c_int32), ("ctas_per_sm", C.c_int32),
                ("max_groups", C.c_int64), ("tile_rows", C.c_int32), ("nstages", C.c_int32)]


class JoinCfg(C.Structure):
    _fields_ = [("load_factor", C.c_float), ("l2_persist", C.c_int32),
                ("block_threads", C.c_int32)]


class SortCfg(C.Structure):
    _fields_ = [("digit_bits", C.c_int32), ("block_threads", C.c_int32),
                ("items_per_thread", C.c_int32)]


class GroupByInstance(C.Structure):
    _fields_ = [("cols", C.c_void_p), ("pred", C.c_void_p), ("out", C.c_void_p),
                ("out_capacity", C.c_int64), ("max_groups", C.c_int64)]


OP_FILTER, OP_GROUPBY, OP_JOIN_PROBE, OP_SORT = 0, 1, 2, 3
MAX_RESULT_COLS = 16


class ServerCfg(C.Structure):
    _fields_ = [("slots", C.c_int32), ("reserved", C.c_int32), ("hbm_budget", C.c_int64)]


class Request(C.Structure):
    _fields_ = [("op", C.c_int32), ("ncols", C.c_int32), ("cols", C.c_void_p),
                ("pred", C.c_void_p), ("idx", C.c_void_p), ("nidx", C.c_int32),
                ("naggs", C.c_int32), ("aggs", C.c_void_p), ("max_groups", C.c_int64),
                ("table", C.c_int32), ("join_type", C.c_int32), ("nkeys", C.c_int32),
                ("want_rowid", C.c_int32), ("orders", C.c_void_p), ("null_orders", C.c_void_p)]


class Result(C.Structure):
    _fields_ = [("status", C.c_int32), ("ncols", C.c_int32),
                ("cols", OutColumn * MAX_RESULT_COLS), ("rowid", C.c_void_p),
                ("rowid2", C.c_void_p), ("rows", C.c_int64), ("submit_ns", C.c_int64),
                ("admit_ns", C.c_int64), ("done_ns", C.c_int64), ("launched_ns", C.c_int64),
                ("slot", C.c_int32), ("reserved", C.c_int32)]


class GTables(C.Structure):
    """GHive's GTables with its fields read out (ghb_gtables)."""
    _fields_ = [("ntables", C.c_int32), ("ncols", C.c_void_p), ("types", C.c_void_p),
                ("row_cnt", C.c_void_p), ("key_cnt", C.c_void_p), ("vertex_name", C.c_void_p),
                ("nlong", C.c_int32), ("long_cols", C.c_void_p),
                ("ndouble", C.c_int32), ("double_cols", C.c_void_p),
                ("nint", C.c_int32), ("int_cols", C.c_void_p),
                ("nstring", C.c_int32), ("string_cols", C.c_void_p),
                ("string_idx_cols", C.c_void_p)]


class PlanOp(C.Structure):
    _fields_ = [("op", C.c_int32), ("join_type", C.c_int32), ("pred", C.c_void_p),
                ("idx", C.c_void_p), ("nidx", C.c_int32), ("naggs", C.c_int32),
                ("aggs", C.c_void_p), ("max_groups", C.c_int64), ("orders", C.c_void_p),
                ("null_orders", C.c_void_p), ("build_table", C.c_int32),
                ("nbuild_keep", C.c_int32), ("build_keep", C.c_void_p)]


class PlanResult(C.Structure):
    _fields_ = [("ncols", C.c_int32), ("types", C.c_int32 * MAX_RESULT_COLS),
                ("data", C.c_void_p * MAX_RESULT_COLS), ("is_null", C.c_void_p * MAX_RESULT_COLS),
                ("sequence", C.c_int32 * MAX_RESULT_COLS), ("rows", C.c_int64),
                ("n_long", C.c_int32), ("n_double", C.c_int32), ("n_int", C.c_int32),
                ("n_string", C.c_int32), ("str_bytes", C.c_void_p * MAX_RESULT_COLS),
                ("str_nbytes", C.c_int64 * MAX_RESULT_COLS)]


class BatchCfg(C.Structure):
    _fields_ = [("autotune", C.c_int32), ("block_threads", C.c_int32),
                ("smem_slots", C.c_int32), ("load_factor", C.c_float),
                ("use_graph", C.c_int32)]


def agg_out_type(agg_type, in_type):
    """Result type of an aggregate, as Hive's UDAFs produce it."""
    if agg_type == CNT:
        return LONG
    if agg_type == AVG:
        return DOUBLE
    if agg_type == SUM:
        return DOUBLE if in_type == DOUBLE else LONG
    return in_type


# ---------------------------------------------------------------- predicates
class Pred:
    """Builder for a GHive-style predicate tree.

    >>> p = Pred.leaf(FILTER_LT, col=3, a=1263)
    >>> q = Pred.and_(p, Pred.leaf(FILTER_NOT_NULL, col=0))
    """

    def __init__(self, mode, col=-1, col2=-1, a=0, b=0, children=()):
        self.mode, self.col, self.col2 = mode, col, col2
        self.a, self.b, self.children = a, b, tuple(children)

    @staticmethod
    def leaf(mode, col, a=0, b=0, col2=-1):
        return Pred(mode, col=col, col2=col2, a=a, b=b)

    @staticmethod
    def and_(x, y):
        return Pred(FILTER_AND, children=(x, y))

    @staticmethod
    def or_(x, y):
        return Pred(FILTER_OR, children=(x, y))

    def flatten(self):
        """Returns (nodes array, root index) in post-order."""
        nodes, strs = [], []

        def rec(p):
            kids = [rec(c) for c in p.children]
            nd = PredNode()
            nd.mode, nd.col, nd.col2 = p.mode, p.col, p.col2
            if isinstance(p.a, (str, bytes)) or isinstance(p.b, (str, bytes)):
                # literals of a STRING column: their bytes, kept alive here
                for j, v in enumerate((p.a, p.b)):
                    b = v.encode() if isinstance(v, str) else (v if isinstance(v, bytes) else b"")
                    buf = C.create_string_buffer(b, max(1, len(b)))
                    strs.append(buf)
                    nd.lit_s[j] = C.addressof(buf)
                    nd.lit_s_len[j] = len(b)
            else:
                is_d = isinstance(p.a, float) or isinstance(p.b, float)
                nd.lit_is_double = 1 if is_d else 0
                for j, v in enumerate((p.a, p.b)):
                    if is_d:
                        nd.lit_d[j] = float(v)
                    else:
                        nd.lit_i[j] = int(v)
            nd.child[0] = kids[0] if kids else -1
            nd.child[1] = kids[1] if len(kids) > 1 else -1
            nodes.append(nd)
            return len(nodes) - 1

        root = rec(self)
        if len(nodes) > MAX_PRED_NODES:
            raise ValueError("predicate tree has more than %d nodes" % MAX_PRED_NODES)
        arr = (PredNode * len(nodes))(*nodes)
        arr._strs = strs   # the string literals live as long as the nodes
        return arr, root

    def as_struct(self):
        arr, root = self.flatten()
        p = Predicate()
        p.n_nodes, p.root = len(arr), root
        p.nodes = C.cast(arr, C.POINTER(PredNode))
        p._keep = arr  # keep the node array alive with the struct
        return p
