"""CPU checks of the boundary: the library loads, exports every entry point
include/ghive_b200.h declares, and the ctypes mirror has the C layout."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from ghive_b200 import _lib, abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    declared = _lib.declared_symbols()
    assert len(declared) >= 17
    missing = [s for s in declared if not hasattr(L, s)]
    assert not missing, missing
    # and the ctypes prototypes cover them all
    assert set(declared) <= set(_lib._PROTOS), set(declared) - set(_lib._PROTOS)


def test_abi_version():
    assert _lib.lib().ghb_abi_version() == 1


def test_struct_layout_matches_header(tmp_path):
    src = tmp_path / "layout.c"
    src.write_text("""
#include <stdio.h>
#include <stddef.h>
#include "ghive_b200.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\\n", sizeof(ghb_column),
         sizeof(ghb_out_column), sizeof(ghb_pred_node), sizeof(ghb_predicate),
         sizeof(ghb_agg_desc), sizeof(ghb_groupby_cfg), sizeof(ghb_join_cfg),
         sizeof(ghb_sort_cfg), offsetof(ghb_pred_node, lit_d), sizeof(ghb_groupby_instance),
         sizeof(ghb_batch_cfg), offsetof(ghb_batch_cfg, load_factor), sizeof(ghb_gtables),
         sizeof(ghb_plan_op), sizeof(ghb_plan_result), offsetof(ghb_plan_result, rows),
         offsetof(ghb_plan_op, build_keep));
  return 0;
}
""")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True,
                                          check=True).stdout.split()]
    exp = [C.sizeof(abi.Column), C.sizeof(abi.OutColumn), C.sizeof(abi.PredNode),
           C.sizeof(abi.Predicate), C.sizeof(abi.AggDesc), C.sizeof(abi.GroupByCfg),
           C.sizeof(abi.JoinCfg), C.sizeof(abi.SortCfg), abi.PredNode.lit_d.offset,
           C.sizeof(abi.GroupByInstance), C.sizeof(abi.BatchCfg), abi.BatchCfg.load_factor.offset,
           C.sizeof(abi.GTables), C.sizeof(abi.PlanOp), C.sizeof(abi.PlanResult),
           abi.PlanResult.rows.offset, abi.PlanOp.build_keep.offset]
    assert got == exp


def test_key_mixer_is_the_same_bijection_in_numpy_and_torch():
    import numpy as np
    import torch

    from ghive_b200 import workloads
    x = np.concatenate([np.arange(0, 5000, dtype=np.int64),
                        np.array([-1, np.iinfo(np.int64).min, np.iinfo(np.int64).max])])
    a = workloads.mix64_np(x)
    b = workloads.mix64_torch(torch.from_numpy(x)).numpy()
    assert np.array_equal(a, b)
    assert len(np.unique(a)) == len(x)


def test_enum_values_are_ghives():
    # ColumnType (Column.hpp:5-11), PredicateMode (FilterPredicate.hpp:17-58),
    # AggregationType (AggregationDesc.hpp:6-25), BaseJoinType (BaseJoinPredicate.hpp:11-25)
    assert (abi.LONG, abi.DOUBLE, abi.INT, abi.STRING) == (0, 1, 2, 3)
    assert (abi.FILTER_EQ, abi.FILTER_LT, abi.FILTER_EQ_RANGE, abi.FILTER_NOT_NULL,
            abi.FILTER_AND, abi.FILTER_OR) == (0, 3, 6, 10, 11, 12)
    assert (abi.SUM, abi.MAX, abi.MIN, abi.AVG, abi.CNT) == (0, 1, 2, 3, 4)
    assert (abi.INNER_JOIN, abi.LEFT_OUTER_JOIN, abi.LEFT_SEMI_JOIN) == (0, 1, 4)


def test_predicate_flattens_post_order():
    p = abi.Pred.or_(abi.Pred.and_(abi.Pred.leaf(abi.FILTER_LT, 0, a=5),
                                   abi.Pred.leaf(abi.FILTER_GT, 1, a=2.5)),
                     abi.Pred.leaf(abi.FILTER_NOT_NULL, 2))
    nodes, root = p.flatten()
    assert root == len(nodes) - 1 == 4
    for i, nd in enumerate(nodes):
        if nd.mode in (abi.FILTER_AND, abi.FILTER_OR):
            assert nd.child[0] < i and nd.child[1] < i
    assert nodes[1].lit_is_double == 1 and nodes[1].lit_d[0] == 2.5
    assert nodes[0].lit_is_double == 0 and nodes[0].lit_i[0] == 5


def test_agg_output_types_follow_hive_udafs():
    assert abi.agg_out_type(abi.SUM, abi.INT) == abi.LONG
    assert abi.agg_out_type(abi.SUM, abi.DOUBLE) == abi.DOUBLE
    assert abi.agg_out_type(abi.AVG, abi.LONG) == abi.DOUBLE
    assert abi.agg_out_type(abi.MIN, abi.INT) == abi.INT
    assert abi.agg_out_type(abi.CNT, abi.DOUBLE) == abi.LONG


def test_context_without_a_gpu_reports_cuda_error():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = C.c_void_p()
    assert _lib.lib().ghb_ctx_create(0, 0, C.byref(h)) == abi.ERR_CUDA
    assert not h.value


def test_ops_layer_refuses_to_run_without_the_library(monkeypatch):
    monkeypatch.setattr(_lib, "_lib", None)
    monkeypatch.setattr(_lib, "LIB_PATH", "/nonexistent/libghive_b200.so")
    with pytest.raises(ImportError):
        _lib.lib()
