"""The per-call JSON log (ghb_ctx_set_log): one line per operator call with
its rows and input bytes; at level 2 the call's device time, GB/s and the
fraction of the given peak."""
import json

import numpy as np
import pytest

from ghive_b200 import abi, workloads

pytestmark = pytest.mark.gpu


def test_log_lines_per_call(tmp_path):
    import torch

    from ghive_b200.ops import Context
    ctx = Context(0)
    dev = torch.device("cuda", 0)
    cols = [torch.from_numpy(c).to(dev) for c in workloads.fact_table(1_000_000, seed_idx=70)]
    path = tmp_path / "calls.jsonl"
    try:
        ctx.set_log(path, level=2, peak_gbs=6650.0)
        ctx.filter(workloads.fact_predicate(), cols)
        ctx.filter_groupby(workloads.fact_predicate(), cols, [0], workloads.AGGS_FACT, capacity=1000,
                           max_groups=1000)
        ctx.sort([cols[3]], payload=[cols[0]])
        ctx.set_log(path, level=1)
        ctx.sort([cols[3]])
        ctx.set_log(None)
        ctx.sort([cols[3]])                       # not logged
    finally:
        ctx.close()
    lines = [json.loads(x) for x in path.read_text().splitlines()]
    assert [x["op"] for x in lines] == ["filter", "filter_groupby", "sort", "sort"]
    assert all(x["status"] == 0 and x["rows"] == 1_000_000 and x["device"] == 0 for x in lines)
    row_bytes = sum(c.element_size() for c in cols)
    assert lines[0]["bytes"] == lines[1]["bytes"] == 1_000_000 * row_bytes
    assert lines[2]["bytes"] == 1_000_000 * (cols[3].element_size() + cols[0].element_size())
    for x in lines[:3]:
        assert x["device_us"] > 0 and x["gbs"] > 0
        assert x["roofline_frac"] == pytest.approx(x["gbs"] / 6650.0, rel=1e-3)
    assert "device_us" not in lines[3] and lines[3]["host_us"] > 0


def test_log_from_the_environment(tmp_path, monkeypatch):
    from ghive_b200.ops import Context
    path = tmp_path / "env.jsonl"
    monkeypatch.setenv("GHB_LOG", str(path))
    monkeypatch.setenv("GHB_LOG_LEVEL", "1")
    ctx = Context(0)
    try:
        a = np.arange(100_000, dtype=np.int64)
        ctx.sort_host([a[::-1].copy()])
    finally:
        ctx.close()
    lines = [json.loads(x) for x in path.read_text().splitlines()]
    assert lines and lines[-1]["op"] == "sort_host" and lines[-1]["rows"] == 100_000
