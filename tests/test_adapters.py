"""The GHive-style C++ operator classes (ghive_b200/csrc/host/ghive_ops.hpp):
the header and its test program compile and link against the library (CPU),
and the program's checks pass on the GPU."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "adapters", "ghive_ops_test.cpp")
LIBDIR = os.path.join(ROOT, "ghive_b200", "lib")


def _build(tmp_path):
    exe = str(tmp_path / "ghive_ops_test")
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", SRC, "-o", exe, "-L" + LIBDIR, "-lghive_b200",
                    "-Wl,-rpath," + LIBDIR], check=True)
    return exe


def test_adapters_compile_and_link(tmp_path):
    assert os.path.exists(_build(tmp_path))


def _golden_chain_file(tmp_path):
    """GHive's N-way join case (tests/golden/ghive_join.json) in the test
    program's text form: tables, steps (type, first, second), expected offsets."""
    import json
    with open(os.path.join(ROOT, "tests", "golden", "ghive_join.json")) as f:
        case = json.load(f)["cases"][0]
    types = {"INNER_JOIN": 0, "LEFT_OUTER_JOIN": 1, "LEFT_SEMI_JOIN": 4}
    lines = [str(len(case["tables"]))]
    lines += ["%d %s" % (len(t), " ".join(map(str, t))) for t in case["tables"]]
    lines.append(str(len(case["join_types"])))
    lines += ["%d %d %d" % (types[n], a, b) for n, a, b in case["join_types"]]
    lines.append("%d %s" % (len(case["expected_offsets"]), " ".join(map(str, case["expected_offsets"]))))
    p = tmp_path / "golden_chain.txt"
    p.write_text("\n".join(lines) + "\n")
    return str(p)


@pytest.mark.gpu
def test_adapters_match_plain_loops_on_gpu(tmp_path):
    exe = _build(tmp_path)
    r = subprocess.run([exe, _golden_chain_file(tmp_path)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stdout + r.stderr
