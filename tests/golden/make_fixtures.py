"""Generates the golden fixtures under tests/golden/ from the reference's tests.

Run in a checkout where the GHive reference tree is available (its root is
the one, required argument).  The script reads the test
sources AS TEXT and extracts their input values and expected outputs; it runs
none of the reference's code.  The JSON it writes is committed, so the test
suite never needs the reference tree.

Sources (paths inside the GHive project):
  hive-rel-release-3.1.0/ql/src/test/org/apache/hadoop/hive/ql/exec/vector/
      TestVectorGroupByOperator.java   SUM/MIN/MAX/AVG/COUNT known answers
  gpu_impl/test/GroupByPredicateTest.cu  shouldSuccess, multipleKeysTest,
      TwoColumndoubleSumTest, bigTableTestTable (absGroupByTest prints its
      result without an expected value, so it yields no fixture)
  gpu_impl/test/JoinPredicateTest.cu     SEMI_OUTER_TEST_TABLE result_offsets
  gpu_impl/test/FilterPredicateTest.cu   simpleOneColTest expected rows

Usage:  python tests/golden/make_fixtures.py <root of the GHive reference tree>
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
HIVE_TEST = ("hive-rel-release-3.1.0/ql/src/test/org/apache/hadoop/hive/ql/exec/vector/"
             "TestVectorGroupByOperator.java")
GHIVE_TEST = "gpu_impl/test"

I64_MIN, I64_MAX = -(1 << 63), (1 << 63) - 1


# ----------------------------------------------------------- Java parsing
def _balanced(s, start):
    """Index just past the parenthesis/brace group opening at s[start]."""
    pairs = {"(": ")", "{": "}", "[": "]"}
    stack = [pairs[s[start]]]
    i = start + 1
    in_str = False
    while stack:
        c = s[i]
        if in_str:
            if c == "\\":
                i += 1
            elif c == '"':
                in_str = False
        elif c == '"':
            in_str = True
        elif c in pairs:
            stack.append(pairs[c])
        elif c == stack[-1]:
            stack.pop()
        i += 1
    return i


def _split_top(s):
    parts, depth, cur, in_str = [], 0, [], False
    i = 0
    while i < len(s):
        c = s[i]
        if in_str:
            cur.append(c)
            if c == "\\":
                cur.append(s[i + 1])
                i += 1
            elif c == '"':
                in_str = False
        elif c == '"':
            in_str = True
            cur.append(c)
        elif c in "({[":
            depth += 1
            cur.append(c)
        elif c in ")}]":
            depth -= 1
            cur.append(c)
        elif c == "," and depth == 0:
            parts.append("".join(cur).strip())
            cur = []
        else:
            cur.append(c)
        i += 1
    if "".join(cur).strip():
        parts.append("".join(cur).strip())
    return parts


def _wrap64(v):
    if isinstance(v, int):
        v &= (1 << 64) - 1
        return v - (1 << 64) if v >= (1 << 63) else v
    return v


def java_expr(e):
    """Evaluates a Java numeric literal expression of the tests to Python."""
    e = e.strip()
    if e == "null":
        return None
    if e.startswith('"'):
        return json.loads(e)
    for name, val in (("Long.MAX_VALUE", str(I64_MAX)), ("Long.MIN_VALUE", "(%d)" % I64_MIN),
                      ("Integer.MAX_VALUE", "2147483647"), ("Integer.MIN_VALUE", "(-2147483648)")):
        e = e.replace(name, val)
    e = re.sub(r"\(long\)\s*", "", e)
    e = re.sub(r"(\d+)[Ll]\b", r"\1", e)
    e = re.sub(r"\b0+(\d)", r"\1", e)
    # (double) X  ->  float(X), X a number or a parenthesised group
    while "(double)" in e:
        i = e.index("(double)")
        j = i + len("(double)")
        while e[j] == " ":
            j += 1
        if e[j] == "(":
            k = _balanced(e, j)
        else:
            m = re.match(r"[-\w.]+", e[j:])
            k = j + m.end()
        e = e[:i] + "float(" + e[j:k] + ")" + e[k:]
    if not re.fullmatch(r"[\d\s+\-*/().a-z]*", e):
        raise ValueError("unsupported expression: %r" % e)
    return _wrap64(eval(e, {"__builtins__": {}}, {"float": float}))


def java_value(e):
    e = e.strip()
    m = re.match(r"Arrays\.asList\(\s*new\s+\w+\s*\[\s*\]\s*\{", e)
    if m:
        i = e.index("{")
        j = _balanced(e, i)
        return [java_value(x) for x in _split_top(e[i + 1:j - 1])]
    if e.startswith("buildHashMap("):
        args = _split_top(e[len("buildHashMap("):_balanced(e, len("buildHashMap")) - 1])
        vals = [java_value(a) for a in args]
        return [[vals[i], vals[i + 1]] for i in range(0, len(vals), 2)]
    return java_expr(e)


def java_batches(e):
    """Values of a FakeVectorRowBatch* source expression (Concat / Repeats / Iterables)."""
    e = e.strip()
    m = re.match(r"new\s+(FakeVectorRowBatchFrom\w+)\s*\(", e)
    kind = m.group(1)
    i = e.index("(", m.start(1))
    args = _split_top(e[i + 1:_balanced(e, i) - 1])
    if kind == "FakeVectorRowBatchFromConcat":
        out = []
        for a in args:
            out += java_batches(a)
        return out
    if kind == "FakeVectorRowBatchFromRepeats":
        vals = java_value(args[0].replace("new Long[]", "Arrays.asList(new Long[]") + ")")
        return vals * int(java_expr(args[1]))
    if kind == "FakeVectorRowBatchFromLongIterables":
        return java_value(args[1])
    raise ValueError(kind)


def hive_groupby_cases(src):
    cases = []
    methods = [(m.start(), m.group(1)) for m in re.finditer(r"public void (test\w+)\s*\(", src)]
    helpers = ("testAggregateLongAggregate", "testAggregateLongRepeats",
               "testAggregateLongKeyAggregate", "testAggregateDouble",
               "testAggregateDoubleStringKeyAggregate", "testAggregateStringKeyAggregate",
               "testAggregateCountStar", "testAggregateLongIterable")
    pat = re.compile(r"\b(%s)\s*\(" % "|".join(helpers))
    for m in pat.finditer(src):
        # skip the helper definitions themselves
        line_start = src.rfind("\n", 0, m.start()) + 1
        if "public void" in src[line_start:m.start()]:
            continue
        owner = [name for pos, name in methods if pos < m.start()][-1]
        i = src.index("(", m.start(1))
        args = _split_top(src[i + 1:_balanced(src, i) - 1])
        h = m.group(1)
        case = {"test": owner, "helper": h}
        if h != "testAggregateCountStar":
            if not args[0].startswith('"'):
                continue  # a call inside another helper, forwarding its arguments
            if java_expr(args[0]) not in ("sum", "min", "max", "avg", "count"):
                continue  # variance / std are outside GHive's AggregationType
        elif not re.match(r"\d", args[0]):
            continue
        if h == "testAggregateLongAggregate":
            case.update(agg=java_expr(args[0]), batch=java_expr(args[1]), value_type="long",
                        values=java_value(args[2]), expected=java_value(args[3]))
        elif h == "testAggregateDouble":
            case.update(agg=java_expr(args[0]), batch=java_expr(args[1]), value_type="double",
                        values=java_value(args[2]), expected=java_value(args[3]))
        elif h == "testAggregateLongRepeats":
            v = java_expr(args[1])
            # stored as one value plus a repeat count to keep the fixture small
            case.update(agg=java_expr(args[0]), batch=java_expr(args[3]), value_type="long",
                        values=[v], repeat=java_expr(args[2]), expected=java_value(args[4]))
        elif h == "testAggregateLongIterable":
            case.update(agg=java_expr(args[0]), batch=None, value_type="long",
                        values=java_batches(args[1]), expected=java_value(args[2]))
        elif h == "testAggregateCountStar":
            case.update(agg="count(*)", batch=java_expr(args[0]), value_type="long",
                        values=java_value(args[1]), expected=java_value(args[2]))
        elif h in ("testAggregateLongKeyAggregate", "testAggregateStringKeyAggregate",
                   "testAggregateDoubleStringKeyAggregate"):
            key_type = "long" if h == "testAggregateLongKeyAggregate" else "string"
            value_type = "double" if h == "testAggregateDoubleStringKeyAggregate" else "long"
            case.update(agg=java_expr(args[0]), batch=java_expr(args[1]), key_type=key_type,
                        value_type=value_type, keys=java_value(args[2]),
                        values=java_value(args[3]), expected=java_value(args[4]))
        if case.get("agg") not in ("sum", "min", "max", "avg", "count", "count(*)"):
            continue
        cases.append(case)
    return cases


# -------------------------------------------------------- GHive C++ tests
def _test_body(src, name):
    m = re.search(r"TEST_F\(\s*\w+\s*,\s*%s\s*\)\s*\{" % name, src)
    i = src.index("{", m.end() - 1)
    return src[i:_balanced(src, i)]


def _c_num(s):
    s = s.strip()
    return float(s) if re.search(r"[.eE]", s) else int(s)


def _indexed(body, var):
    vals = {}
    for m in re.finditer(r"\b%s\[(\d+)\]\s*=\s*([-+\d.eE]+)\s*;" % var, body):
        vals[int(m.group(1))] = _c_num(m.group(2))
    return [vals[i] for i in range(len(vals))]


def _brace_array(body, var):
    m = re.search(r"\b%s\s*(?:\[\d*\])?\s*(?:=\s*new\s+\w+\s*\[\d+\]\s*)?=?\s*\{([^}]*)\}" % var, body)
    return [_c_num(x) for x in m.group(1).split(",") if x.strip()]


def _cxx_string_literal(body, var):
    m = re.search(r"std::string\s+%s\s*=\s*((?:\"(?:[^\"\\]|\\.)*\"\s*)+);" % var, body)
    return "".join(json.loads(x) for x in re.findall(r"\"(?:[^\"\\]|\\.)*\"", m.group(1)))


def _parse_table_text(text):
    rows = []
    for m in re.finditer(r"row\[\d+\]: \[(.*)\]", text):
        rows.append([x.strip() for x in m.group(1).split(",")])
    types = [int(x) for x in re.search(r"column types: ([\d; ]+)", text).group(1).split(";")]
    return types, rows


def _keys_aggs(body):
    keys = [int(x) for x in re.search(r"vector<uint32_t>\s*\w+\s*=\s*\{([^}]*)\}", body)
            .group(1).split(",")]
    aggs = [[t, int(c)] for t, c in re.findall(r"\{\s*(SUM|MAX|MIN|AVG|CNT)\s*,\s*(\d+)\s*\}", body)]
    return keys, aggs


def ghive_groupby_cases(src):
    out = []
    # shouldSuccess: LONG, DOUBLE, INT, STRING(1 char per row)
    b = _test_body(src, "shouldSuccess")
    chars = re.search(r'strcpy\(strCol,\s*"([^"]*)"\)', b).group(1)
    keys, aggs = _keys_aggs(b)
    exp_t, exp = _parse_table_text(_cxx_string_literal(b, "result"))
    out.append({"test": "shouldSuccess",
                "columns": [["long", _indexed(b, "longCol")], ["double", _indexed(b, "doubleCol")],
                            ["int", _indexed(b, "intCol")],
                            ["string", chars, [int(x) for x in re.search(
                                r"strIdxCol = new int\[\d+\]\s*\{([^}]*)\}", b).group(1).split(",")]]],
                "keys": keys, "aggs": aggs, "expected_types": exp_t, "expected_rows": exp})
    # multipleKeysTest: DOUBLE, INT, STRING from a vector<string>
    b = _test_body(src, "multipleKeysTest")
    strs = re.findall(r'"(MFGR#\d+)"', b.split("std::vector<std::string> all_str")[1].split("};")[0])
    idx, pos = [], 0
    for s_ in strs:
        idx += [pos, pos + len(s_)]
        pos += len(s_)
    keys, aggs = _keys_aggs(b)
    exp_t, exp = _parse_table_text(_cxx_string_literal(b, "result"))
    out.append({"test": "multipleKeysTest",
                "columns": [["double", _indexed(b, "doubleCol")], ["int", _indexed(b, "intCol")],
                            ["string", "".join(strs), idx]],
                "keys": keys, "aggs": aggs, "expected_types": exp_t, "expected_rows": exp})
    # TwoColumndoubleSumTest: DOUBLE, LONG
    b = _test_body(src, "TwoColumndoubleSumTest")
    keys, aggs = _keys_aggs(b)
    exp_t, exp = _parse_table_text(_cxx_string_literal(b, "result"))
    out.append({"test": "TwoColumndoubleSumTest",
                "columns": [["double", _indexed(b, "doubleCol")], ["long", _indexed(b, "longCol")]],
                "keys": keys, "aggs": aggs, "expected_types": exp_t, "expected_rows": exp})
    # bigTableTestTable: INT key, DOUBLE value, 2550 rows
    b = _test_body(src, "bigTableTestTable")
    keys, aggs = _keys_aggs(b)
    exp_t, exp = _parse_table_text(_cxx_string_literal(b, "res"))
    out.append({"test": "bigTableTestTable",
                "columns": [["int", _indexed(b, "key")], ["double", _indexed(b, "value")]],
                "keys": keys, "aggs": aggs, "expected_types": exp_t, "expected_rows": exp})
    return out


def ghive_join_cases(src):
    b = _test_body(src, "SEMI_OUTER_TEST_TABLE")
    cols = [_brace_array(b, "long_col_%d" % i) for i in range(1, 5)]
    jt = re.findall(r"\{\s*(LEFT_SEMI_JOIN|LEFT_OUTER_JOIN|INNER_JOIN)\s*,\s*\{\s*(\d+)\s*,\s*(\d+)\s*\}\s*\}", b)
    exp = _brace_array(b, "expect_result_bitmap")
    return [{"test": "SEMI_OUTER_TEST_TABLE", "tables": cols,
             "join_types": [[t, int(a), int(c)] for t, a, c in jt], "expected_offsets": exp}]


def ghive_filter_cases(src):
    b = _test_body(src, "simpleOneColTest")
    exp_t, exp = _parse_table_text(_cxx_string_literal(b, "result_1"))
    mode = re.search(r"predicate->mode\s*=\s*(FILTER_\w+)", b).group(1)
    col = int(re.search(r"predicate->filterCol\[0\]\s*=\s*(\d+)", b).group(1))
    lit = _c_num(re.search(r"predicate->doubleFilterParams\[0\]\s*=\s*([-\d.]+)", b).group(1))
    return [{"test": "simpleOneColTest",
             "columns": [["long", _indexed(b, "longCol")], ["double", _indexed(b, "doubleCol")],
                         ["int", _indexed(b, "intCol")]],
             "mode": mode, "col": col, "literal": lit, "literal_type": "double",
             "expected_types": exp_t, "expected_rows": exp}]


def main(ref):
    with open(os.path.join(ref, HIVE_TEST)) as f:
        hive = hive_groupby_cases(f.read())
    with open(os.path.join(ref, GHIVE_TEST, "GroupByPredicateTest.cu")) as f:
        gb = ghive_groupby_cases(f.read())
    with open(os.path.join(ref, GHIVE_TEST, "JoinPredicateTest.cu")) as f:
        jn = ghive_join_cases(f.read())
    with open(os.path.join(ref, GHIVE_TEST, "FilterPredicateTest.cu")) as f:
        fl = ghive_filter_cases(f.read())
    outs = {"hive_groupby.json": {"source": HIVE_TEST, "cases": hive},
            "ghive_groupby.json": {"source": GHIVE_TEST + "/GroupByPredicateTest.cu", "cases": gb},
            "ghive_join.json": {"source": GHIVE_TEST + "/JoinPredicateTest.cu", "cases": jn},
            "ghive_filter.json": {"source": GHIVE_TEST + "/FilterPredicateTest.cu", "cases": fl}}
    for name, obj in outs.items():
        with open(os.path.join(HERE, name), "w") as f:
            json.dump(obj, f, separators=(",", ":"), allow_nan=False)
            f.write("\n")
        print(name, len(obj["cases"]), "cases")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit("usage: python tests/golden/make_fixtures.py <root of the GHive reference tree>")
    main(sys.argv[1])
