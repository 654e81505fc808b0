"""Vectorised parity checks shared by the GPU tests (numpy, no Python loops
over rows, so they stay fast at the workloads' full sizes).

The bar: keys, counts, integer sums and MIN/MAX bit-exact; DOUBLE SUM/AVG
within REL_TOL relative of the oracle's Hive-order sequential sum.  Each
double result's relative error against the oracle's FP64 Neumaier
compensated sum is returned as well, so a test can state it.
"""
import numpy as np

from ghive_b200 import abi

REL_TOL = 1e-12


def host_cols(cols):
    """[(values, isnull)] of device tensors -> numpy pairs."""
    out = []
    for v, nl in cols:
        v = v.cpu().numpy() if hasattr(v, "cpu") else np.asarray(v)
        nl = nl.cpu().numpy() if hasattr(nl, "cpu") else np.asarray(nl)
        out.append((v, nl.astype(bool)))
    return out


def _order(keys):
    """Row order sorting groups by their keys (NULL first), keys as arrays."""
    if not keys:
        return np.arange(1)
    cols = []
    for v, nl in reversed(keys):
        cols.append(np.where(nl, 0, v.view(np.int64) if v.dtype == np.float64 else v))
        cols.append(~nl)
    return np.lexsort(cols)


def compare_groupby(got_keys, got_aggs, exp_keys, exp_aggs, out_types, comp=None):
    """Asserts parity of one group-by result; returns the relative errors of
    the double results against the compensated sums (empty without comp)."""
    n = len(exp_aggs[0][0]) if exp_aggs else len(exp_keys[0][0])
    assert (len(got_aggs[0][0]) if got_aggs else len(got_keys[0][0])) == n
    go, eo = _order(got_keys), _order(exp_keys)
    for (gv, gn), (ev, en) in zip(got_keys, exp_keys):
        assert np.array_equal(gn[go], en[eo])
        m = ~en[eo]
        assert np.array_equal(gv[go][m].view(np.uint8), ev[eo][m].view(np.uint8))
    errs = []
    for j, ((gv, gn), (ev, en), t) in enumerate(zip(got_aggs, exp_aggs, out_types)):
        gv, gn, ev, en = gv[go], gn[go], ev[eo], en[eo]
        assert np.array_equal(gn, en), j
        m = ~en
        if t == abi.DOUBLE:
            den = np.maximum(np.abs(ev[m]), 1e-300)
            rel = np.abs(gv[m] - ev[m]) / den
            assert rel.size == 0 or rel.max() <= REL_TOL, (j, float(rel.max()))
            if comp is not None and np.any(comp[j] != 0):
                c = comp[j][eo][m]
                errs.append(np.abs(gv[m] - c) / np.maximum(np.abs(c), 1e-300))
        else:
            assert np.array_equal(gv[m], ev[m]), (j, np.flatnonzero(gv[m] != ev[m])[:5])
    return np.concatenate(errs) if errs else np.zeros(0)


def error_summary(errs):
    if errs.size == 0:
        return {"results": 0}
    return {"results": int(errs.size), "max_rel": float(errs.max()),
            "median_rel": float(np.median(errs))}
