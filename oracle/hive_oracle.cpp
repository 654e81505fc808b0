// hive_oracle.cpp — CPU restatement of Hive's vectorized operators.
//
// TEST INFRASTRUCTURE.  This file is the parity oracle and the timed CPU
// baseline; it is not part of the product.  Only the test suite, the smoke
// check and bench.py (its cpu_baseline leg and `--impl reference` arm) load
// it, and only as the checker / the reference being timed.  The product
// library never links or calls it.
//
// What it restates (paths inside the GHive project, hive-rel-release-3.1.0/
// abbreviated hive/):
//   filter   hive/ql/src/gen/vectorization/ExpressionTemplates/
//            FilterColumnCompareScalar.txt:53-135 (compare with a scalar,
//            NULL rows dropped), FilterColumnBetween.txt:52-135 (BETWEEN /
//            NOT BETWEEN), FilterExprAndExpr / FilterExprOrExpr (AND runs the
//            children one after the other on selected[]; OR unions them),
//            driven per 1024-row batch as VectorFilterOperator.java:110-141.
//            GHive's extra modes (FilterPredicate.hpp:283-346: RANGE a<x<b,
//            NOT_EQ_RANGE x<=a||x>=b) keep GHive's definitions.
//   group-by hive/.../exec/vector/VectorGroupByOperator.java:388-502 (hash
//            mode: one aggregation-buffer row per distinct key tuple, NULL
//            keys form their own group), UDAFs VectorUDAFSum.txt:59-71
//            (sequential += in row order; all-NULL -> NULL; long SUM wraps,
//            TestVectorGroupByOperator.java:1517-1533), VectorUDAFAvg.txt:
//            56-71,509 (double sum + long count, result sum/count),
//            VectorUDAFMinMax.txt:65-72, COUNT(*) / COUNT(col) as bigint.
//            A global aggregate (no keys) emits one row even on empty input.
//   join     hive/.../mapjoin/fast/VectorMapJoinFastLongHashTable.java:99-254
//            (power-of-two slot pairs (valueRef,key), HashCodeUtil.
//            calculateLongHashCode (common/.../HashCodeUtil.java:36-45),
//            triangular probing probeSlot += ++i, expand-and-rehash at the
//            load factor, read probe bounded by largestNumberOfSteps) with
//            VectorMapJoinFastLongHashMap.java:71-84 value lists; probe
//            semantics of VectorMapJoinInnerLongOperator.java:104-395 (inner),
//            LeftSemi (one row per matching probe row) and LeftOuter (a miss
//            emits the probe row with a NULL build side).
//   sort     hive/serde/.../binarysortable/BinarySortableSerDe.java:921-960
//            byte order (sign bit flipped for integers, IEEE total-order
//            transform for doubles, DESC inverts the bytes) with the null
//            markers of BinarySortableSerDe.java:195-220; stable, ties keep
//            input order (the Tez sorter itself is not in the reference).
//
// Multi-threaded variants (suffix _mt) are the CPU baseline: row ranges are
// split over T std::threads, each with private state, then merged, the way T
// Tez tasks plus a final merge would run.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <map>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../include/ghive_b200.h"

namespace {

constexpr int kBatch = 1024;  // VectorizedRowBatch.DEFAULT_SIZE

inline bool col_is_null(const ghb_column& c, int64_t i) {
  if (c.type == GHB_STRING) return ((const int32_t*)c.aux)[2 * i] < 0;   // GTable.java:240-257
  switch (c.null_mode) {
    case GHB_NULLS_BYTEMAP: return c.is_null && c.is_null[i] != 0;
    case GHB_NULLS_SENTINEL:
      switch (c.type) {
        case GHB_LONG: return ((const int64_t*)c.data)[i] == INT64_MAX;
        case GHB_DOUBLE: return std::isnan(((const double*)c.data)[i]);
        case GHB_INT: return ((const int32_t*)c.data)[i] == INT32_MAX;
        case GHB_STRING: return ((const int32_t*)c.aux)[2 * i] < 0;
      }
      return false;
    default: return false;
  }
}

inline int64_t col_i64(const ghb_column& c, int64_t i) {
  if (c.type == GHB_LONG) return ((const int64_t*)c.data)[i];
  if (c.type == GHB_INT) return ((const int32_t*)c.data)[i];
  return (int64_t)((const double*)c.data)[i];
}
inline double col_f64(const ghb_column& c, int64_t i) {
  if (c.type == GHB_DOUBLE) return ((const double*)c.data)[i];
  if (c.type == GHB_LONG) return (double)((const int64_t*)c.data)[i];
  return (double)((const int32_t*)c.data)[i];
}

// ---------------------------------------------------------------- filter
// A leaf compares in double when the column or the literal is double
// (FilterLongColLessDoubleScalar and friends), else in int64.
template <typename T>
inline bool cmp_mode(int mode, T x, T a, T b) {
  switch (mode) {
    case GHB_FILTER_EQ: return x == a;
    case GHB_FILTER_LE: return x <= a;
    case GHB_FILTER_GE: return x >= a;
    case GHB_FILTER_LT: return x < a;
    case GHB_FILTER_GT: return x > a;
    case GHB_FILTER_RANGE: return x > a && x < b;
    case GHB_FILTER_EQ_RANGE: return a <= x && x <= b;
    case GHB_FILTER_NOT_EQ: return x != a;
    case GHB_FILTER_NOT_RANGE: return x < a || x > b;
    case GHB_FILTER_NOT_EQ_RANGE: return x <= a || x >= b;
  }
  return false;
}

// Hive's StringExpr.compare (storage-api/src/java/org/apache/hadoop/hive/ql/
// exec/vector/expressions/StringExpr.java:37-47): unsigned bytes, then length.
inline int string_compare(const uint8_t* a, int la, const uint8_t* b, int lb) {
  for (int i = 0; i < la && i < lb; i++)
    if (a[i] != b[i]) return (int)a[i] - (int)b[i];
  return la - lb;
}

inline const uint8_t* string_at(const ghb_column& c, int64_t i, int* len) {
  const int32_t* idx = (const int32_t*)c.aux;
  *len = idx[2 * i + 1] - idx[2 * i];
  return (const uint8_t*)c.data + idx[2 * i];
}

// A STRING leaf: FilterStringGroupColumnCompareStringGroupScalarBase.txt /
// FilterStringColumnBetween.txt (ql/src/gen/vectorization/
// ExpressionTemplates), with a column compare for col2 >= 0.
bool string_leaf_pass(const ghb_pred_node& nd, const ghb_column* cols, int64_t i) {
  int lx = 0;
  const uint8_t* x = string_at(cols[nd.col], i, &lx);
  int ca, cb = 0;
  if (nd.col2 >= 0) {
    int ly = 0;
    const uint8_t* y = string_at(cols[nd.col2], i, &ly);
    ca = string_compare(x, lx, y, ly);
  } else {
    ca = string_compare(x, lx, (const uint8_t*)nd.lit_s[0], nd.lit_s_len[0]);
    cb = string_compare(x, lx, (const uint8_t*)nd.lit_s[1], nd.lit_s_len[1]);
  }
  switch (nd.mode) {
    case GHB_FILTER_EQ: return ca == 0;
    case GHB_FILTER_LE: return ca <= 0;
    case GHB_FILTER_GE: return ca >= 0;
    case GHB_FILTER_LT: return ca < 0;
    case GHB_FILTER_GT: return ca > 0;
    case GHB_FILTER_RANGE: return ca > 0 && cb < 0;
    case GHB_FILTER_EQ_RANGE: return ca >= 0 && cb <= 0;
    case GHB_FILTER_NOT_EQ: return ca != 0;
    case GHB_FILTER_NOT_RANGE: return ca < 0 || cb > 0;
    case GHB_FILTER_NOT_EQ_RANGE: return ca <= 0 || cb >= 0;
  }
  return false;
}

bool leaf_pass(const ghb_pred_node& nd, const ghb_column* cols, int64_t i) {
  const ghb_column& c = cols[nd.col];
  if (col_is_null(c, i)) return false;
  if (nd.mode == GHB_FILTER_NOT_NULL) return true;
  if (c.type == GHB_STRING) {
    if (nd.col2 >= 0 && col_is_null(cols[nd.col2], i)) return false;
    return string_leaf_pass(nd, cols, i);
  }
  if (nd.col2 >= 0) {
    const ghb_column& c2 = cols[nd.col2];
    if (col_is_null(c2, i)) return false;
    if (c.type == GHB_DOUBLE || c2.type == GHB_DOUBLE)
      return cmp_mode<double>(nd.mode, col_f64(c, i), col_f64(c2, i), 0.0);
    return cmp_mode<int64_t>(nd.mode, col_i64(c, i), col_i64(c2, i), 0);
  }
  if (c.type == GHB_DOUBLE || nd.lit_is_double) {
    double a = nd.lit_is_double ? nd.lit_d[0] : (double)nd.lit_i[0];
    double b = nd.lit_is_double ? nd.lit_d[1] : (double)nd.lit_i[1];
    return cmp_mode<double>(nd.mode, col_f64(c, i), a, b);
  }
  return cmp_mode<int64_t>(nd.mode, col_i64(c, i), nd.lit_i[0], nd.lit_i[1]);
}

// Rewrites sel[0..n) in place to the rows that pass `node`; returns the new
// size.  This is the selected[]-rewriting contract of Hive's filter
// expressions.
int eval_node(const ghb_predicate& p, int node, const ghb_column* cols,
              int64_t base, int* sel, int n) {
  const ghb_pred_node& nd = p.nodes[node];
  if (nd.mode == GHB_FILTER_AND) {
    n = eval_node(p, nd.child[0], cols, base, sel, n);
    if (n == 0) return 0;
    return eval_node(p, nd.child[1], cols, base, sel, n);
  }
  if (nd.mode == GHB_FILTER_OR) {
    // FilterExprOrExpr: the first child's survivors, then the second child
    // on the rows the first rejected; the union keeps the batch order.
    std::vector<int> a(sel, sel + n);
    int na = eval_node(p, nd.child[0], cols, base, a.data(), n);
    std::vector<int> rest;
    rest.reserve(n - na);
    int j = 0;
    for (int k = 0; k < n; k++) {
      if (j < na && a[j] == sel[k]) { j++; continue; }
      rest.push_back(sel[k]);
    }
    int nb = eval_node(p, nd.child[1], cols, base, rest.data(), (int)rest.size());
    int out = 0, ia = 0, ib = 0;
    while (ia < na || ib < nb) {
      if (ib >= nb || (ia < na && a[ia] < rest[ib])) sel[out++] = a[ia++];
      else sel[out++] = rest[ib++];
    }
    return out;
  }
  int out = 0;
  for (int k = 0; k < n; k++)
    if (leaf_pass(nd, cols, base + sel[k])) sel[out++] = sel[k];
  return out;
}

int64_t filter_range(const ghb_predicate* pred, const ghb_column* cols,
                     int64_t lo, int64_t hi, int64_t* sel_out) {
  int sel[kBatch];
  int64_t total = 0;
  for (int64_t b = lo; b < hi; b += kBatch) {
    int n = (int)std::min<int64_t>(kBatch, hi - b);
    for (int k = 0; k < n; k++) sel[k] = k;
    if (pred && pred->n_nodes > 0) n = eval_node(*pred, pred->root, cols, b, sel, n);
    for (int k = 0; k < n; k++) sel_out[total++] = b + sel[k];
  }
  return total;
}

// -------------------------------------------------------------- group-by
struct KeyPart {
  bool null;
  int64_t bits;      // integer value or double bit pattern
  std::string str;   // GHB_STRING keys
  bool operator==(const KeyPart& o) const {
    return null == o.null && (null || (bits == o.bits && str == o.str));
  }
};
struct Key {
  std::vector<KeyPart> parts;
  bool operator==(const Key& o) const { return parts == o.parts; }
};
struct KeyHash {
  size_t operator()(const Key& k) const {
    uint64_t h = 1469598103934665603ull;
    for (const auto& p : k.parts) {
      uint64_t v = p.null ? 0x9e3779b97f4a7c15ull : (uint64_t)p.bits;
      h = (h ^ v) * 1099511628211ull;
      if (!p.str.empty()) h ^= std::hash<std::string>()(p.str);
    }
    return (size_t)(h ^ (h >> 29));
  }
};

struct AggBuf {
  bool null = true;     // no non-NULL input seen
  int64_t cnt = 0;      // COUNT / AVG count
  int64_t isum = 0;     // SUM over integers (wraps)
  double dsum = 0.0;    // SUM/AVG over doubles, Hive order
  double ns = 0.0, nc = 0.0;  // Neumaier compensated sum (error report only)
  int64_t imm = 0;      // MIN/MAX integer
  double dmm = 0.0;     // MIN/MAX double
};

inline void neumaier(AggBuf& a, double x) {
  double t = a.ns + x;
  if (std::fabs(a.ns) >= std::fabs(x)) a.nc += (a.ns - t) + x;
  else a.nc += (x - t) + a.ns;
  a.ns = t;
}

inline void agg_update(AggBuf& a, const ghb_agg_desc& d, const ghb_column* cols,
                       int64_t i) {
  if (d.type == GHB_AGG_CNT && d.col < 0) { a.cnt++; a.null = false; return; }
  const ghb_column& c = cols[d.col];
  if (col_is_null(c, i)) return;
  switch (d.type) {
    case GHB_AGG_CNT: a.cnt++; a.null = false; break;
    case GHB_AGG_SUM:
      if (c.type == GHB_DOUBLE) {
        double v = col_f64(c, i);
        if (a.null) a.dsum = v; else a.dsum += v;
        neumaier(a, v);
      } else {
        int64_t v = col_i64(c, i);
        a.isum = (int64_t)((uint64_t)a.isum + (uint64_t)v);
      }
      a.null = false;
      break;
    case GHB_AGG_AVG: {
      double v = col_f64(c, i);
      if (a.null) { a.dsum = v; a.cnt = 1; } else { a.dsum += v; a.cnt++; }
      neumaier(a, v);
      a.null = false;
      break;
    }
    case GHB_AGG_MIN:
    case GHB_AGG_MAX: {
      bool mn = d.type == GHB_AGG_MIN;
      if (c.type == GHB_DOUBLE) {
        double v = col_f64(c, i);
        if (a.null || (mn ? v < a.dmm : v > a.dmm)) a.dmm = v;
      } else {
        int64_t v = col_i64(c, i);
        if (a.null || (mn ? v < a.imm : v > a.imm)) a.imm = v;
      }
      a.null = false;
      break;
    }
  }
}

inline void agg_merge(AggBuf& a, const AggBuf& b, const ghb_agg_desc& d,
                      const ghb_column* cols) {
  if (b.null) return;
  switch (d.type) {
    case GHB_AGG_CNT: a.cnt += b.cnt; break;
    case GHB_AGG_SUM:
      if (cols[d.col].type == GHB_DOUBLE) a.dsum = a.null ? b.dsum : a.dsum + b.dsum;
      else a.isum = (int64_t)((uint64_t)a.isum + (uint64_t)b.isum);
      break;
    case GHB_AGG_AVG:
      a.dsum = a.null ? b.dsum : a.dsum + b.dsum;
      a.cnt += b.cnt;
      break;
    case GHB_AGG_MIN:
    case GHB_AGG_MAX: {
      bool mn = d.type == GHB_AGG_MIN;
      if (cols[d.col].type == GHB_DOUBLE) {
        if (a.null || (mn ? b.dmm < a.dmm : b.dmm > a.dmm)) a.dmm = b.dmm;
      } else {
        if (a.null || (mn ? b.imm < a.imm : b.imm > a.imm)) a.imm = b.imm;
      }
      break;
    }
  }
  double t = a.ns + b.ns;
  a.nc += b.nc + ((std::fabs(a.ns) >= std::fabs(b.ns)) ? (a.ns - t) + b.ns : (b.ns - t) + a.ns);
  a.ns = t;
  a.null = false;
}

Key make_key(const ghb_column* cols, const int32_t* key_cols, int nkeys, int64_t i) {
  Key k;
  k.parts.resize(nkeys);
  for (int j = 0; j < nkeys; j++) {
    const ghb_column& c = cols[key_cols[j]];
    KeyPart& p = k.parts[j];
    p.null = col_is_null(c, i);
    p.bits = 0;
    if (p.null) continue;
    if (c.type == GHB_STRING) {
      const int32_t* idx = (const int32_t*)c.aux;
      p.str.assign((const char*)c.data + idx[2 * i], idx[2 * i + 1] - idx[2 * i]);
    } else if (c.type == GHB_DOUBLE) {
      double v = ((const double*)c.data)[i];
      std::memcpy(&p.bits, &v, 8);
    } else {
      p.bits = col_i64(c, i);
    }
  }
  return k;
}

using GroupMap = std::unordered_map<Key, std::vector<AggBuf>, KeyHash>;

void groupby_rows(GroupMap& m, std::vector<Key>& order, const ghb_column* cols,
                  const int64_t* rows, int64_t nrows, const int32_t* key_cols,
                  int nkeys, const ghb_agg_desc* aggs, int naggs) {
  for (int64_t r = 0; r < nrows; r++) {
    int64_t i = rows[r];
    Key k = make_key(cols, key_cols, nkeys, i);
    auto it = m.find(k);
    if (it == m.end()) {
      it = m.emplace(k, std::vector<AggBuf>(naggs)).first;
      order.push_back(k);
    }
    for (int a = 0; a < naggs; a++) agg_update(it->second[a], aggs[a], cols, i);
  }
}

// Key order used to emit groups deterministically: NULL first, then numeric
// (signed / IEEE total order) or byte order.
bool key_less(const Key& a, const Key& b, const ghb_column* cols, const int32_t* key_cols) {
  for (size_t j = 0; j < a.parts.size(); j++) {
    const KeyPart& x = a.parts[j];
    const KeyPart& y = b.parts[j];
    if (x.null != y.null) return x.null;
    if (x.null) continue;
    int t = cols[key_cols[j]].type;
    if (t == GHB_STRING) {
      if (x.str != y.str) return x.str < y.str;
    } else if (t == GHB_DOUBLE) {
      double dx, dy;
      std::memcpy(&dx, &x.bits, 8);
      std::memcpy(&dy, &y.bits, 8);
      if (dx != dy) return dx < dy;
    } else if (x.bits != y.bits) {
      return x.bits < y.bits;
    }
  }
  return false;
}

int agg_out_type(const ghb_agg_desc& d, const ghb_column* cols) {
  switch (d.type) {
    case GHB_AGG_CNT: return GHB_LONG;
    case GHB_AGG_AVG: return GHB_DOUBLE;
    case GHB_AGG_SUM: return cols[d.col].type == GHB_DOUBLE ? GHB_DOUBLE : GHB_LONG;
    default: return cols[d.col].type;
  }
}

void write_value(ghb_out_column& o, int64_t row, bool null, int64_t iv, double dv) {
  if (o.is_null) o.is_null[row] = null ? 1 : 0;
  switch (o.type) {
    case GHB_LONG: ((int64_t*)o.data)[row] = null ? INT64_MAX : iv; break;
    case GHB_INT: ((int32_t*)o.data)[row] = null ? INT32_MAX : (int32_t)iv; break;
    case GHB_DOUBLE: ((double*)o.data)[row] = null ? NAN : dv; break;
  }
}

int64_t emit_groups(GroupMap& m, std::vector<Key>& order, const ghb_column* cols,
                    const int32_t* key_cols, int nkeys, const ghb_agg_desc* aggs,
                    int naggs, ghb_out_column* out, int64_t cap, double* comp_out) {
  std::sort(order.begin(), order.end(), [&](const Key& a, const Key& b) {
    return key_less(a, b, cols, key_cols);
  });
  int64_t g = (int64_t)order.size();
  if (g > cap) return -g;
  for (int64_t r = 0; r < g; r++) {
    const Key& k = order[r];
    const std::vector<AggBuf>& bufs = m[k];
    for (int j = 0; j < nkeys; j++) {
      ghb_out_column& o = out[j];
      const KeyPart& p = k.parts[j];
      if (o.type == GHB_STRING) continue;  // string keys are reported through hive_groupby_string_key
      double dv;
      std::memcpy(&dv, &p.bits, 8);
      write_value(o, r, p.null, p.bits, dv);
    }
    for (int a = 0; a < naggs; a++) {
      const AggBuf& b = bufs[a];
      ghb_out_column& o = out[nkeys + a];
      const ghb_agg_desc& d = aggs[a];
      bool null = b.null;
      int64_t iv = 0;
      double dv = 0.0;
      switch (d.type) {
        case GHB_AGG_CNT: null = false; iv = b.cnt; break;
        case GHB_AGG_SUM: iv = b.isum; dv = b.dsum; break;
        case GHB_AGG_AVG: dv = null ? 0.0 : b.dsum / (double)b.cnt; break;
        default: iv = b.imm; dv = b.dmm; break;
      }
      write_value(o, r, null, iv, dv);
      if (comp_out) {
        double c = 0.0;
        if (!b.null && (d.type == GHB_AGG_SUM || d.type == GHB_AGG_AVG)) {
          c = b.ns + b.nc;
          if (d.type == GHB_AGG_AVG) c /= (double)b.cnt;
        }
        comp_out[(int64_t)a * cap + r] = c;
      }
    }
  }
  return g;
}

// ------------------------------------------------------------------ join
// HashCodeUtil.calculateLongHashCode (HashCodeUtil.java:36-45), Java >>> is
// a logical shift.
inline int64_t hive_long_hash(int64_t key) {
  uint64_t k = (uint64_t)key;
  k ^= (k >> 7) ^ (k >> 4);
  k ^= (k >> 20) ^ (k >> 12);
  return (int64_t)k;
}

struct FastLongHashMap {
  std::vector<int64_t> slot_pairs;  // (valueRef, key) pairs; valueRef 0 = empty
  std::vector<std::vector<int32_t>> values;  // valueRef-1 -> build rows
  int32_t bucket_count, mask, resize_threshold, keys_assigned = 0, largest_steps = 0;
  float load_factor;

  FastLongHashMap(int64_t initial, float lf) : load_factor(lf) {
    int32_t cap = 1;
    while (cap < initial) cap <<= 1;
    if (cap < 2) cap = 2;
    bucket_count = cap;
    mask = cap - 1;
    resize_threshold = (int32_t)(cap * lf);
    slot_pairs.assign((size_t)cap * 2, 0);
  }

  void expand() {
    int32_t nc = bucket_count * 2, nm = nc - 1, nlargest = 0;
    std::vector<int64_t> np((size_t)nc * 2, 0);
    for (int32_t s = 0; s < bucket_count; s++) {
      int64_t ref = slot_pairs[2 * s];
      if (!ref) continue;
      int64_t key = slot_pairs[2 * s + 1];
      int32_t ns = (int32_t)hive_long_hash(key) & nm;
      int64_t probe = ns;
      int32_t i = 0;
      while (np[2 * (size_t)ns] != 0) {
        probe += ++i;
        ns = (int32_t)(probe & nm);
      }
      if (nlargest < i) nlargest = i;
      np[2 * (size_t)ns] = ref;
      np[2 * (size_t)ns + 1] = key;
    }
    slot_pairs.swap(np);
    bucket_count = nc;
    mask = nm;
    largest_steps = nlargest;
    resize_threshold = (int32_t)(bucket_count * load_factor);
  }

  void add(int64_t key, int32_t row) {
    if (resize_threshold <= keys_assigned) expand();
    int32_t slot = (int32_t)hive_long_hash(key) & mask;
    int64_t probe = slot;
    int32_t i = 0;
    bool is_new;
    while (true) {
      int64_t ref = slot_pairs[2 * (size_t)slot];
      if (ref == 0) { is_new = true; break; }
      if (slot_pairs[2 * (size_t)slot + 1] == key) { is_new = false; break; }
      probe += ++i;
      slot = (int32_t)(probe & mask);
    }
    if (largest_steps < i) largest_steps = i;
    if (is_new) {
      values.push_back({row});
      slot_pairs[2 * (size_t)slot] = (int64_t)values.size();
      slot_pairs[2 * (size_t)slot + 1] = key;
      keys_assigned++;
    } else {
      values[slot_pairs[2 * (size_t)slot] - 1].push_back(row);
    }
  }

  // findReadSlot: the value list or nullptr.
  const std::vector<int32_t>* find(int64_t key) const {
    int32_t slot = (int32_t)hive_long_hash(key) & mask;
    int64_t probe = slot;
    int32_t i = 0;
    while (true) {
      int64_t ref = slot_pairs[2 * (size_t)slot];
      if (ref == 0) return nullptr;
      if (slot_pairs[2 * (size_t)slot + 1] == key) return &values[ref - 1];
      probe += ++i;
      if (i > largest_steps) return nullptr;
      slot = (int32_t)(probe & mask);
    }
  }
};

FastLongHashMap* build_map(const ghb_column* bk, float lf) {
  FastLongHashMap* m = new FastLongHashMap(std::max<int64_t>(bk->n / 2, 16), lf);
  for (int64_t i = 0; i < bk->n; i++) {
    if (col_is_null(*bk, i)) continue;
    m->add(col_i64(*bk, i), (int32_t)i);
  }
  return m;
}

// Appends (probe row, build row) pairs for probe rows [lo, hi).
void probe_range(const FastLongHashMap& m, const ghb_column* pk, int jt, int64_t lo,
                 int64_t hi, std::vector<int32_t>& pr, std::vector<int32_t>& br) {
  for (int64_t i = lo; i < hi; i++) {
    const std::vector<int32_t>* v = col_is_null(*pk, i) ? nullptr : m.find(col_i64(*pk, i));
    if (jt == GHB_INNER_JOIN) {
      if (v) for (int32_t b : *v) { pr.push_back((int32_t)i); br.push_back(b); }
    } else if (jt == GHB_LEFT_SEMI_JOIN) {
      if (v) { pr.push_back((int32_t)i); br.push_back(-1); }
    } else {  // LEFT OUTER
      if (v) for (int32_t b : *v) { pr.push_back((int32_t)i); br.push_back(b); }
      else { pr.push_back((int32_t)i); br.push_back(-1); }
    }
  }
}

void gather_value(const ghb_column& src, int64_t row, ghb_out_column& o, int64_t at) {
  bool null = row < 0 || col_is_null(src, row);
  write_value(o, at, null, null ? 0 : col_i64(src, row), null ? 0.0 : col_f64(src, row));
}

// ------------------------------------------------------------------ sort
// BinarySortable order of one key value as an unsigned 64-bit word; NULLs
// are ordered by the marker byte handled in row_less.
inline uint64_t sortable_bits(const ghb_column& c, int64_t i) {
  if (c.type == GHB_DOUBLE) {
    double d = ((const double*)c.data)[i];
    uint64_t v;
    std::memcpy(&v, &d, 8);
    return (v & (1ull << 63)) ? ~v : (v ^ (1ull << 63));
  }
  return (uint64_t)col_i64(c, i) ^ (1ull << 63);
}

struct SortSpec {
  const ghb_column* keys;
  const int32_t* orders;
  const int32_t* null_orders;
  int nkeys;
  bool less(int64_t a, int64_t b) const {
    for (int j = 0; j < nkeys; j++) {
      const ghb_column& c = keys[j];
      bool desc = orders && orders[j] == GHB_DESC;
      int no = null_orders ? null_orders[j] : GHB_NULLS_DEFAULT;
      bool nulls_first = no == GHB_NULLS_FIRST || (no == GHB_NULLS_DEFAULT && !desc);
      bool na = col_is_null(c, a), nb = col_is_null(c, b);
      if (na || nb) {
        if (na && nb) continue;
        return na ? nulls_first : !nulls_first;
      }
      if (c.type == GHB_STRING) {
        const int32_t* idx = (const int32_t*)c.aux;
        const char* s = (const char*)c.data;
        std::string x(s + idx[2 * a], idx[2 * a + 1] - idx[2 * a]);
        std::string y(s + idx[2 * b], idx[2 * b + 1] - idx[2 * b]);
        if (x != y) return desc ? y < x : x < y;
        continue;
      }
      uint64_t x = sortable_bits(c, a), y = sortable_bits(c, b);
      if (x != y) return desc ? x > y : x < y;
    }
    return false;
  }
};

}  // namespace

extern "C" {

int32_t hive_oracle_version(void) { return 1; }

int64_t hive_long_hash_code(int64_t key) { return hive_long_hash(key); }

// Result column type of an aggregate (Hive's UDAF output types).
int32_t hive_agg_out_type(const ghb_agg_desc* d, const ghb_column* cols) {
  return agg_out_type(*d, cols);
}

// Selected row indices (ascending) of rows [0, n) passing `pred`.
int64_t hive_filter(const ghb_predicate* pred, const ghb_column* cols, int32_t ncols,
                    int64_t n, int64_t* sel_out) {
  (void)ncols;
  return filter_range(pred, cols, 0, n, sel_out);
}

// Group-by over the rows passing `pred` (NULL = all rows).  Groups are
// emitted in key order (NULL first).  Returns the group count, or -count when
// it exceeds cap.  comp_out (nullable, naggs*cap) receives the Neumaier
// compensated SUM / AVG per group.
int64_t hive_filter_groupby(const ghb_predicate* pred, const ghb_column* cols,
                            int32_t ncols, int64_t n, const int32_t* key_cols,
                            int32_t nkeys, const ghb_agg_desc* aggs, int32_t naggs,
                            ghb_out_column* out, int64_t cap, double* comp_out) {
  (void)ncols;
  std::vector<int64_t> sel(n > 0 ? n : 1);
  int64_t ns = filter_range(pred, cols, 0, n, sel.data());
  GroupMap m;
  std::vector<Key> order;
  groupby_rows(m, order, cols, sel.data(), ns, key_cols, nkeys, aggs, naggs);
  if (nkeys == 0 && order.empty()) {  // global aggregate over empty input
    order.push_back(Key{});
    m.emplace(Key{}, std::vector<AggBuf>(naggs));
  }
  return emit_groups(m, order, cols, key_cols, nkeys, aggs, naggs, out, cap, comp_out);
}

// Same as hive_filter_groupby with one STRING key column: the key of group r
// is written as [start,end) into key_idx_out[2r..2r+1] of the concatenated
// bytes in key_chars_out (capacity chars_cap).
int64_t hive_groupby_string_key(const ghb_column* cols, int32_t ncols, int64_t n,
                                const int32_t* key_cols, int32_t nkeys,
                                const ghb_agg_desc* aggs, int32_t naggs,
                                ghb_out_column* out, int64_t cap,
                                int32_t* key_idx_out, char* key_chars_out,
                                int64_t chars_cap) {
  (void)ncols;
  std::vector<int64_t> rows(n > 0 ? n : 1);
  for (int64_t i = 0; i < n; i++) rows[i] = i;
  GroupMap m;
  std::vector<Key> order;
  groupby_rows(m, order, cols, rows.data(), n, key_cols, nkeys, aggs, naggs);
  int64_t g = emit_groups(m, order, cols, key_cols, nkeys, aggs, naggs, out, cap, nullptr);
  if (g < 0) return g;
  int64_t pos = 0;
  for (int64_t r = 0; r < g; r++) {
    for (int j = 0; j < nkeys; j++) {
      if (cols[key_cols[j]].type != GHB_STRING) continue;
      const KeyPart& p = order[r].parts[j];
      if (p.null) { key_idx_out[2 * (r * nkeys + j)] = -1; key_idx_out[2 * (r * nkeys + j) + 1] = -1; continue; }
      if (pos + (int64_t)p.str.size() > chars_cap) return INT64_MIN;
      std::memcpy(key_chars_out + pos, p.str.data(), p.str.size());
      key_idx_out[2 * (r * nkeys + j)] = (int32_t)pos;
      pos += (int64_t)p.str.size();
      key_idx_out[2 * (r * nkeys + j) + 1] = (int32_t)pos;
    }
  }
  return g;
}

// Hash join restating Hive's fast long hash map.  Writes (probe row, build
// row) pairs in probe-row order; within one probe row, build rows in the
// order they were added.  Returns the pair count, or -count beyond cap.
int64_t hive_hash_join(const ghb_column* build_key, const ghb_column* probe_key,
                       int32_t join_type, float load_factor, int32_t* out_probe_rows,
                       int32_t* out_build_rows, int64_t cap) {
  FastLongHashMap* m = build_map(build_key, load_factor > 0 ? load_factor : 0.75f);
  std::vector<int32_t> pr, br;
  probe_range(*m, probe_key, join_type, 0, probe_key->n, pr, br);
  delete m;
  int64_t cnt = (int64_t)pr.size();
  if (cnt > cap) return -cnt;
  if (cnt) {
    std::memcpy(out_probe_rows, pr.data(), cnt * 4);
    std::memcpy(out_build_rows, br.data(), cnt * 4);
  }
  return cnt;
}

// Inspection of the restated Hive table (for the TestVectorMapJoinFastLongHashMap
// behaviours): builds from `keys`, then looks up `queries`; found[i] = number of
// values for queries[i] (0 if absent).  Returns the final bucket count.
int64_t hive_hashmap_lookup(const int64_t* keys, int64_t nkeys, float load_factor,
                            int64_t initial_capacity, const int64_t* queries,
                            int64_t nq, int64_t* found) {
  FastLongHashMap m(initial_capacity, load_factor);
  for (int64_t i = 0; i < nkeys; i++) m.add(keys[i], (int32_t)i);
  for (int64_t q = 0; q < nq; q++) {
    const std::vector<int32_t>* v = m.find(queries[q]);
    found[q] = v ? (int64_t)v->size() : 0;
  }
  return m.bucket_count;
}

// Stable ORDER BY permutation in BinarySortable order.
void hive_sort_perm(const ghb_column* keys, const int32_t* orders,
                    const int32_t* null_orders, int32_t nkeys, int64_t n,
                    int64_t* perm_out) {
  SortSpec s{keys, orders, null_orders, nkeys};
  for (int64_t i = 0; i < n; i++) perm_out[i] = i;
  std::stable_sort(perm_out, perm_out + n, [&](int64_t a, int64_t b) { return s.less(a, b); });
}

// ------------------------------------------------- CPU baseline (threads)
// Filter + group-by over T threads: each thread takes a contiguous row range
// in 1024-row batches with a private HashMap; partial maps merge at the end.
int64_t hive_filter_groupby_mt(int32_t threads, const ghb_predicate* pred,
                               const ghb_column* cols, int32_t ncols, int64_t n,
                               const int32_t* key_cols, int32_t nkeys,
                               const ghb_agg_desc* aggs, int32_t naggs,
                               ghb_out_column* out, int64_t cap) {
  (void)ncols;
  if (threads < 1) threads = 1;
  std::vector<GroupMap> maps(threads);
  std::vector<std::vector<Key>> orders(threads);
  std::vector<std::thread> ts;
  for (int t = 0; t < threads; t++) {
    ts.emplace_back([&, t] {
      int64_t lo = n * t / threads, hi = n * (t + 1) / threads;
      std::vector<int64_t> sel(kBatch);
      for (int64_t b = lo; b < hi; b += kBatch) {
        int64_t e = std::min<int64_t>(b + kBatch, hi);
        int64_t ns = filter_range(pred, cols, b, e, sel.data());
        groupby_rows(maps[t], orders[t], cols, sel.data(), ns, key_cols, nkeys, aggs, naggs);
      }
    });
  }
  for (auto& th : ts) th.join();
  GroupMap& m = maps[0];
  std::vector<Key>& order = orders[0];
  for (int t = 1; t < threads; t++) {
    for (const Key& k : orders[t]) {
      auto it = m.find(k);
      if (it == m.end()) {
        m.emplace(k, maps[t][k]);
        order.push_back(k);
      } else {
        for (int a = 0; a < naggs; a++) agg_merge(it->second[a], maps[t][k][a], aggs[a], cols);
      }
    }
  }
  if (nkeys == 0 && order.empty()) {
    order.push_back(Key{});
    m.emplace(Key{}, std::vector<AggBuf>(naggs));
  }
  return emit_groups(m, order, cols, key_cols, nkeys, aggs, naggs, out, cap, nullptr);
}

// Hash join over T threads: one build (as Hive builds one table per task),
// probe rows split in T ranges against the shared read-only table, payloads
// gathered into the output columns.  Output is in probe-row order.
int64_t hive_hash_join_mt(int32_t threads, const ghb_column* build_key,
                          const ghb_column* probe_key, int32_t join_type,
                          const ghb_column* build_payload, int32_t nbp,
                          ghb_out_column* out_build, int32_t* out_probe_rows,
                          int64_t cap) {
  if (threads < 1) threads = 1;
  FastLongHashMap* m = build_map(build_key, 0.75f);
  std::vector<std::vector<int32_t>> pr(threads), br(threads);
  std::vector<std::thread> ts;
  for (int t = 0; t < threads; t++) {
    ts.emplace_back([&, t] {
      int64_t lo = probe_key->n * t / threads, hi = probe_key->n * (t + 1) / threads;
      pr[t].reserve(hi - lo);
      br[t].reserve(hi - lo);
      probe_range(*m, probe_key, join_type, lo, hi, pr[t], br[t]);
    });
  }
  for (auto& th : ts) th.join();
  ts.clear();
  std::vector<int64_t> off(threads + 1, 0);
  for (int t = 0; t < threads; t++) off[t + 1] = off[t] + (int64_t)pr[t].size();
  int64_t total = off[threads];
  if (total > cap) { delete m; return -total; }
  for (int t = 0; t < threads; t++) {
    ts.emplace_back([&, t] {
      for (size_t r = 0; r < pr[t].size(); r++) {
        int64_t at = off[t] + (int64_t)r;
        if (out_probe_rows) out_probe_rows[at] = pr[t][r];
        for (int j = 0; j < nbp; j++) gather_value(build_payload[j], br[t][r], out_build[j], at);
      }
    });
  }
  for (auto& th : ts) th.join();
  delete m;
  return total;
}

// Stable sort over T threads: T chunks sorted with std::stable_sort, then
// pairwise stable merges (left chunk first on ties).
void hive_sort_perm_mt(int32_t threads, const ghb_column* keys, const int32_t* orders,
                       const int32_t* null_orders, int32_t nkeys, int64_t n,
                       int64_t* perm_out) {
  if (threads < 1) threads = 1;
  SortSpec s{keys, orders, null_orders, nkeys};
  auto cmp = [&](int64_t a, int64_t b) { return s.less(a, b); };
  for (int64_t i = 0; i < n; i++) perm_out[i] = i;
  std::vector<int64_t> bounds(threads + 1);
  for (int t = 0; t <= threads; t++) bounds[t] = n * t / threads;
  std::vector<std::thread> ts;
  for (int t = 0; t < threads; t++)
    ts.emplace_back([&, t] { std::stable_sort(perm_out + bounds[t], perm_out + bounds[t + 1], cmp); });
  for (auto& th : ts) th.join();
  std::vector<int64_t> tmp(n > 0 ? n : 1);
  for (int width = 1; width < threads; width *= 2) {
    ts.clear();
    for (int t = 0; t < threads; t += 2 * width) {
      int64_t lo = bounds[t], mid = bounds[std::min(t + width, threads)],
              hi = bounds[std::min(t + 2 * width, threads)];
      ts.emplace_back([&, lo, mid, hi] {
        std::merge(perm_out + lo, perm_out + mid, perm_out + mid, perm_out + hi, tmp.data() + lo, cmp);
        std::copy(tmp.data() + lo, tmp.data() + hi, perm_out + lo);
      });
    }
    for (auto& th : ts) th.join();
  }
}

}  // extern "C"
