// ghive_ops.hpp — GHive's operator classes, kept as a C++ interface over the
// ghive_b200 C ABI (header only; link with -lghive_b200).
//
// A GHive plan calls its operators on host Tables of sentinel-NULL columns:
//   FilterPredicate::process(Table*)      gpu_impl/inc/Operator/FilterPredicate.hpp:60-117,
//                                         then FilterOperator::clean_data compacts the table
//                                         (gpu_impl/src/Operator/FilterOperator.cu:36-93)
//   GroupByPredicate::gpu_execute(Table*) gpu_impl/inc/Operator/GroupByPredicate.hpp:157-215
//   BaseJoinPredicate::process(tables)    gpu_impl/inc/Operator/BaseJoinPredicate.hpp:47-86
//   SinkOperator ORDER BY (key_offsets, "+-" sort_orders)
//                                         gpu_impl/src/Operator/SinkOperator.cu:98-306
// The classes below keep those names, fields and argument meanings and run on
// the library's host-buffer entry points (ghb_*_host): the columns go to the
// device, the operator runs there, the result comes back as a new Table.
// Differences, by design:
//   - inputs are never written: FilterPredicate::process replaces the
//     Table's columns with new compacted ones instead of rewriting the
//     caller's buffers (the reference compacted them in place);
//   - errors: functions returning a Table* return nullptr on failure, as the
//     reference does, and the reason is last_error() (per thread);
//   - joins are hash joins (left = probe side, right = build side): two
//     tables on one LONG or INT key run on the pipelined host join; N-way
//     chains, keys of several or STRING columns and semi joins run as one
//     device plan (ghb_run_plan) whose intermediates stay on the device.
// One device context per host thread is created on first use (device 0, or
// the one set_device() names first).
#pragma once

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <string>
#include <utility>
#include <vector>

#include "../../../include/ghive_b200.h"

namespace ghive_b200 {

// Column types with GHive's values (Column.hpp:5-11).
enum ColumnType : int { LONG = GHB_LONG, DOUBLE = GHB_DOUBLE, INT = GHB_INT, STRING = GHB_STRING, DEPEND = -1 };

// GHive's AggregationType (AggregationDesc.hpp:6-25) and AggregationDesc.
enum AggregationType : int { SUM = GHB_AGG_SUM, MAX = GHB_AGG_MAX, MIN = GHB_AGG_MIN, AVG = GHB_AGG_AVG, CNT = GHB_AGG_CNT };
struct AggregationDesc {
  AggregationType type;
  uint32_t index;   // input column; COUNT(*) when the column index is out of range
  AggregationDesc(AggregationType t, uint32_t i) : type(t), index(i) {}
};

// GHive's PredicateMode (FilterPredicate.hpp:17-58).
enum PredicateMode : int {
  EQ = GHB_FILTER_EQ, LE = GHB_FILTER_LE, GE = GHB_FILTER_GE, LT = GHB_FILTER_LT, GT = GHB_FILTER_GT,
  RANGE = GHB_FILTER_RANGE, EQ_RANGE = GHB_FILTER_EQ_RANGE, NOT_EQ = GHB_FILTER_NOT_EQ,
  NOT_RANGE = GHB_FILTER_NOT_RANGE, NOT_EQ_RANGE = GHB_FILTER_NOT_EQ_RANGE, NOT_NULL = GHB_FILTER_NOT_NULL,
  AND = GHB_FILTER_AND, OR = GHB_FILTER_OR
};

// GHive's BaseJoinType (BaseJoinPredicate.hpp:11-25), the kinds the device join runs.
enum BaseJoinType : int { INNER_JOIN = GHB_INNER_JOIN, LEFT_OUTER_JOIN = GHB_LEFT_OUTER_JOIN, LEFT_SEMI_JOIN = GHB_LEFT_SEMI_JOIN };

namespace detail {
struct State {
  ghb_ctx* ctx = nullptr;
  int device = 0;
  std::string error;
  ~State() {
    if (ctx) ghb_ctx_destroy(ctx);
  }
};
inline State& state() {
  static thread_local State s;
  return s;
}
inline ghb_ctx* ctx() {
  State& s = state();
  if (!s.ctx && ghb_ctx_create(s.device, 0, &s.ctx) != GHB_OK) {
    s.ctx = nullptr;
    s.error = "cannot create a device context";
  }
  return s.ctx;
}
inline bool fail(int32_t st) {
  if (st == GHB_OK) return false;
  State& s = state();
  s.error = s.ctx ? ghb_last_error(s.ctx) : "no device context";
  if (s.error.empty()) s.error = "status " + std::to_string(st);
  return true;
}
inline size_t width(ColumnType t) { return t == INT ? 4 : 8; }
}  // namespace detail

inline void set_device(int device) { detail::state().device = device; }
inline const std::string& last_error() { return detail::state().error; }

// A host column as GHive's Column (Column.hpp:13-35): values in data_ptr, NULLs
// as in-band sentinels (Table.hpp:29-52).  A column made with a row count owns
// its buffer; one made around a pointer does not.
struct Column {
  void* data_ptr = nullptr;
  void* data_ptr_aux = nullptr;
  ColumnType type = LONG;
  uint32_t row_num = 0;
  uint32_t char_size = 0;
  bool owned = false;

  Column(ColumnType t, uint32_t n) : type(t), row_num(n), owned(true) {
    data_ptr = std::calloc(n ? n : 1, detail::width(t));
  }
  Column(ColumnType t, uint32_t n, void* p) : data_ptr(p), type(t), row_num(n) {}
  // A STRING column around caller memory: char_size bytes of UTF-8 text in
  // chars and an int32 [start,end) pair per row in pairs (-1,-1: NULL).
  Column(ColumnType t, uint32_t n, void* chars, void* pairs, uint32_t csize)
      : data_ptr(chars), data_ptr_aux(pairs), type(t), row_num(n), char_size(csize) {}
  // A STRING column owning copies of its bytes and pairs.
  static Column* string_copy(uint32_t n, const void* chars, uint32_t nchars, const void* pairs) {
    Column* c = new Column(STRING, n, std::malloc(nchars ? nchars : 1), std::malloc(n ? 8 * (size_t)n : 8), nchars);
    c->owned = true;
    if (nchars) std::memcpy(c->data_ptr, chars, nchars);
    if (n) std::memcpy(c->data_ptr_aux, pairs, 8 * (size_t)n);
    return c;
  }
  Column(const Column&) = delete;
  Column& operator=(const Column&) = delete;
  ~Column() {
    if (owned) {
      std::free(data_ptr);
      std::free(data_ptr_aux);
    }
  }
  ghb_column desc() const {
    ghb_column c{};
    c.type = type;
    c.null_mode = GHB_NULLS_SENTINEL;
    c.data = data_ptr;
    c.aux = data_ptr_aux;
    c.n = row_num;
    return c;
  }
  template <class T>
  T* as() const { return (T*)data_ptr; }
};

// GHive's Table (Table.hpp:7-53): columns and a row count.  It deletes the
// columns it holds.
class Table {
 public:
  std::vector<Column*> columns;
  uint32_t row_num = 0;
  uint32_t key_num = 0;
  Table() = default;
  Table(const Table&) = delete;
  Table& operator=(const Table&) = delete;
  ~Table() {
    for (Column* c : columns) delete c;
  }
  uint32_t rowNum() const { return row_num; }
};

namespace detail {
// Output columns of the given types and capacity, and their descriptors.
struct Outs {
  std::vector<Column*> cols;
  std::vector<ghb_out_column> descs;
  Outs(const std::vector<ColumnType>& types, int64_t cap) {
    for (ColumnType t : types) {
      Column* c = new Column(t, (uint32_t)(cap > 0 ? cap : 1));
      cols.push_back(c);
      ghb_out_column o{};
      o.type = t;
      o.data = c->data_ptr;   // no NULL byte map: NULL results carry the sentinel
      descs.push_back(o);
    }
  }
  ~Outs() {
    for (Column* c : cols) delete c;
  }
  // Moves the first `rows` rows into a new Table.
  Table* take(int64_t rows) {
    Table* t = new Table();
    for (Column* c : cols) {
      c->row_num = (uint32_t)rows;
      t->columns.push_back(c);
    }
    cols.clear();
    t->row_num = (uint32_t)rows;
    return t;
  }
};

inline std::vector<ghb_column> descs(const Table* t) {
  std::vector<ghb_column> d;
  for (const Column* c : t->columns) d.push_back(c->desc());
  return d;
}
}  // namespace detail

// GHive's FilterPredicate: a leaf compares column filterCol[0] with one or
// two literals (or with column filterCol[1] when predColNum == 2), AND/OR
// nodes combine childrenPredicate[0..1].  dataType says how the literals are
// read: 0 long, 1 double, 2 int (Hive compares across numeric types).
class FilterPredicate {
 public:
  PredicateMode mode = EQ;
  int predColNum = 1;
  uint32_t filterCol[2] = {0, 0};
  uint8_t paramNum = 1;
  int64_t longFilterParams[2] = {0, 0};
  int32_t intFilterParams[2] = {0, 0};
  double doubleFilterParams[2] = {0, 0};
  uint8_t dataType = 0;
  FilterPredicate* childrenPredicate[2] = {nullptr, nullptr};

  // The predicate as the C ABI's node array (children before parents).
  int32_t flatten(std::vector<ghb_pred_node>* nodes) const {
    ghb_pred_node n{};
    n.mode = mode;
    n.col = -1;
    n.col2 = -1;
    if (mode == AND || mode == OR) {
      n.child[0] = childrenPredicate[0]->flatten(nodes);
      n.child[1] = childrenPredicate[1]->flatten(nodes);
    } else {
      n.col = (int32_t)filterCol[0];
      if (predColNum == 2) n.col2 = (int32_t)filterCol[1];
      n.lit_is_double = dataType == 1;
      for (int i = 0; i < 2; i++) {
        n.lit_d[i] = doubleFilterParams[i];
        n.lit_i[i] = dataType == 2 ? (int64_t)intFilterParams[i] : longFilterParams[i];
      }
    }
    nodes->push_back(n);
    return (int32_t)nodes->size() - 1;
  }

  // Keeps the rows of `table` that pass, in order: the Table gets new
  // compacted columns (the old ones are deleted; the caller's buffers they
  // pointed to are not written).  GHB_OK or the failing status.
  int32_t process(Table* table) const {
    ghb_ctx* c = detail::ctx();
    if (!c) return GHB_ERR_CUDA;
    std::vector<ghb_pred_node> nodes;
    const int32_t root = flatten(&nodes);
    ghb_predicate pred{(int32_t)nodes.size(), root, nodes.data()};
    std::vector<ghb_column> in = detail::descs(table);
    std::vector<int32_t> proj;
    std::vector<ColumnType> types;
    for (size_t j = 0; j < in.size(); j++) {
      proj.push_back((int32_t)j);
      types.push_back(table->columns[j]->type);
    }
    detail::Outs out(types, table->row_num);
    int64_t rows = 0;
    int32_t st = ghb_filter_host(c, &pred, in.data(), (int32_t)in.size(), proj.data(), (int32_t)proj.size(),
                                 out.descs.data(), table->row_num, &rows);
    if (detail::fail(st)) return st;
    Table* t = out.take(rows);
    for (Column* col : table->columns) delete col;
    table->columns = t->columns;
    table->row_num = t->row_num;
    t->columns.clear();
    delete t;
    return GHB_OK;
  }
};

// GHive's GroupByPredicate: GROUP BY `keys` (none or one column) computing
// `aggregation_descs`; the result holds the key column, then one column per
// aggregate, with Hive's result types (COUNT and SUM over integers: LONG,
// SUM and AVG over doubles: DOUBLE, MIN/MAX: the input type).
class GroupByPredicate {
 public:
  std::vector<uint32_t> keys;
  std::vector<AggregationDesc> aggregation_descs;
  GroupByPredicate() = default;
  GroupByPredicate(std::vector<uint32_t> k, std::vector<AggregationDesc> a)
      : keys(std::move(k)), aggregation_descs(std::move(a)) {}

  Table* gpu_execute(Table* input_tbl) const { return execute(input_tbl, nullptr); }

  // The same with a filter fused in front (FilterOperator -> GroupByOperator).
  Table* execute(Table* input_tbl, const FilterPredicate* filter) const {
    ghb_ctx* c = detail::ctx();
    if (!c) return nullptr;
    std::vector<ghb_column> in = detail::descs(input_tbl);
    std::vector<int32_t> kc(keys.begin(), keys.end());
    std::vector<ghb_agg_desc> ag;
    std::vector<ColumnType> types;
    for (uint32_t k : keys) types.push_back(input_tbl->columns[k]->type);
    for (const AggregationDesc& d : aggregation_descs) {
      const bool star = d.type == CNT && d.index >= in.size();
      ag.push_back(ghb_agg_desc{(int32_t)d.type, star ? -1 : (int32_t)d.index});
      const ColumnType it = star ? LONG : input_tbl->columns[d.index]->type;
      ColumnType ot = it;
      if (d.type == CNT) ot = LONG;
      else if (d.type == AVG) ot = DOUBLE;
      else if (d.type == SUM) ot = it == DOUBLE ? DOUBLE : LONG;
      types.push_back(ot);
    }
    std::vector<ghb_pred_node> nodes;
    ghb_predicate pred{0, 0, nullptr};
    if (filter) {
      const int32_t root = filter->flatten(&nodes);
      pred = ghb_predicate{(int32_t)nodes.size(), root, nodes.data()};
    }
    int64_t cap = keys.empty() ? 1 : std::max<int64_t>(1, std::min<int64_t>(input_tbl->row_num, 1 << 16));
    for (int attempt = 0; attempt < 2; attempt++) {
      detail::Outs out(types, cap);
      int64_t groups = 0;
      int32_t st = ghb_filter_groupby_host(c, filter ? &pred : nullptr, in.data(), (int32_t)in.size(), kc.data(),
                                           (int32_t)kc.size(), ag.data(), (int32_t)ag.size(), out.descs.data(),
                                           cap, &groups, nullptr);
      if (st == GHB_ERR_CAPACITY && groups > cap && attempt == 0) {
        cap = groups;   // more groups than the first guess: once more with room for all
        continue;
      }
      if (detail::fail(st)) return nullptr;
      Table* t = out.take(groups);
      t->key_num = (uint32_t)keys.size();
      return t;
    }
    return nullptr;
  }
};

// GHive's BaseJoinPredicate (BaseJoinPredicate.hpp:47-86) as a hash join.
// join_cols[i] are table i's key columns (the same count for every table),
// maintain_cols[i] the columns table i contributes to the result, join_types
// the chain's steps {type, {first, second}}: step 0 joins table 0 (the probe
// side) with its second table, each later step joins the tuples so far, by
// the key columns of the already joined table `first`, with table `second`
// (SortMergeJoinPredicate.cu:138-454).  A semi join's table contributes no
// columns.  The result holds the maintained columns of table 0, then of each
// further non-semi table in step order (table 0 keeps column 0 when it names
// none, BaseJoinPredicate.cu:13-19); result_offsets receives, per result row,
// the row of each of those tables (-1 where an outer join found no match).
// Result rows come in no particular order (the reference's in key order).
class HashJoinPredicate {
 public:
  std::vector<std::vector<uint32_t>> join_cols;
  std::vector<std::vector<uint32_t>> maintain_cols;
  std::vector<std::pair<BaseJoinType, std::pair<uint32_t, uint32_t>>> join_types;
  std::vector<int32_t> result_offsets;

  Table* process(const std::vector<Table*>& tables) {
    ghb_ctx* c = detail::ctx();
    if (!c) return nullptr;
    if (tables.size() != 2 || join_types.size() != 1 || join_types[0].second != std::make_pair(0u, 1u) ||
        join_types[0].first == LEFT_SEMI_JOIN || join_cols.size() != 2 || join_cols[0].size() != 1 ||
        join_cols[1].size() != 1 || join_cols[0][0] >= tables[0]->columns.size() ||
        join_cols[1][0] >= tables[1]->columns.size() || tables[0]->columns[join_cols[0][0]]->type == STRING ||
        tables[0]->columns[join_cols[0][0]]->type == DOUBLE)
      return chain(tables);
    const Table* left = tables[0];
    const Table* right = tables[1];
    const ghb_column lkey = left->columns[join_cols[0][0]]->desc();
    const ghb_column rkey = right->columns[join_cols[1][0]]->desc();
    std::vector<ghb_column> lpay, rpay;
    std::vector<ColumnType> ltypes, rtypes;
    if (maintain_cols.size() > 0)
      for (uint32_t j : maintain_cols[0]) {
        lpay.push_back(left->columns[j]->desc());
        ltypes.push_back(left->columns[j]->type);
      }
    if (maintain_cols.size() > 1)
      for (uint32_t j : maintain_cols[1]) {
        rpay.push_back(right->columns[j]->desc());
        rtypes.push_back(right->columns[j]->type);
      }
    int64_t cap = std::max<int64_t>(1, std::max(left->row_num, right->row_num));
    for (int attempt = 0; attempt < 2; attempt++) {
      detail::Outs lo(ltypes, cap), ro(rtypes, cap);
      std::vector<int32_t> lrow((size_t)cap), rrow((size_t)cap);
      int64_t rows = 0;
      int32_t st = ghb_hash_join_host(c, &rkey, &lkey, join_types[0].first, rpay.data(), (int32_t)rpay.size(),
                                      ro.descs.data(), lpay.data(), (int32_t)lpay.size(), lo.descs.data(),
                                      lrow.data(), rrow.data(), cap, &rows, nullptr);
      if (st == GHB_ERR_CAPACITY && rows > cap && attempt == 0) {
        cap = rows;
        continue;
      }
      if (detail::fail(st)) return nullptr;
      result_offsets.clear();
      result_offsets.reserve((size_t)rows * 2);
      for (int64_t i = 0; i < rows; i++) {
        result_offsets.push_back(lrow[(size_t)i]);
        result_offsets.push_back(rrow[(size_t)i]);
      }
      Table* t = lo.take(rows);
      Table* r = ro.take(rows);
      for (Column* col : r->columns) t->columns.push_back(col);
      r->columns.clear();
      delete r;
      return t;
    }
    return nullptr;
  }

 private:
  // The general chain as one device plan: a GTables of the columns each table
  // must bring (its maintained columns and the key columns of the steps that
  // read it), each table with its row ids appended as an INT column; one
  // JOIN_PROBE per step, the tuples so far as its probe side; a final
  // projection to the maintained columns and the row ids.
  Table* chain(const std::vector<Table*>& tables) {
    ghb_ctx* c = detail::ctx();
    detail::State& s = detail::state();
    auto bad = [&](const std::string& m) -> Table* {
      s.error = m;
      return nullptr;
    };
    const size_t nt = tables.size();
    if (nt < 2 || join_cols.size() != nt || join_types.empty())
      return bad("a join takes two or more tables, key columns for each and at least one step");
    for (size_t t = 0; t < nt; t++)
      for (uint32_t k : join_cols[t])
        if (k >= tables[t]->columns.size()) return bad("join key column out of range");
    // the tables in the result, in order, and each table's columns on the device
    std::vector<int> state(nt, 0);   // 1: joined, 2: semi-joined
    state[0] = 1;
    std::vector<size_t> result_tbl{0};
    std::vector<std::vector<uint32_t>> need(nt);
    auto add = [&](size_t t, uint32_t col) {
      if (std::find(need[t].begin(), need[t].end(), col) == need[t].end()) need[t].push_back(col);
    };
    for (const auto& step : join_types) {
      const uint32_t f = step.second.first, sc = step.second.second;
      if (f >= nt || sc >= nt || state[f] != 1 || state[sc] != 0)
        return bad("join step {" + std::to_string(f) + ", " + std::to_string(sc) +
                   "}: the first table must be joined already and the second not");
      if (join_cols[f].empty() || join_cols[f].size() != join_cols[sc].size())
        return bad("join step: both tables need the same number of key columns");
      if (step.first != INNER_JOIN && step.first != LEFT_OUTER_JOIN && step.first != LEFT_SEMI_JOIN)
        return bad("join type " + std::to_string((int)step.first) + " is not run on the device");
      for (uint32_t k : join_cols[f]) add(f, k);
      for (uint32_t k : join_cols[sc]) add(sc, k);
      state[sc] = step.first == LEFT_SEMI_JOIN ? 2 : 1;
      if (step.first != LEFT_SEMI_JOIN) result_tbl.push_back(sc);
    }
    std::vector<std::vector<uint32_t>> keep(nt);
    for (size_t i = 0; i < result_tbl.size(); i++) {
      const size_t t = result_tbl[i];
      keep[t] = t < maintain_cols.size() ? maintain_cols[t] : std::vector<uint32_t>{};
      if (keep[t].empty() && i == 0) keep[t].push_back(0);
      for (uint32_t col : keep[t]) {
        if (col >= tables[t]->columns.size()) return bad("maintained column out of range");
        add(t, col);
      }
    }
    // the GTables: table t's columns need[t] then its row ids
    std::vector<std::vector<int32_t>> types(nt), rowids(nt);
    std::vector<int32_t> ncols(nt), rows(nt), keys(nt, 0);
    std::vector<const char*> names(nt, "v");
    std::vector<const void*> bufs[4], idx_bufs;
    for (size_t t = 0; t < nt; t++) {
      for (uint32_t col : need[t]) {
        const Column* cl = tables[t]->columns[col];
        if (cl->type < LONG || cl->type > STRING) return bad("DEPEND columns cannot be joined");
        types[t].push_back((int32_t)cl->type);
        bufs[cl->type].push_back(cl->data_ptr);
        if (cl->type == STRING) idx_bufs.push_back(cl->data_ptr_aux);
      }
      rowids[t].resize(tables[t]->row_num);
      for (uint32_t r = 0; r < tables[t]->row_num; r++) rowids[t][r] = (int32_t)r;
      types[t].push_back(INT);
      bufs[INT].push_back(rowids[t].data());
      ncols[t] = (int32_t)types[t].size();
      rows[t] = (int32_t)tables[t]->row_num;
    }
    std::vector<const int32_t*> type_ptrs(nt);
    for (size_t t = 0; t < nt; t++) type_ptrs[t] = types[t].data();
    ghb_gtables g{};
    g.ntables = (int32_t)nt;
    g.ncols = ncols.data();
    g.types = type_ptrs.data();
    g.row_cnt = rows.data();
    g.key_cnt = keys.data();
    g.vertex_name = names.data();
    g.nlong = (int32_t)bufs[LONG].size();
    g.long_cols = bufs[LONG].data();
    g.ndouble = (int32_t)bufs[DOUBLE].size();
    g.double_cols = bufs[DOUBLE].data();
    g.nint = (int32_t)bufs[INT].size();
    g.int_cols = bufs[INT].data();
    g.nstring = (int32_t)bufs[STRING].size();
    g.string_cols = bufs[STRING].data();
    g.string_idx_cols = idx_bufs.data();
    // the plan: the tuples so far as (table, GTables column) pairs
    auto gcol = [&](size_t t, uint32_t col) {
      return (int32_t)(std::find(need[t].begin(), need[t].end(), col) - need[t].begin());
    };
    std::vector<std::pair<size_t, int32_t>> acc;
    for (int32_t j = 0; j < ncols[0]; j++) acc.push_back({0, j});
    auto pos = [&](size_t t, int32_t j) {
      return (int32_t)(std::find(acc.begin(), acc.end(), std::make_pair(t, j)) - acc.begin());
    };
    std::vector<std::vector<int32_t>> idx(join_types.size()), bkeep(join_types.size());
    std::vector<ghb_plan_op> ops;
    for (size_t i = 0; i < join_types.size(); i++) {
      const uint32_t f = join_types[i].second.first, sc = join_types[i].second.second;
      for (uint32_t k : join_cols[f]) idx[i].push_back(pos(f, gcol(f, k)));
      for (uint32_t k : join_cols[sc]) idx[i].push_back(gcol(sc, k));
      if (join_types[i].first != LEFT_SEMI_JOIN)
        for (int32_t j = 0; j < ncols[sc]; j++) {
          bkeep[i].push_back(j);
          acc.push_back({sc, j});
        }
      ghb_plan_op op{};
      op.op = GHB_OP_JOIN_PROBE;
      op.join_type = (int32_t)join_types[i].first;
      op.idx = idx[i].data();
      op.nidx = (int32_t)idx[i].size();
      op.build_table = (int32_t)sc;
      op.nbuild_keep = (int32_t)bkeep[i].size();
      op.build_keep = bkeep[i].data();
      ops.push_back(op);
    }
    std::vector<int32_t> proj;
    for (size_t t : result_tbl)
      for (uint32_t col : keep[t]) proj.push_back(pos(t, gcol(t, col)));
    for (size_t t : result_tbl) proj.push_back(pos(t, ncols[t] - 1));
    ghb_plan_op last{};
    last.op = GHB_OP_FILTER;
    last.idx = proj.data();
    last.nidx = (int32_t)proj.size();
    ops.push_back(last);
    ghb_plan_result res;
    if (detail::fail(ghb_run_plan(c, &g, 0, ops.data(), (int32_t)ops.size(), &res))) return nullptr;
    // the maintained columns (NULLs as sentinels), then the row ids
    const int64_t n = res.rows;
    Table* out = new Table();
    out->row_num = (uint32_t)n;
    const int nkeep = (int)proj.size() - (int)result_tbl.size();
    for (int j = 0; j < nkeep; j++) {
      const ColumnType t = (ColumnType)res.types[j];
      if (t == STRING) {
        out->columns.push_back(Column::string_copy((uint32_t)n, res.str_bytes[j], (uint32_t)res.str_nbytes[j],
                                                   res.data[j]));
        continue;
      }
      Column* col = new Column(t, (uint32_t)n);
      if (n) std::memcpy(col->data_ptr, res.data[j], (size_t)n * detail::width(t));
      out->columns.push_back(col);
    }
    result_offsets.assign((size_t)n * result_tbl.size(), -1);
    for (size_t i = 0; i < result_tbl.size(); i++) {
      const int32_t* ids = (const int32_t*)res.data[nkeep + i];
      const uint8_t* nul = res.is_null[nkeep + i];
      for (int64_t r = 0; r < n; r++)
        if (!(nul && nul[r])) result_offsets[(size_t)r * result_tbl.size() + i] = ids[r];
    }
    ghb_plan_result_free(&res);
    return out;
  }
};

// The ORDER BY of GHive's root SinkOperator: key columns key_offsets, one
// order character per key in sort_orders ('+' ascending, '-' descending;
// NULLs first ascending, last descending, Hive's defaults).  The result
// holds the key columns first, then the other columns (SinkOperator.cu:
// 98-306 reorders them the same way), sorted; equal keys keep input order.
class SinkSort {
 public:
  std::vector<uint32_t> key_offsets;
  std::string sort_orders;

  Table* execute(Table* tbl) const {
    ghb_ctx* c = detail::ctx();
    if (!c) return nullptr;
    if (sort_orders.size() != key_offsets.size()) {
      detail::state().error = "one sort order character per key";
      return nullptr;
    }
    std::vector<ghb_column> keys, pay;
    std::vector<ColumnType> ktypes, ptypes;
    std::vector<int32_t> orders;
    std::vector<bool> is_key(tbl->columns.size(), false);
    for (size_t i = 0; i < key_offsets.size(); i++) {
      const uint32_t k = key_offsets[i];
      keys.push_back(tbl->columns[k]->desc());
      ktypes.push_back(tbl->columns[k]->type);
      orders.push_back(sort_orders[i] == '-' ? GHB_DESC : GHB_ASC);
      is_key[k] = true;
    }
    for (size_t j = 0; j < tbl->columns.size(); j++)
      if (!is_key[j]) {
        pay.push_back(tbl->columns[j]->desc());
        ptypes.push_back(tbl->columns[j]->type);
      }
    detail::Outs ko(ktypes, tbl->row_num), po(ptypes, tbl->row_num);
    int32_t st = ghb_sort_host(c, keys.data(), orders.data(), nullptr, (int32_t)keys.size(), pay.data(),
                               (int32_t)pay.size(), ko.descs.data(), po.descs.data(), nullptr, nullptr);
    if (detail::fail(st)) return nullptr;
    Table* t = ko.take(tbl->row_num);
    Table* p = po.take(tbl->row_num);
    for (Column* col : p->columns) t->columns.push_back(col);
    p->columns.clear();
    delete p;
    t->key_num = (uint32_t)key_offsets.size();
    return t;
  }
};

}  // namespace ghive_b200
