// Drives the GHive-style operator classes (ghive_ops.hpp) on small host
// tables and checks each result against the same operator written as plain
// loops here, with Hive's rules (a NULL never passes a filter, aggregates
// skip NULLs, an outer join keeps unmatched left rows).  Prints "ok" and
// exits 0 when every check passes.
#include <cmath>
#include <cstdio>
#include <map>
#include <random>
#include <set>
#include <tuple>

#include "../../ghive_b200/csrc/host/ghive_ops.hpp"

using namespace ghive_b200;

static int failures = 0;
#define CHECK(c)                                                     \
  do {                                                               \
    if (!(c)) {                                                      \
      std::printf("FAILED %s:%d: %s (%s)\n", __FILE__, __LINE__, #c, \
                  last_error().c_str());                             \
      failures++;                                                    \
    }                                                                \
  } while (0)

static const int64_t kLongNull = INT64_MAX;
static const int32_t kIntNull = INT32_MAX;

static Table* make_fact(uint32_t n, uint32_t seed) {
  std::mt19937_64 g(seed);
  Table* t = new Table();
  Column* k = new Column(LONG, n);
  Column* x = new Column(DOUBLE, n);
  Column* d = new Column(INT, n);
  for (uint32_t i = 0; i < n; i++) {
    k->as<int64_t>()[i] = (g() % 50 == 0) ? kLongNull : (int64_t)(g() % 1000);
    x->as<double>()[i] = (double)(g() % 100000) / 100000.0;
    d->as<int32_t>()[i] = (g() % 40 == 0) ? kIntNull : (int32_t)(g() % 1000);
  }
  t->columns = {k, x, d};
  t->row_num = n;
  return t;
}

static void test_filter() {
  Table* t = make_fact(50000, 1);
  const int64_t* k = t->columns[0]->as<int64_t>();
  const double* x = t->columns[1]->as<double>();
  const int32_t* d = t->columns[2]->as<int32_t>();
  // (d < 500 AND k >= 100) OR x > 0.9
  std::vector<uint32_t> expect;
  for (uint32_t i = 0; i < t->row_num; i++) {
    bool a = d[i] != kIntNull && d[i] < 500 && k[i] != kLongNull && k[i] >= 100;
    if (a || x[i] > 0.9) expect.push_back(i);
  }
  std::vector<int64_t> ek;
  for (uint32_t i : expect) ek.push_back(k[i]);
  FilterPredicate lt, ge, gt, land, lor;
  lt.mode = LT; lt.filterCol[0] = 2; lt.dataType = 2; lt.intFilterParams[0] = 500;
  ge.mode = GE; ge.filterCol[0] = 0; ge.dataType = 0; ge.longFilterParams[0] = 100;
  gt.mode = GT; gt.filterCol[0] = 1; gt.dataType = 1; gt.doubleFilterParams[0] = 0.9;
  land.mode = AND; land.childrenPredicate[0] = &lt; land.childrenPredicate[1] = &ge;
  lor.mode = OR; lor.childrenPredicate[0] = &land; lor.childrenPredicate[1] = &gt;
  CHECK(lor.process(t) == GHB_OK);
  CHECK(t->row_num == expect.size());
  bool same = t->row_num == expect.size();
  for (uint32_t i = 0; same && i < t->row_num; i++) same = t->columns[0]->as<int64_t>()[i] == ek[i];
  CHECK(same);
  delete t;
}

static void test_groupby() {
  Table* t = make_fact(80000, 2);
  const int64_t* k = t->columns[0]->as<int64_t>();
  const double* x = t->columns[1]->as<double>();
  const int32_t* d = t->columns[2]->as<int32_t>();
  // GROUP BY d: COUNT(*), SUM(k), AVG(x), MIN(k), MAX(k)
  struct Acc { int64_t cnt = 0, sum = 0, nk = 0, mn = INT64_MAX, mx = INT64_MIN; double sx = 0; };
  std::map<int64_t, Acc> ref;   // key INT64_MIN stands for the NULL key
  for (uint32_t i = 0; i < t->row_num; i++) {
    Acc& a = ref[d[i] == kIntNull ? INT64_MIN : d[i]];
    a.cnt++;
    a.sx += x[i];
    if (k[i] != kLongNull) {
      a.sum += k[i];
      a.nk++;
      a.mn = std::min(a.mn, k[i]);
      a.mx = std::max(a.mx, k[i]);
    }
  }
  GroupByPredicate gb({2}, {AggregationDesc(CNT, 99), AggregationDesc(SUM, 0), AggregationDesc(AVG, 1),
                            AggregationDesc(MIN, 0), AggregationDesc(MAX, 0)});
  Table* r = gb.gpu_execute(t);
  CHECK(r != nullptr);
  if (r) {
    CHECK(r->row_num == ref.size());
    CHECK(r->columns.size() == 6);
    bool ok = r->row_num == ref.size();
    for (uint32_t i = 0; ok && i < r->row_num; i++) {
      const int32_t key = r->columns[0]->as<int32_t>()[i];
      auto it = ref.find(key == kIntNull ? INT64_MIN : key);
      if (it == ref.end()) { ok = false; break; }
      const Acc& a = it->second;
      ok = r->columns[1]->as<int64_t>()[i] == a.cnt;
      const int64_t sum = r->columns[2]->as<int64_t>()[i];
      ok = ok && (a.nk ? sum == a.sum : sum == kLongNull);
      const double avg = r->columns[3]->as<double>()[i];
      ok = ok && std::fabs(avg - a.sx / a.cnt) <= 1e-12 * std::fabs(a.sx / a.cnt);
      ok = ok && r->columns[4]->as<int64_t>()[i] == (a.nk ? a.mn : kLongNull);
      ok = ok && r->columns[5]->as<int64_t>()[i] == (a.nk ? a.mx : kLongNull);
    }
    CHECK(ok);
    delete r;
  }
  delete t;
}

static void test_join() {
  std::mt19937_64 g(3);
  const uint32_t nl = 20000, nr = 1000;
  Table* left = new Table();
  Column* lk = new Column(LONG, nl);
  Column* lv = new Column(INT, nl);
  for (uint32_t i = 0; i < nl; i++) {
    lk->as<int64_t>()[i] = (g() % 30 == 0) ? kLongNull : (int64_t)(g() % 1200);
    lv->as<int32_t>()[i] = (int32_t)i;
  }
  left->columns = {lk, lv};
  left->row_num = nl;
  Table* right = new Table();
  Column* rk = new Column(LONG, nr);
  Column* rv = new Column(LONG, nr);
  for (uint32_t i = 0; i < nr; i++) {
    rk->as<int64_t>()[i] = (int64_t)i;
    rv->as<int64_t>()[i] = (int64_t)(i * 7 + 3);
  }
  right->columns = {rk, rv};
  right->row_num = nr;
  for (BaseJoinType jt : {INNER_JOIN, LEFT_OUTER_JOIN}) {
    std::multiset<std::tuple<int32_t, int64_t>> expect;
    for (uint32_t i = 0; i < nl; i++) {
      const int64_t key = lk->as<int64_t>()[i];
      const bool hit = key != kLongNull && key < (int64_t)nr;
      if (hit) expect.insert(std::make_tuple((int32_t)i, rv->as<int64_t>()[key]));
      else if (jt == LEFT_OUTER_JOIN) expect.insert(std::make_tuple((int32_t)i, kLongNull));
    }
    HashJoinPredicate j;
    j.join_cols = {{0}, {0}};
    j.maintain_cols = {{1}, {1}};
    j.join_types = {{jt, {0u, 1u}}};
    Table* r = j.process({left, right});
    CHECK(r != nullptr);
    if (!r) continue;
    std::multiset<std::tuple<int32_t, int64_t>> got;
    for (uint32_t i = 0; i < r->row_num; i++)
      got.insert(std::make_tuple(r->columns[0]->as<int32_t>()[i], r->columns[1]->as<int64_t>()[i]));
    CHECK(got == expect);
    CHECK(j.result_offsets.size() == 2 * (size_t)r->row_num);
    bool offs = true;
    for (uint32_t i = 0; offs && i < r->row_num; i++)
      offs = j.result_offsets[2 * i] == r->columns[0]->as<int32_t>()[i];
    CHECK(offs);
    delete r;
  }
  HashJoinPredicate three;
  three.join_cols = {{0}, {0}, {0}};
  three.join_types = {{INNER_JOIN, {0u, 1u}}, {INNER_JOIN, {0u, 2u}}};
  CHECK(three.process({left, right, right}) == nullptr && !last_error().empty());
  delete left;
  delete right;
}

static void test_sort() {
  Table* t = make_fact(60000, 4);
  Column* rowid = new Column(INT, t->row_num);
  for (uint32_t i = 0; i < t->row_num; i++) rowid->as<int32_t>()[i] = (int32_t)i;
  t->columns.push_back(rowid);
  const int32_t* d = t->columns[2]->as<int32_t>();
  const int64_t* k = t->columns[0]->as<int64_t>();
  SinkSort s;
  s.key_offsets = {2, 0};
  s.sort_orders = "+-";
  Table* r = s.execute(t);
  CHECK(r != nullptr);
  if (r) {
    // keys first (d, k), then x and the row id
    CHECK(r->columns.size() == 4 && r->row_num == t->row_num);
    const int32_t* rd = r->columns[0]->as<int32_t>();
    const int64_t* rk = r->columns[1]->as<int64_t>();
    const int32_t* rid = r->columns[3]->as<int32_t>();
    auto dkey = [](int32_t v) { return v == kIntNull ? INT64_MIN : (int64_t)v; };   // NULL first ascending
    auto kkey = [](int64_t v) { return v == kLongNull ? INT64_MAX : -v; };          // descending, NULL last
    bool ok = true;
    std::vector<bool> seen(t->row_num, false);
    for (uint32_t i = 0; ok && i < r->row_num; i++) {
      ok = rd[i] == d[rid[i]] && rk[i] == k[rid[i]] && !seen[rid[i]];
      seen[rid[i]] = true;
      if (ok && i > 0) {
        const auto a = std::make_tuple(dkey(rd[i - 1]), kkey(rk[i - 1]), rid[i - 1]);
        const auto b = std::make_tuple(dkey(rd[i]), kkey(rk[i]), rid[i]);
        ok = a < b;   // ordered, and equal keys in input order
      }
    }
    CHECK(ok);
    delete r;
  }
  delete t;
}

int main() {
  test_filter();
  test_groupby();
  test_join();
  test_sort();
  if (failures) {
    std::printf("%d checks failed\n", failures);
    return 1;
  }
  std::printf("ok\n");
  return 0;
}
