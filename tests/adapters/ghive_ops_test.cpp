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
  // a three-table chain: left joins right on its key, then the tuples join a
  // third table by the right table's key (join_cols[1] serves both steps),
  // LEFT OUTER: right keys without a third row keep their tuple with NULLs
  {
    const uint32_t n3 = 400;
    Table* third = new Table();
    Column* tk = new Column(LONG, n3);
    Column* tv = new Column(LONG, n3);
    for (uint32_t i = 0; i < n3; i++) {
      tk->as<int64_t>()[i] = (int64_t)(2 * i);   // the even right keys below 800
      tv->as<int64_t>()[i] = (int64_t)i * 11 - 5;
    }
    third->columns = {tk, tv};
    third->row_num = n3;
    HashJoinPredicate three;
    three.join_cols = {{0}, {0}, {0}};
    three.maintain_cols = {{1}, {1}, {1}};
    three.join_types = {{INNER_JOIN, {0u, 1u}}, {LEFT_OUTER_JOIN, {1u, 2u}}};
    Table* r = three.process({left, right, third});
    CHECK(r != nullptr);
    if (r) {
      std::multiset<std::tuple<int32_t, int64_t, int64_t, int32_t, int32_t, int32_t>> expect, got;
      for (uint32_t i = 0; i < nl; i++) {
        const int64_t key = lk->as<int64_t>()[i];
        if (key == kLongNull || key >= (int64_t)nr) continue;
        const bool t3 = key % 2 == 0 && key < 2 * (int64_t)n3;
        expect.insert(std::make_tuple((int32_t)i, rv->as<int64_t>()[key], t3 ? tv->as<int64_t>()[key / 2] : kLongNull,
                                      (int32_t)i, (int32_t)key, t3 ? (int32_t)(key / 2) : -1));
      }
      CHECK(r->columns.size() == 3 && three.result_offsets.size() == 3 * (size_t)r->row_num);
      for (uint32_t i = 0; r->columns.size() == 3 && i < r->row_num; i++)
        got.insert(std::make_tuple(r->columns[0]->as<int32_t>()[i], r->columns[1]->as<int64_t>()[i],
                                   r->columns[2]->as<int64_t>()[i], three.result_offsets[3 * i],
                                   three.result_offsets[3 * i + 1], three.result_offsets[3 * i + 2]));
      CHECK(got == expect);
      delete r;
    }
    delete third;
  }
  // a semi join: the right table contributes no columns and no offsets
  {
    HashJoinPredicate semi;
    semi.join_cols = {{0}, {0}};
    semi.maintain_cols = {{1, 0}, {1}};
    semi.join_types = {{LEFT_SEMI_JOIN, {0u, 1u}}};
    Table* r = semi.process({left, right});
    CHECK(r != nullptr);
    if (r) {
      std::multiset<int32_t> expect, got;
      for (uint32_t i = 0; i < nl; i++) {
        const int64_t key = lk->as<int64_t>()[i];
        if (key != kLongNull && key < (int64_t)nr) expect.insert((int32_t)i);
      }
      bool ok = r->columns.size() == 2 && semi.result_offsets.size() == (size_t)r->row_num;
      for (uint32_t i = 0; ok && i < r->row_num; i++) {
        got.insert(r->columns[0]->as<int32_t>()[i]);
        ok = semi.result_offsets[i] == r->columns[0]->as<int32_t>()[i] &&
             r->columns[1]->as<int64_t>()[i] == lk->as<int64_t>()[semi.result_offsets[i]];
      }
      CHECK(ok && got == expect);
      delete r;
    }
  }
  // a step that reads a table not joined yet is refused
  HashJoinPredicate wrong;
  wrong.join_cols = {{0}, {0}, {0}};
  wrong.join_types = {{INNER_JOIN, {0u, 1u}}, {INNER_JOIN, {2u, 1u}}};
  CHECK(wrong.process({left, right, right}) == nullptr && !last_error().empty());
  delete left;
  delete right;
}

// A join on a STRING key column (with NULL keys) that keeps a STRING column
// of the build side: the strings come back as their own bytes and pairs.
static void test_string_join() {
  const char* names[] = {"ALGERIA", "ARGENTINA", "BRAZIL", "CANADA", "EGYPT", "", "\xc3\x89TATS"};
  const uint32_t nn = 7, nl = 5000;
  std::string lchars;
  std::vector<int32_t> lpairs;
  std::mt19937_64 g(5);
  std::vector<int> pick(nl);
  for (uint32_t i = 0; i < nl; i++) {
    pick[i] = (int)(g() % (nn + 2)) - 1;   // -1: NULL, nn: a name no build row has
    if (pick[i] < 0) {
      lpairs.insert(lpairs.end(), {-1, -1});
      continue;
    }
    const std::string v = pick[i] < (int)nn ? names[pick[i]] : "NOWHERE";
    lpairs.push_back((int32_t)lchars.size());
    lchars += v;
    lpairs.push_back((int32_t)lchars.size());
  }
  std::string rchars;
  std::vector<int32_t> rpairs, apairs;
  std::string achars;
  for (uint32_t i = 0; i < nn; i++) {
    rpairs.push_back((int32_t)rchars.size());
    rchars += names[i];
    rpairs.push_back((int32_t)rchars.size());
    const std::string a = std::string("region-") + std::to_string(i % 3);
    apairs.push_back((int32_t)achars.size());
    achars += a;
    apairs.push_back((int32_t)achars.size());
  }
  Table* left = new Table();
  left->columns = {new Column(STRING, nl, (void*)lchars.data(), lpairs.data(), (uint32_t)lchars.size())};
  left->row_num = nl;
  Table* right = new Table();
  right->columns = {new Column(STRING, nn, (void*)rchars.data(), rpairs.data(), (uint32_t)rchars.size()),
                    new Column(STRING, nn, (void*)achars.data(), apairs.data(), (uint32_t)achars.size())};
  right->row_num = nn;
  HashJoinPredicate j;
  j.join_cols = {{0}, {0}};
  j.maintain_cols = {{0}, {1}};
  j.join_types = {{INNER_JOIN, {0u, 1u}}};
  Table* r = j.process({left, right});
  CHECK(r != nullptr);
  if (r) {
    auto str = [](const Column* c, uint32_t i) {
      const int32_t* p = (const int32_t*)c->data_ptr_aux;
      return std::string((const char*)c->data_ptr + p[2 * i], p[2 * i + 1] - p[2 * i]);
    };
    std::multiset<std::pair<std::string, std::string>> expect, got;
    for (uint32_t i = 0; i < nl; i++)
      if (pick[i] >= 0 && pick[i] < (int)nn)
        expect.insert({names[pick[i]], std::string("region-") + std::to_string(pick[i] % 3)});
    bool ok = r->columns.size() == 2 && r->columns[0]->type == STRING && r->columns[1]->type == STRING;
    for (uint32_t i = 0; ok && i < r->row_num; i++) {
      got.insert({str(r->columns[0], i), str(r->columns[1], i)});
      ok = str(r->columns[0], i) == names[pick[j.result_offsets[2 * i]]];
    }
    CHECK(ok && got == expect);
    delete r;
  }
  delete left;   // the columns wrap the strings above and own nothing
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

// GHive's own N-way join case (JoinPredicateTest.cu), read from a text file
// the test driver writes from the committed fixture: the tables (one LONG
// key column each), the chain's steps, and the expected result_offsets.
// The offsets are compared as a multiset of per-row tuples (the reference's
// come in key order, these in no particular order).
static void test_golden_chain(const char* path) {
  FILE* f = std::fopen(path, "r");
  CHECK(f != nullptr);
  if (!f) return;
  int nt = 0;
  CHECK(std::fscanf(f, "%d", &nt) == 1);
  std::vector<Table*> tables;
  for (int t = 0; t < nt; t++) {
    int n = 0;
    CHECK(std::fscanf(f, "%d", &n) == 1);
    Column* c = new Column(LONG, (uint32_t)n);
    for (int i = 0; i < n; i++) CHECK(std::fscanf(f, "%ld", &c->as<int64_t>()[i]) == 1);
    Table* tb = new Table();
    tb->columns = {c};
    tb->row_num = (uint32_t)n;
    tables.push_back(tb);
  }
  HashJoinPredicate j;
  j.join_cols.assign(nt, {0});
  j.maintain_cols.assign(nt, {0});
  int ns = 0;
  CHECK(std::fscanf(f, "%d", &ns) == 1);
  for (int i = 0; i < ns; i++) {
    int type = 0;
    unsigned a = 0, b = 0;
    CHECK(std::fscanf(f, "%d %u %u", &type, &a, &b) == 3);
    j.join_types.push_back({(BaseJoinType)type, {a, b}});
  }
  int ne = 0;
  CHECK(std::fscanf(f, "%d", &ne) == 1);
  std::vector<int32_t> expect(ne);
  for (int i = 0; i < ne; i++) CHECK(std::fscanf(f, "%d", &expect[i]) == 1);
  std::fclose(f);
  Table* r = j.process(tables);
  CHECK(r != nullptr);
  if (r) {
    const size_t w = j.result_offsets.size() / std::max<size_t>(1, r->row_num);
    CHECK(w > 0 && expect.size() % w == 0);
    std::multiset<std::vector<int32_t>> got, exp;
    for (size_t i = 0; w && i + w <= j.result_offsets.size(); i += w)
      got.insert(std::vector<int32_t>(j.result_offsets.begin() + i, j.result_offsets.begin() + i + w));
    for (size_t i = 0; w && i + w <= expect.size(); i += w)
      exp.insert(std::vector<int32_t>(expect.begin() + i, expect.begin() + i + w));
    CHECK(got == exp);
    delete r;
  }
  for (Table* t : tables) delete t;
}

int main(int argc, char** argv) {
  test_filter();
  test_groupby();
  test_join();
  test_string_join();
  test_sort();
  if (argc > 1) test_golden_chain(argv[1]);
  if (failures) {
    std::printf("%d checks failed\n", failures);
    return 1;
  }
  std::printf("ok\n");
  return 0;
}
