// ghb_plan.cu — GHive's JNI marshaling (GTables in, GPUResult out) and a
// vertex's operator chain run on device-resident intermediates.
//
// GHive's entry point GPUProcess (gpu_impl/src/ghive_JNIInterface.cu:13-215)
// reads the Tez task's GTables object: per input table its column types,
// row and key counts, and the columns as direct ByteBuffers, concatenated by
// type over the tables in table order (each table takes its columns, in its
// types[] order, from the next unused buffer of the type, :152-201).  It then
// runs the vertex's plan, root_op->execute() (gpu_impl/src/Parser/
// Parser.cu:675), where every operator copies its input in and its output
// back to host columns (FilterOperator.cu:53-89, GroupByPredicate.cu:39-91),
// and builds a GPUResult: the result's columns grouped by type (long[][],
// double[][], int[][], String[][]) and sequence[i] = the index of result
// column i in the concatenation long || double || int || string
// (ghive_JNIInterface.cu:217-340).
//
// Here:
//   ghb_gtables_table   one input table's columns as descriptors over the
//                       JVM's buffers (no copy), NULLs as GHive's sentinels;
//   ghb_run_plan        the vertex's chain of operators on one input table
//                       (and build tables made from the others): the input
//                       columns are copied to the device once, each
//                       operator's output stays on the device as the next
//                       one's input, and only the final table comes back,
//                       with GPUResult's grouping and sequence.
#include <algorithm>
#include <cstdlib>
#include <vector>

#include "ghb_ctx.hpp"
#include "ghb_log.hpp"

namespace ghb {
namespace {

size_t width_of(int32_t t) { return type_width(t); }

// Columns of an input table or an intermediate the plan holds (each
// operator checks the columns it touches against its own limit).
constexpr int kPlanCols = 64;

// A device column the plan owns.  A STRING column is its int32 [start,end)
// pairs (start < 0: NULL) in `data` and the bytes they index in `bytes`,
// which operators pass through unchanged: a filter, group-by, join or sort
// moves pairs, never bytes, and the result gathers the bytes it references.
struct DevCol {
  int32_t type = GHB_LONG;
  void* data = nullptr;
  uint8_t* is_null = nullptr;   // NULL map (nullptr: no NULLs, or sentinels)
  int32_t null_mode = GHB_NULLS_NONE;
  const uint8_t* bytes = nullptr;
  int64_t nbytes = 0;
};

// (start, end) + add for each non-NULL pair: the build side's pairs moved
// behind the probe side's bytes in a joined dictionary.
__global__ void __launch_bounds__(256) offset_pairs_kernel(const int2* in, int64_t n, int32_t add, int2* out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    int2 v = in[i];
    if (v.x >= 0) {
      v.x += add;
      v.y += add;
    }
    out[i] = v;
  }
}

// Copies each non-NULL row's bytes from src[from) to dst[to): the result's
// strings packed one after the other.
__global__ void __launch_bounds__(256) gather_string_bytes_kernel(const uint8_t* src, const int2* from,
                                                                  const int2* to, int64_t n, uint8_t* dst) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int2 f = from[i];
    if (f.x < 0) continue;
    const int2 t = to[i];
    for (int b = 0; b < f.y - f.x; b++) dst[t.x + b] = src[f.x + b];
  }
}

struct DevTable {
  std::vector<DevCol> cols;
  int64_t rows = 0;
};

struct Plan {
  ghb_ctx* ctx;
  cudaStream_t s;
  std::vector<void*> owned;

  ~Plan() {
    cudaStreamSynchronize(s);
    for (void* p : owned) cudaFreeAsync(p, s);
    cudaStreamSynchronize(s);
  }
  int32_t alloc(size_t bytes, void** out) {
    *out = nullptr;
    if (cudaMallocAsync(out, std::max<size_t>(bytes, 16), s) != cudaSuccess) {
      cudaGetLastError();
      return set_error(ctx, GHB_ERR_OOM, "cannot allocate %zu bytes of device memory", bytes);
    }
    owned.push_back(*out);
    return GHB_OK;
  }
  // an output column of `rows` rows with a NULL map; a STRING one is its
  // pairs only (a NULL is a negative start) and takes `bytes` from its source
  int32_t out_col(int32_t type, int64_t rows, DevCol* c, ghb_out_column* o, const DevCol* src = nullptr) {
    int32_t st;
    c->type = type;
    if ((st = alloc((size_t)std::max<int64_t>(rows, 1) * width_of(type), &c->data))) return st;
    if (type == GHB_STRING) {
      c->null_mode = GHB_NULLS_SENTINEL;
      c->bytes = src ? src->bytes : nullptr;
      c->nbytes = src ? src->nbytes : 0;
      *o = ghb_out_column{type, 0, c->data, nullptr};
      return GHB_OK;
    }
    if ((st = alloc((size_t)std::max<int64_t>(rows, 1), (void**)&c->is_null))) return st;
    c->null_mode = GHB_NULLS_BYTEMAP;
    *o = ghb_out_column{type, 0, c->data, c->is_null};
    return GHB_OK;
  }
  int32_t read_count(const int64_t* d, int64_t* h) {
    GHB_CUDA_TRY(ctx, cudaMemcpyAsync(h, d, 8, cudaMemcpyDeviceToHost, s));
    return ghb_sync(ctx, s);
  }
};

ghb_column desc(const DevCol& c, int64_t rows) {
  if (c.type == GHB_STRING) return ghb_column{GHB_STRING, GHB_NULLS_SENTINEL, c.bytes, nullptr, c.data, rows};
  return ghb_column{c.type, c.null_mode, c.data, c.null_mode == GHB_NULLS_BYTEMAP ? c.is_null : nullptr,
                    nullptr, rows};
}

// A column as an operator's fixed-width payload: a STRING column travels as
// its pairs, 8 bytes a row (a NULL string's pair is copied like any value).
ghb_column payload_desc(const DevCol& c, int64_t rows) {
  if (c.type == GHB_STRING) return ghb_column{GHB_LONG, GHB_NULLS_NONE, c.data, nullptr, nullptr, rows};
  return desc(c, rows);
}

// The output slot of such a payload: a STRING column's pairs as LONG words
// with no NULL map, so an outer join's miss writes the LONG sentinel, whose
// low word -1 is a NULL pair.
ghb_out_column payload_out(const ghb_out_column& o) {
  if (o.type == GHB_STRING) return ghb_out_column{GHB_LONG, 0, o.data, nullptr};
  return o;
}

// Copies host table columns to the device (GHive's sentinels kept).
int32_t upload(Plan& P, const ghb_column* h, int32_t ncols, int64_t rows, DevTable* t) {
  t->rows = rows;
  t->cols.assign(ncols, DevCol{});
  std::vector<CopyTask> copies;   // every column's copies, issued together
  for (int c = 0; c < ncols; c++) {
    if (h[c].type == GHB_STRING) {
      // the pairs, and the bytes up to the largest end a non-NULL row uses
      DevCol& d = t->cols[c];
      d.type = GHB_STRING;
      d.null_mode = GHB_NULLS_SENTINEL;
      const int2* pairs = (const int2*)h[c].aux;
      if (rows > 0 && !pairs) return set_error(P.ctx, GHB_ERR_INVALID, "column %d: STRING without its index", c);
      int64_t nb = 0;
      for (int64_t r = 0; r < rows; r++)
        if (pairs[r].x >= 0) {
          if (pairs[r].y < pairs[r].x)
            return set_error(P.ctx, GHB_ERR_INVALID, "column %d row %lld: end before start", c, (long long)r);
          nb = std::max<int64_t>(nb, pairs[r].y);
        }
      if (nb > 0 && !h[c].data) return set_error(P.ctx, GHB_ERR_INVALID, "column %d: STRING without its bytes", c);
      int32_t st = P.alloc((size_t)std::max<int64_t>(rows, 1) * 8, &d.data);
      void* bytes = nullptr;
      if (!st) st = P.alloc((size_t)std::max<int64_t>(nb, 1), &bytes);
      if (st) return st;
      d.bytes = (const uint8_t*)bytes;
      d.nbytes = nb;
      if (rows > 0) copies.push_back({d.data, pairs, (size_t)rows * 8});
      if (nb > 0) copies.push_back({bytes, h[c].data, (size_t)nb});
      continue;
    }
    DevCol& d = t->cols[c];
    d.type = h[c].type;
    d.null_mode = h[c].null_mode;
    int32_t st = P.alloc((size_t)std::max<int64_t>(rows, 1) * width_of(d.type), &d.data);
    if (st) return st;
    if (rows > 0) {
      if (!h[c].data) return set_error(P.ctx, GHB_ERR_INVALID, "column %d: data is NULL", c);
      copies.push_back({d.data, h[c].data, (size_t)rows * width_of(d.type)});
    }
    if (h[c].null_mode == GHB_NULLS_BYTEMAP) {
      if ((st = P.alloc((size_t)std::max<int64_t>(rows, 1), (void**)&d.is_null))) return st;
      if (rows > 0) copies.push_back({d.is_null, h[c].is_null, (size_t)rows});
    }
  }
  return copy_h2d_many(P.ctx, copies, P.s);
}

std::vector<ghb_column> descs(const DevTable& t) {
  std::vector<ghb_column> v;
  for (const DevCol& c : t.cols) v.push_back(desc(c, t.rows));
  return v;
}

int32_t run_filter(Plan& P, const ghb_plan_op& op, DevTable& t) {
  std::vector<ghb_column> in = descs(t);
  std::vector<int32_t> proj;
  if (op.idx)
    proj.assign(op.idx, op.idx + op.nidx);
  else
    for (int c = 0; c < (int)t.cols.size(); c++) proj.push_back(c);
  if (proj.size() > (size_t)kPlanCols) return set_error(P.ctx, GHB_ERR_UNSUPPORTED, "projection of %zu columns", proj.size());
  for (int32_t c : proj)
    if (c < 0 || c >= (int)t.cols.size()) return set_error(P.ctx, GHB_ERR_INVALID, "projection column %d", c);
  if (!op.pred || op.pred->n_nodes == 0) {
    // a projection alone (GHive's SelectOperator): the columns, no copy
    DevTable o;
    o.rows = t.rows;
    for (int32_t c : proj) o.cols.push_back(t.cols[c]);
    t = std::move(o);
    return GHB_OK;
  }
  if (proj.size() > (size_t)kMaxCols) return set_error(P.ctx, GHB_ERR_UNSUPPORTED, "projection of %zu columns", proj.size());
  DevTable o;
  std::vector<ghb_out_column> out(proj.size());
  o.cols.resize(proj.size());
  int32_t st;
  for (size_t j = 0; j < proj.size(); j++)
    if ((st = P.out_col(t.cols[proj[j]].type, t.rows, &o.cols[j], &out[j], &t.cols[proj[j]]))) return st;
  int64_t* d_rows = nullptr;
  if ((st = P.alloc(8, (void**)&d_rows))) return st;
  if ((st = ghb_filter(P.ctx, op.pred, in.data(), (int32_t)in.size(), proj.data(), (int32_t)proj.size(),
                       out.data(), t.rows, d_rows, P.s)))
    return st;
  if ((st = P.read_count(d_rows, &o.rows))) return st;
  t = std::move(o);
  return GHB_OK;
}

int32_t agg_type(int32_t agg, int32_t in) {
  if (agg == GHB_AGG_CNT) return GHB_LONG;
  if (agg == GHB_AGG_AVG) return GHB_DOUBLE;
  if (agg == GHB_AGG_SUM) return in == GHB_DOUBLE ? GHB_DOUBLE : GHB_LONG;
  return in;
}

int32_t run_groupby(Plan& P, const ghb_plan_op& op, DevTable& t) {
  std::vector<ghb_column> in = descs(t);
  const int32_t nkeys = op.nidx, naggs = op.naggs;
  if (nkeys < 0 || naggs < 0 || nkeys + naggs > GHB_MAX_RESULT_COLS || (nkeys > 0 && !op.idx) ||
      (naggs > 0 && !op.aggs))
    return set_error(P.ctx, GHB_ERR_INVALID, "group-by: %d keys, %d aggregates", nkeys, naggs);
  int64_t cap = nkeys == 0 ? 1 : (op.max_groups > 0 ? op.max_groups : std::max<int64_t>(t.rows, 1));
  DevTable o;
  o.cols.resize(nkeys + naggs);
  std::vector<ghb_out_column> out(nkeys + naggs);
  int32_t st;
  for (int j = 0; j < nkeys; j++) {
    if (op.idx[j] < 0 || op.idx[j] >= (int)t.cols.size())
      return set_error(P.ctx, GHB_ERR_INVALID, "group-by key column %d", op.idx[j]);
    if ((st = P.out_col(t.cols[op.idx[j]].type, cap, &o.cols[j], &out[j], &t.cols[op.idx[j]]))) return st;
  }
  for (int a = 0; a < naggs; a++) {
    const int32_t c = op.aggs[a].col;
    const int32_t in_t = c >= 0 && c < (int)t.cols.size() ? t.cols[c].type : GHB_LONG;
    if ((st = P.out_col(agg_type(op.aggs[a].type, in_t), cap, &o.cols[nkeys + a], &out[nkeys + a]))) return st;
  }
  int64_t* d_groups = nullptr;
  if ((st = P.alloc(8, (void**)&d_groups))) return st;
  ghb_groupby_cfg cfg{};
  cfg.max_groups = cap;
  if ((st = ghb_filter_groupby(P.ctx, nullptr, in.data(), (int32_t)in.size(), op.idx, nkeys, op.aggs, naggs,
                               out.data(), cap, d_groups, &cfg, P.s)))
    return st;
  if ((st = P.read_count(d_groups, &o.rows))) return st;
  t = std::move(o);
  return GHB_OK;
}

// A STRING join key of both sides as LONG ids that are equal exactly when the
// strings are: the two sides' pairs over one byte array (the build side's
// bytes behind the probe side's), each row mapped to the row of its value's
// first occurrence in that joined column (a device hash table of the
// strings, bytes compared on a tag match); a NULL string gets the LONG
// sentinel and so matches nothing.
int32_t string_key_ids(Plan& P, const DevCol& pc, int64_t prows, const DevCol& bc, int64_t brows, DevCol* pid,
                       DevCol* bid) {
  const int64_t n = prows + brows;
  if (pc.nbytes + bc.nbytes >= INT32_MAX)
    return set_error(P.ctx, GHB_ERR_UNSUPPORTED, "join: STRING keys of 2^31 bytes together");
  void *bytes = nullptr, *pairs = nullptr, *rep = nullptr, *table = nullptr;
  int64_t slots = 1024;
  while (slots < 2 * n) slots <<= 1;
  int32_t st = P.alloc((size_t)std::max<int64_t>(pc.nbytes + bc.nbytes, 1), &bytes);
  if (!st) st = P.alloc((size_t)std::max<int64_t>(n, 1) * 8, &pairs);
  if (!st) st = P.alloc((size_t)std::max<int64_t>(n, 1) * 8, &rep);
  if (!st) st = P.alloc((size_t)slots * 8, &table);
  if (st) return st;
  if (pc.nbytes > 0)
    GHB_CUDA_TRY(P.ctx, cudaMemcpyAsync(bytes, pc.bytes, pc.nbytes, cudaMemcpyDeviceToDevice, P.s));
  if (bc.nbytes > 0)
    GHB_CUDA_TRY(P.ctx, cudaMemcpyAsync((uint8_t*)bytes + pc.nbytes, bc.bytes, bc.nbytes, cudaMemcpyDeviceToDevice, P.s));
  if (prows > 0) GHB_CUDA_TRY(P.ctx, cudaMemcpyAsync(pairs, pc.data, prows * 8, cudaMemcpyDeviceToDevice, P.s));
  if (brows > 0) {
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((brows + 255) / 256, (int64_t)P.ctx->num_sms * 8));
    offset_pairs_kernel<<<grid, 256, 0, P.s>>>((const int2*)bc.data, brows, (int32_t)pc.nbytes,
                                               (int2*)pairs + prows);
    GHB_LAUNCH_CHECK(P.ctx);
  }
  const ghb_column joined{GHB_STRING, GHB_NULLS_SENTINEL, bytes, nullptr, pairs, n};
  if ((st = string_rep_rows(P.ctx, joined, nullptr, (int64_t*)rep, (unsigned long long*)table, slots, P.s)))
    return st;
  for (DevCol* d : {pid, bid}) {
    d->type = GHB_LONG;
    d->null_mode = GHB_NULLS_SENTINEL;
    d->is_null = nullptr;
  }
  pid->data = rep;
  bid->data = (int64_t*)rep + prows;
  return GHB_OK;
}

// The current table probes a hash table built from input table op.build_table:
// output = the current table's columns, then the kept build columns.  Keys
// of several columns are packed into one; STRING key columns first become
// ids shared by both sides (string_key_ids); STRING payloads travel as
// their pairs into their own side's bytes.
int32_t run_join(Plan& P, const ghb_plan_op& op, const ghb_gtables* in, DevTable& t) {
  // idx: the probe key columns, then as many build key columns
  if (!op.idx || op.nidx < 2 || op.nidx % 2 || op.nidx / 2 > kMaxPackKeys)
    return set_error(P.ctx, GHB_ERR_INVALID, "join: idx must hold k probe and k build key columns");
  const int nk = op.nidx / 2;
  ghb_column hb[kPlanCols];
  int32_t nb = 0;
  int64_t brows = 0;
  int32_t st = ghb_gtables_table(in, op.build_table, hb, kPlanCols, &nb, &brows);
  if (st) return set_error(P.ctx, st, "join: build table %d is missing or malformed", op.build_table);
  for (int j = 0; j < nk; j++) {
    if (op.idx[j] < 0 || op.idx[j] >= (int)t.cols.size() || op.idx[nk + j] < 0 || op.idx[nk + j] >= nb)
      return set_error(P.ctx, GHB_ERR_INVALID, "join key columns %d / %d", op.idx[j], op.idx[nk + j]);
    if ((t.cols[op.idx[j]].type == GHB_STRING) != (hb[op.idx[nk + j]].type == GHB_STRING))
      return set_error(P.ctx, GHB_ERR_INVALID, "join key %d: a STRING column against a numeric one", j);
  }
  if ((int)t.cols.size() > GHB_MAX_JOIN_PAYLOAD || op.nbuild_keep > GHB_MAX_JOIN_PAYLOAD || op.nbuild_keep < 0)
    return set_error(P.ctx, GHB_ERR_UNSUPPORTED, "join: at most %d columns from each side", GHB_MAX_JOIN_PAYLOAD);
  // the build side's key and kept columns on the device
  std::vector<ghb_column> bsel;
  for (int j = 0; j < nk; j++) bsel.push_back(hb[op.idx[nk + j]]);
  for (int j = 0; j < op.nbuild_keep; j++) {
    const int32_t c = op.build_keep[j];
    if (c < 0 || c >= nb) return set_error(P.ctx, GHB_ERR_INVALID, "join: build column %d", c);
    bsel.push_back(hb[c]);
  }
  DevTable b;
  if ((st = upload(P, bsel.data(), (int32_t)bsel.size(), brows, &b))) return st;
  // the key columns of both sides: STRING ones as shared ids
  std::vector<DevCol> pkc(nk), bkc(nk);
  for (int j = 0; j < nk; j++) {
    pkc[j] = t.cols[op.idx[j]];
    bkc[j] = b.cols[j];
    if (pkc[j].type == GHB_STRING && (st = string_key_ids(P, pkc[j], t.rows, bkc[j], b.rows, &pkc[j], &bkc[j])))
      return st;
  }
  ghb_column pkey = desc(pkc[0], t.rows), bkey = desc(bkc[0], b.rows);
  if (nk > 1) {
    // several key columns: both sides' tuples packed with one plan
    std::vector<ghb_column> pk(nk), bk(nk);
    for (int j = 0; j < nk; j++) {
      pk[j] = desc(pkc[j], t.rows);
      bk[j] = desc(bkc[j], b.rows);
    }
    DevCol pp, bp;
    for (DevCol* c : {&pp, &bp}) {
      const int64_t rows = c == &pp ? t.rows : b.rows;
      c->type = GHB_LONG;
      c->null_mode = GHB_NULLS_BYTEMAP;
      if ((st = P.alloc((size_t)std::max<int64_t>(rows, 1) * 8, &c->data)) ||
          (st = P.alloc((size_t)std::max<int64_t>(rows, 1), (void**)&c->is_null)))
        return st;
    }
    scratch_reset(P.ctx);
    if ((st = scratch_reserve(P.ctx, 4096, P.s))) return st;
    if ((st = keypack_join(P.ctx, pk.data(), bk.data(), nk, (int64_t*)pp.data, pp.is_null, (int64_t*)bp.data,
                           bp.is_null, P.s)))
      return st;
    pkey = desc(pp, t.rows);
    bkey = desc(bp, b.rows);
  }
  std::vector<ghb_column> bpay;
  for (int j = 0; j < op.nbuild_keep; j++) bpay.push_back(payload_desc(b.cols[nk + j], b.rows));
  ghb_join_table* jt = nullptr;
  if ((st = ghb_join_build(P.ctx, &bkey, bpay.data(), op.nbuild_keep, nullptr, &jt, P.s))) return st;
  int64_t rows = 0, max_dup = 1, slots = 0;
  if ((st = ghb_sync(P.ctx, P.s)) || (st = ghb_join_table_info(P.ctx, jt, &rows, &max_dup, &slots))) {
    ghb_join_table_free(P.ctx, jt);
    return st;
  }
  int64_t per = op.join_type == GHB_LEFT_SEMI_JOIN ? 1 : std::max<int64_t>(1, max_dup);
  const int64_t cap = std::max<int64_t>(1, t.rows * per);
  DevTable o;
  const int np = (int)t.cols.size();
  o.cols.resize(np + op.nbuild_keep);
  std::vector<ghb_out_column> op_out(np), ob_out(op.nbuild_keep);
  std::vector<ghb_column> probe(np);
  for (int j = 0; j < np && !st; j++) {
    probe[j] = payload_desc(t.cols[j], t.rows);
    st = P.out_col(t.cols[j].type, cap, &o.cols[j], &op_out[j], &t.cols[j]);
    op_out[j] = payload_out(op_out[j]);
  }
  for (int j = 0; j < op.nbuild_keep && !st; j++) {
    st = P.out_col(b.cols[nk + j].type, cap, &o.cols[np + j], &ob_out[j], &b.cols[nk + j]);
    ob_out[j] = payload_out(ob_out[j]);
  }
  int64_t* d_rows = nullptr;
  if (!st) st = P.alloc(8, (void**)&d_rows);
  if (!st)
    st = ghb_join_probe(P.ctx, jt, &pkey, op.join_type, ob_out.data(), probe.data(), np, op_out.data(),
                        nullptr, nullptr, cap, d_rows, P.s);
  if (!st) st = P.read_count(d_rows, &o.rows);
  ghb_join_table_free(P.ctx, jt);
  if (st) return st;
  t = std::move(o);
  return GHB_OK;
}

// ORDER BY: the key columns first, then the others (GHive's Sink keeps that
// order, SinkOperator.cu:98-306).
int32_t run_sort(Plan& P, const ghb_plan_op& op, DevTable& t) {
  if (!op.idx || op.nidx < 1) return set_error(P.ctx, GHB_ERR_INVALID, "sort without keys");
  std::vector<ghb_column> in = descs(t);
  std::vector<bool> is_key(t.cols.size(), false);
  std::vector<ghb_column> keys, pay;
  std::vector<int32_t> pay_idx;
  for (int j = 0; j < op.nidx; j++) {
    const int32_t c = op.idx[j];
    if (c < 0 || c >= (int)t.cols.size() || is_key[c])
      return set_error(P.ctx, GHB_ERR_INVALID, "sort key column %d", c);
    is_key[c] = true;
    keys.push_back(in[c]);
  }
  for (int c = 0; c < (int)t.cols.size(); c++)
    if (!is_key[c]) {
      pay.push_back(payload_desc(t.cols[c], t.rows));
      pay_idx.push_back(c);
    }
  DevTable o;
  o.rows = t.rows;
  o.cols.resize(t.cols.size());
  std::vector<ghb_out_column> ok(keys.size()), opay(pay.size());
  int32_t st;
  for (size_t j = 0; j < keys.size(); j++)
    if ((st = P.out_col(keys[j].type, t.rows, &o.cols[j], &ok[j], &t.cols[op.idx[j]]))) return st;
  for (size_t j = 0; j < pay.size(); j++) {
    const DevCol& src = t.cols[pay_idx[j]];
    if ((st = P.out_col(src.type, t.rows, &o.cols[keys.size() + j], &opay[j], &src))) return st;
    opay[j] = payload_out(opay[j]);
  }
  if ((st = ghb_sort(P.ctx, keys.data(), op.orders, op.null_orders, (int32_t)keys.size(), pay.data(),
                     (int32_t)pay.size(), ok.data(), opay.data(), nullptr, nullptr, P.s)))
    return st;
  if ((st = ghb_sync(P.ctx, P.s))) return st;
  t = std::move(o);
  return GHB_OK;
}

// A STRING result column: its rows' bytes packed one after the other into
// out->str_bytes[c] and its pairs, rebased onto them, into out->data[c]
// (GPUResult builds each row's String from its [start,end)).
int32_t download_string(Plan& P, const DevCol& d, int64_t rows, ghb_plan_result* out, int c) {
  std::vector<int2> from((size_t)std::max<int64_t>(rows, 1)), to((size_t)std::max<int64_t>(rows, 1));
  int32_t st;
  if (rows > 0 && (st = copy_d2h_many(P.ctx, {CopyTask{from.data(), d.data, (size_t)rows * 8}}, P.s))) return st;
  int64_t total = 0;
  for (int64_t r = 0; r < rows; r++) {
    if (from[r].x < 0) {
      to[r] = make_int2(-1, -1);
      continue;
    }
    to[r] = make_int2((int32_t)total, (int32_t)(total + (from[r].y - from[r].x)));
    total += from[r].y - from[r].x;
    if (total >= INT32_MAX) return set_error(P.ctx, GHB_ERR_UNSUPPORTED, "result column %d: 2^31 bytes of strings", c);
  }
  out->data[c] = std::malloc((size_t)std::max<int64_t>(rows, 1) * 8);
  out->str_bytes[c] = (uint8_t*)std::malloc((size_t)std::max<int64_t>(total, 1));
  if (!out->data[c] || !out->str_bytes[c]) return set_error(P.ctx, GHB_ERR_OOM, "cannot allocate host memory for the result");
  std::memcpy(out->data[c], to.data(), (size_t)rows * 8);
  out->str_nbytes[c] = total;
  if (total == 0) return GHB_OK;
  void *d_to = nullptr, *d_bytes = nullptr;
  st = P.alloc((size_t)rows * 8, &d_to);
  if (!st) st = P.alloc((size_t)total, &d_bytes);
  if (st) return st;
  if ((st = copy_h2d(P.ctx, d_to, to.data(), (size_t)rows * 8, P.s))) return st;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((rows + 255) / 256, (int64_t)P.ctx->num_sms * 8));
  gather_string_bytes_kernel<<<grid, 256, 0, P.s>>>(d.bytes, (const int2*)d.data, (const int2*)d_to, rows,
                                                    (uint8_t*)d_bytes);
  GHB_LAUNCH_CHECK(P.ctx);
  return copy_d2h_many(P.ctx, {CopyTask{out->str_bytes[c], d_bytes, (size_t)total}}, P.s);
}

}  // namespace
}  // namespace ghb

using namespace ghb;

extern "C" {

int32_t ghb_gtables_table(const ghb_gtables* in, int32_t table, ghb_column* cols, int32_t cap,
                          int32_t* ncols, int64_t* rows) {
  if (!in || !ncols || table < 0 || table >= in->ntables || !in->ncols || !in->types || !in->row_cnt)
    return GHB_ERR_INVALID;
  if (in->vertex_name && !in->vertex_name[table]) return GHB_ERR_INVALID;   // the table is missing
  // the next unused buffer of each type: the tables before this one took theirs
  int32_t next[4] = {0, 0, 0, 0};
  for (int t = 0; t < table; t++)
    for (int c = 0; c < in->ncols[t]; c++) {
      const int32_t ty = in->types[t][c];
      if (ty < 0 || ty > 3) return GHB_ERR_INVALID;
      next[ty]++;
    }
  const int32_t n = in->ncols[table];
  if (n > cap) return GHB_ERR_INVALID;
  const int64_t r = in->row_cnt[table];
  const int32_t have[4] = {in->nlong, in->ndouble, in->nint, in->nstring};
  const void* const* bufs[4] = {in->long_cols, in->double_cols, in->int_cols, in->string_cols};
  for (int c = 0; c < n; c++) {
    const int32_t ty = in->types[table][c];
    if (ty < 0 || ty > 3 || next[ty] >= have[ty] || !bufs[ty]) return GHB_ERR_INVALID;
    ghb_column& d = cols[c];
    d.type = ty;
    d.null_mode = GHB_NULLS_SENTINEL;
    d.data = bufs[ty][next[ty]];
    d.is_null = nullptr;
    d.aux = ty == GHB_STRING && in->string_idx_cols ? in->string_idx_cols[next[ty]] : nullptr;
    d.n = r;
    next[ty]++;
  }
  *ncols = n;
  if (rows) *rows = r;
  return GHB_OK;
}

static int32_t ghb_run_plan_body(ghb_ctx* ctx, const ghb_gtables* in, int32_t input, const ghb_plan_op* ops,
                     int32_t nops, ghb_plan_result* out) {
  if (!ctx || !in || !out || (nops > 0 && !ops) || nops < 0) return GHB_ERR_INVALID;
  std::memset(out, 0, sizeof(*out));
  ghb_column hc[kPlanCols];
  int32_t nc = 0;
  int64_t rows = 0;
  if (ghb_gtables_table(in, input, hc, kPlanCols, &nc, &rows))
    return set_error(ctx, GHB_ERR_INVALID, "input table %d is missing or malformed", input);
  if (!ctx->hstream[1]) GHB_CUDA_TRY(ctx, cudaStreamCreateWithFlags(&ctx->hstream[1], cudaStreamNonBlocking));
  Plan P{ctx, ctx->hstream[1], {}};
  DevTable t;
  int32_t st;
  {
    CallScope cs(ctx, "plan_upload", P.s, true);
    cs.rows(rows);
    cs.bytes(cols_bytes(hc, nc));
    st = cs.done(upload(P, hc, nc, rows, &t));
    if (!st) st = cs.done(ghb_sync(ctx, P.s));
  }
  if (st) return st;
  for (int i = 0; i < nops && !st; i++) {
    switch (ops[i].op) {
      case GHB_OP_FILTER: st = run_filter(P, ops[i], t); break;
      case GHB_OP_GROUPBY: st = run_groupby(P, ops[i], t); break;
      case GHB_OP_JOIN_PROBE: st = run_join(P, ops[i], in, t); break;
      case GHB_OP_SORT: st = run_sort(P, ops[i], t); break;
      default: st = set_error(ctx, GHB_ERR_INVALID, "plan op %d: unknown operator %d", i, ops[i].op);
    }
  }
  if (st) return st;
  if ((int)t.cols.size() > GHB_MAX_RESULT_COLS)
    return set_error(ctx, GHB_ERR_UNSUPPORTED, "result of %zu columns (at most %d)", t.cols.size(),
                     GHB_MAX_RESULT_COLS);
  CallScope dl(ctx, "plan_download", P.s, true);
  dl.rows(t.rows);
  // the result: host columns (NULLs as GHive's sentinels, and a NULL map),
  // grouped by type the way GPUResult holds them
  out->ncols = (int32_t)t.cols.size();
  out->rows = t.rows;
  int32_t count[4] = {0, 0, 0, 0};
  for (const DevCol& c : t.cols) count[c.type]++;
  out->n_long = count[GHB_LONG];
  out->n_double = count[GHB_DOUBLE];
  out->n_int = count[GHB_INT];
  out->n_string = count[GHB_STRING];
  const int32_t base[4] = {0, count[0], count[0] + count[1], count[0] + count[1] + count[2]};
  int32_t seen[4] = {0, 0, 0, 0};
  std::vector<CopyTask> copies;   // every fixed-width column's copies, issued together
  for (int c = 0; c < out->ncols; c++) {
    const DevCol& d = t.cols[c];
    out->types[c] = d.type;
    out->sequence[c] = base[d.type] + seen[d.type]++;
    if (d.type == GHB_STRING) {
      if ((st = download_string(P, d, t.rows, out, c))) {
        ghb_plan_result_free(out);
        return st;
      }
      continue;
    }
    const size_t bytes = (size_t)std::max<int64_t>(t.rows, 1) * width_of(d.type);
    out->data[c] = std::malloc(bytes);
    if (d.is_null) out->is_null[c] = (uint8_t*)std::malloc((size_t)std::max<int64_t>(t.rows, 1));
    if (!out->data[c] || (d.is_null && !out->is_null[c])) {
      ghb_plan_result_free(out);
      return set_error(ctx, GHB_ERR_OOM, "cannot allocate host memory for the result");
    }
    if (t.rows > 0) {
      copies.push_back({out->data[c], d.data, (size_t)t.rows * width_of(d.type)});
      if (d.is_null) copies.push_back({out->is_null[c], d.is_null, (size_t)t.rows});
    }
  }
  if ((st = copy_d2h_many(ctx, copies, P.s))) {
    ghb_plan_result_free(out);
    return st;
  }
  return GHB_OK;
}

int32_t ghb_run_plan(ghb_ctx* ctx, const ghb_gtables* in, int32_t input, const ghb_plan_op* ops, int32_t nops,
                     ghb_plan_result* out) {
  CallScope cs(ctx, "run_plan", 0, true);
  ghb_column hc[kPlanCols];
  int32_t nc = 0;
  int64_t rows = 0;
  if (ghb_gtables_table(in, input, hc, kPlanCols, &nc, &rows) == GHB_OK) {
    cs.rows(rows);
    cs.bytes(cols_bytes(hc, nc));
  }
  return cs.done(ghb_run_plan_body(ctx, in, input, ops, nops, out));
}

int32_t ghb_plan_result_free(ghb_plan_result* r) {
  if (!r) return GHB_ERR_INVALID;
  for (int c = 0; c < GHB_MAX_RESULT_COLS; c++) {
    std::free(r->data[c]);
    std::free(r->is_null[c]);
    std::free(r->str_bytes[c]);
    r->data[c] = nullptr;
    r->is_null[c] = nullptr;
    r->str_bytes[c] = nullptr;
    r->str_nbytes[c] = 0;
  }
  r->ncols = 0;
  r->rows = 0;
  return GHB_OK;
}

}  // extern "C"
