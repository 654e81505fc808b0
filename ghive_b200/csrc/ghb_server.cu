// ghb_server.cu — a long-lived operator server: requests from many host
// threads, admitted by free execution slots and HBM budget, run concurrently.
//
// GHive's JNI entry point (GPUProcess, gpu_impl/src/ghive_JNIInterface.cu:
// 13-340) runs one Tez task's operator plan at a time and keeps no device
// state between calls.  Here:
//
//   slots      each slot owns a context (scratch, status word, group-by table)
//              and a CUDA stream, and a worker thread that runs one request at
//              a time on them; N slots = N requests overlapping on the GPU.
//   admission  a request waits in a FIFO queue until a slot is idle and its
//              footprint (its outputs plus the working memory the operator
//              will use) fits the HBM budget; a request that does not fit
//              lets later, smaller ones pass unless it has waited longer than
//              kStarveNs, after which it goes first.  Admission runs when a
//              request is submitted and whenever one finishes, so requests
//              join the running set continuously.
//   residency  join build tables are registered once and probed by any slot;
//              the slot contexts keep their scratch arenas (they grow with
//              stream-ordered allocation, never with a device-wide sync).
//   results    outputs are carved from one stream-ordered allocation per
//              request and stay valid until the caller releases the ticket.
#include <time.h>

#include <algorithm>
#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "ghb_groupby.cuh"

namespace ghb {
size_t sort_scratch_bytes(int64_t n);
size_t join_probe_scratch_bytes(int64_t n);
}  // namespace ghb

using namespace ghb;

namespace {

constexpr int64_t kStarveNs = 20'000'000;   // 20 ms

int64_t now_ns() {
  timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (int64_t)ts.tv_sec * 1000000000ll + ts.tv_nsec;
}

int32_t agg_result_type(int32_t agg, int32_t in_type) {
  if (agg == GHB_AGG_CNT) return GHB_LONG;
  if (agg == GHB_AGG_AVG) return GHB_DOUBLE;
  if (agg == GHB_AGG_SUM) return in_type == GHB_DOUBLE ? GHB_DOUBLE : GHB_LONG;
  return in_type;
}

struct Req {
  uint64_t ticket = 0;
  int32_t op = 0;
  std::vector<ghb_column> cols;
  std::vector<ghb_pred_node> nodes;
  ghb_predicate pred{};
  bool has_pred = false;
  std::vector<int32_t> idx, orders, null_orders;
  std::vector<ghb_agg_desc> aggs;
  int64_t max_groups = 0;
  int32_t table = -1, join_type = 0, nkeys = 0, want_rowid = 0;
  int64_t n = 0;
  // outputs: one block, carved
  std::vector<int32_t> out_types;
  std::vector<bool> out_nulls;
  int64_t out_rows = 0;          // capacity in rows
  size_t out_bytes = 0, work_bytes = 0;
  void* block = nullptr;
  ghb_result res{};
  bool admitted = false, done = false;
};

struct Table {
  ghb_join_table* t = nullptr;
  std::vector<int32_t> pay_types;
  std::vector<bool> pay_nulls;
  int64_t max_dup = 1;
};

}  // namespace

struct ghb_server;

namespace {
struct Slot {
  int32_t id = 0;
  ghb_server* srv = nullptr;
  ghb_ctx* ctx = nullptr;
  cudaStream_t stream = nullptr;
  int64_t* pinned = nullptr;   // [0] row count, [1] device status
  Req* cur = nullptr;
  std::condition_variable cv;
  std::thread th;
};
}  // namespace

struct ghb_server {
  int device = 0;
  std::vector<std::unique_ptr<Slot>> slots;
  std::mutex mu;
  std::condition_variable cv_done;
  std::deque<Req*> queue;
  std::unordered_map<uint64_t, Req*> reqs;
  uint64_t next_ticket = 1;
  int64_t budget = 0, admitted_bytes = 0;
  int64_t completed = 0, running = 0;
  bool stop = false;
  std::vector<Table> tables;
  ghb_ctx* table_ctx = nullptr;
  cudaStream_t table_stream = nullptr;
  // Request outputs and the slots' working memory come from this pool, which
  // never makes one stream wait on another to reuse a block (it grows
  // instead); a released request's outputs are freed on free_stream, which
  // runs nothing, so the block is reusable at once rather than after whatever
  // its slot started next.
  cudaMemPool_t pool = nullptr;
  cudaStream_t free_stream = nullptr;
  std::string last_error;
};

namespace {

int32_t srv_error(ghb_server* s, int32_t code, const std::string& msg) {
  std::lock_guard<std::mutex> g(s->mu);
  s->last_error = msg;
  return code;
}

// Output layout and footprint of a request (host arithmetic only).
int32_t plan_outputs(ghb_server* s, Req* q, std::string* err) {
  const int64_t n = q->n;
  switch (q->op) {
    case GHB_OP_FILTER: {
      if (q->idx.empty())
        for (int i = 0; i < (int)q->cols.size(); i++) q->idx.push_back(i);
      for (int32_t j : q->idx) {
        if (j < 0 || j >= (int)q->cols.size()) return *err = "projection index out of range", GHB_ERR_INVALID;
        q->out_types.push_back(q->cols[j].type);
        q->out_nulls.push_back(q->cols[j].null_mode != GHB_NULLS_NONE);
      }
      q->out_rows = n;
      q->work_bytes = (size_t)(n / 2048 + 1) * 8 + (1 << 16);
      break;
    }
    case GHB_OP_GROUPBY: {
      if (q->idx.size() > (size_t)kMaxPackKeys) return *err = "too many group-by key columns", GHB_ERR_UNSUPPORTED;
      for (int32_t k : q->idx) {
        if (k < 0 || k >= (int)q->cols.size()) return *err = "key column out of range", GHB_ERR_INVALID;
        q->out_types.push_back(q->cols[k].type);
        q->out_nulls.push_back(true);
      }
      for (const ghb_agg_desc& a : q->aggs) {
        int32_t in = (a.col >= 0 && a.col < (int)q->cols.size()) ? q->cols[a.col].type : GHB_LONG;
        q->out_types.push_back(agg_result_type(a.type, in));
        q->out_nulls.push_back(true);
      }
      int64_t g = q->idx.empty() ? 1 : std::max<int64_t>(1, q->max_groups > 0 ? q->max_groups : n);
      q->out_rows = g;
      int64_t C = next_pow2_i64(std::max<int64_t>(2 * std::min<int64_t>(g, std::max<int64_t>(n, 1)) + 1, 64));
      q->work_bytes = gb_table_bytes(C, 1 + 2 * (int32_t)q->aggs.size() + 1);
      if (q->idx.size() > 1) q->work_bytes += keypack_scratch_bytes(n, g);   // the packed keys
      break;
    }
    case GHB_OP_JOIN_PROBE: {
      if (q->table < 0 || q->table >= (int)s->tables.size()) return *err = "unknown join table", GHB_ERR_INVALID;
      if (q->cols.size() != 1) return *err = "a probe request has one column (the probe key)", GHB_ERR_INVALID;
      const Table& t = s->tables[q->table];
      for (size_t j = 0; j < t.pay_types.size(); j++) {
        q->out_types.push_back(t.pay_types[j]);
        q->out_nulls.push_back(t.pay_nulls[j] || q->join_type == GHB_LEFT_OUTER_JOIN);
      }
      q->out_rows = n * (q->join_type == GHB_LEFT_SEMI_JOIN ? 1 : std::max<int64_t>(1, t.max_dup));
      q->work_bytes = join_probe_scratch_bytes(n);
      break;
    }
    case GHB_OP_SORT: {
      if (q->nkeys < 1 || q->nkeys > (int)q->cols.size()) return *err = "nkeys out of range", GHB_ERR_INVALID;
      for (const ghb_column& c : q->cols) {
        q->out_types.push_back(c.type);
        q->out_nulls.push_back(c.null_mode == GHB_NULLS_BYTEMAP);
      }
      q->out_rows = n;
      q->work_bytes = sort_scratch_bytes(n);
      break;
    }
    default:
      return *err = "unknown operator", GHB_ERR_INVALID;
  }
  if (q->out_types.size() > GHB_MAX_RESULT_COLS) return *err = "too many result columns", GHB_ERR_UNSUPPORTED;
  const int64_t rows = std::max<int64_t>(q->out_rows, 1);
  size_t b = 256;  // row count
  for (size_t j = 0; j < q->out_types.size(); j++) {
    b += ((size_t)rows * type_width(q->out_types[j]) + 255) & ~(size_t)255;
    if (q->out_nulls[j]) b += ((size_t)rows + 255) & ~(size_t)255;
  }
  const bool rowid = q->op == GHB_OP_JOIN_PROBE || (q->op == GHB_OP_SORT && q->want_rowid);
  const bool rowid2 = q->op == GHB_OP_JOIN_PROBE && q->want_rowid;
  if (rowid) b += ((size_t)rows * 4 + 255) & ~(size_t)255;
  if (rowid2) b += ((size_t)rows * 4 + 255) & ~(size_t)255;
  q->out_bytes = b;
  return GHB_OK;
}

int64_t footprint(const Req* q) { return (int64_t)(q->out_bytes + q->work_bytes); }

// Called with mu held: hands queued requests to idle slots while they fit.
void try_admit(ghb_server* s) {
  const int64_t t = now_ns();
  for (auto it = s->queue.begin(); it != s->queue.end();) {
    Slot* idle = nullptr;
    for (auto& sl : s->slots)
      if (!sl->cur) {
        idle = sl.get();
        break;
      }
    if (!idle) return;
    Req* q = *it;
    const int64_t need = footprint(q);
    // With nothing running a request is admitted whatever the budget says:
    // a request larger than the budget runs alone, and outputs that callers
    // have not released yet cannot hold the queue back for good.
    const bool fits = s->admitted_bytes + need <= s->budget || s->running == 0;
    if (fits) {
      it = s->queue.erase(it);
      s->admitted_bytes += need;
      q->admitted = true;
      q->res.admit_ns = t;
      q->res.slot = idle->id;
      s->running++;
      idle->cur = q;
      idle->cv.notify_one();
      continue;
    }
    // the oldest request that does not fit holds the rest back once it starves
    if (t - q->res.submit_ns > kStarveNs) return;
    ++it;
  }
}

// Runs request q on slot sl (slot thread, no lock held).
void execute(ghb_server* s, Slot* sl, Req* q) {
  ghb_ctx* ctx = sl->ctx;
  cudaStream_t st = sl->stream;
  ghb_result& r = q->res;
  int32_t rc = GHB_OK;
  if (cudaMallocFromPoolAsync(&q->block, q->out_bytes, s->pool, st) != cudaSuccess) {
    cudaGetLastError();
    q->block = nullptr;
    rc = GHB_ERR_OOM;
  }
  int64_t* d_count = (int64_t*)q->block;
  if (rc == GHB_OK) {
    // carve the outputs
    char* p = (char*)q->block + 256;
    const int64_t rows = std::max<int64_t>(q->out_rows, 1);
    r.ncols = (int32_t)q->out_types.size();
    for (size_t j = 0; j < q->out_types.size(); j++) {
      ghb_out_column& o = r.cols[j];
      o.type = q->out_types[j];
      o.data = p;
      p += ((size_t)rows * type_width(o.type) + 255) & ~(size_t)255;
      o.is_null = nullptr;
      if (q->out_nulls[j]) {
        o.is_null = (uint8_t*)p;
        p += ((size_t)rows + 255) & ~(size_t)255;
      }
    }
    const bool rowid = q->op == GHB_OP_JOIN_PROBE || (q->op == GHB_OP_SORT && q->want_rowid);
    const bool rowid2 = q->op == GHB_OP_JOIN_PROBE && q->want_rowid;
    r.rowid = rowid ? (int32_t*)p : nullptr;
    if (rowid) p += ((size_t)rows * 4 + 255) & ~(size_t)255;
    r.rowid2 = rowid2 ? (int32_t*)p : nullptr;
    const ghb_predicate* pred = q->has_pred ? &q->pred : nullptr;
    const int32_t nc = (int32_t)q->cols.size();
    switch (q->op) {
      case GHB_OP_FILTER:
        rc = ghb_filter(ctx, pred, q->cols.data(), nc, q->idx.data(), (int32_t)q->idx.size(), r.cols,
                        q->out_rows, d_count, st);
        break;
      case GHB_OP_GROUPBY: {
        ghb_groupby_cfg cfg{};
        cfg.max_groups = q->out_rows;
        rc = ghb_filter_groupby(ctx, pred, q->cols.data(), nc, q->idx.data(), (int32_t)q->idx.size(),
                                q->aggs.data(), (int32_t)q->aggs.size(), r.cols, q->out_rows, d_count,
                                &cfg, st);
        break;
      }
      case GHB_OP_JOIN_PROBE:
        rc = ghb_join_probe(ctx, s->tables[q->table].t, &q->cols[0], q->join_type, r.cols, nullptr, 0,
                            nullptr, r.rowid, r.rowid2, q->out_rows, d_count, st);
        break;
      case GHB_OP_SORT: {
        const int32_t nk = q->nkeys;
        rc = ghb_sort(ctx, q->cols.data(), q->orders.empty() ? nullptr : q->orders.data(),
                      q->null_orders.empty() ? nullptr : q->null_orders.data(), nk, q->cols.data() + nk,
                      nc - nk, r.cols, r.cols + nk, r.rowid, nullptr, st);
        break;
      }
    }
  }
  r.launched_ns = now_ns();
  if (rc == GHB_OK) {
    cudaMemcpyAsync(&sl->pinned[0], d_count, 8, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(&sl->pinned[1], ctx->d_status, 4, cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) {
      cudaGetLastError();
      rc = GHB_ERR_CUDA;
    } else {
      const int32_t dev = (int32_t)(sl->pinned[1] & 0xffffffff);
      r.rows = q->op == GHB_OP_SORT ? q->n : sl->pinned[0];
      if (dev) {
        // the status word is per slot: clear it for the next request
        cudaMemsetAsync(ctx->d_status, 0, sizeof(int32_t), st);
        ctx->gb_dirty = true;
        rc = dev;
      }
    }
  } else {
    std::lock_guard<std::mutex> g(s->mu);
    s->last_error = ghb_last_error(ctx);
  }
  r.status = rc;
  r.done_ns = now_ns();
}

void slot_loop(ghb_server* s, Slot* sl) {
  cudaSetDevice(s->device);
  std::unique_lock<std::mutex> lk(s->mu);
  for (;;) {
    sl->cv.wait(lk, [&] { return sl->cur != nullptr || s->stop; });
    if (!sl->cur) return;   // stopping and idle
    Req* q = sl->cur;
    lk.unlock();
    execute(s, sl, q);
    lk.lock();
    q->done = true;
    s->admitted_bytes -= (int64_t)q->work_bytes;   // outputs stay until release
    s->running--;
    s->completed++;
    sl->cur = nullptr;
    try_admit(s);
    s->cv_done.notify_all();
  }
}

}  // namespace

extern "C" int32_t ghb_server_create(int32_t device, const ghb_server_cfg* cfg, ghb_server** out) {
  if (!out) return GHB_ERR_INVALID;
  *out = nullptr;
  if (cudaSetDevice(device) != cudaSuccess) {
    cudaGetLastError();
    return GHB_ERR_CUDA;
  }
  ghb_server* s = new ghb_server();
  s->device = device;
  const int nslots = (cfg && cfg->slots > 0) ? std::min(cfg->slots, 64) : 8;
  size_t free_b = 0, total_b = 0;
  cudaMemGetInfo(&free_b, &total_b);
  s->budget = (cfg && cfg->hbm_budget > 0) ? cfg->hbm_budget : (int64_t)(free_b * 0.4);
  int32_t st = ghb_ctx_create(device, 0, &s->table_ctx);
  if (st == GHB_OK && (cudaStreamCreateWithFlags(&s->table_stream, cudaStreamNonBlocking) != cudaSuccess ||
                       cudaStreamCreateWithFlags(&s->free_stream, cudaStreamNonBlocking) != cudaSuccess))
    st = GHB_ERR_CUDA;
  if (st == GHB_OK) {
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    int no = 0;
    uint64_t keep = UINT64_MAX;
    if (cudaMemPoolCreate(&s->pool, &props) != cudaSuccess ||
        cudaMemPoolSetAttribute(s->pool, cudaMemPoolReuseAllowInternalDependencies, &no) != cudaSuccess ||
        cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep) != cudaSuccess) {
      cudaGetLastError();
      st = GHB_ERR_CUDA;
    }
  }
  if (st == GHB_OK) {
    // Map the whole budget into the pool now: growing a pool maps physical
    // memory under a driver lock, which stalls every other slot's calls
    // while it runs.
    void* p = nullptr;
    if (cudaMallocFromPoolAsync(&p, (size_t)s->budget, s->pool, s->table_stream) != cudaSuccess ||
        cudaFreeAsync(p, s->table_stream) != cudaSuccess ||
        cudaStreamSynchronize(s->table_stream) != cudaSuccess) {
      cudaGetLastError();
      st = GHB_ERR_OOM;
    }
  }
  for (int i = 0; i < nslots && st == GHB_OK; i++) {
    auto sl = std::make_unique<Slot>();
    sl->srv = s;
    sl->id = i;
    st = ghb_ctx_create(device, 0, &sl->ctx);
    if (st) break;
    sl->ctx->stream_ordered = true;
    sl->ctx->pool = s->pool;
    if (cudaStreamCreateWithFlags(&sl->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMallocHost((void**)&sl->pinned, 16) != cudaSuccess) {
      cudaGetLastError();
      st = GHB_ERR_CUDA;
      s->slots.push_back(std::move(sl));
      break;
    }
    s->slots.push_back(std::move(sl));
  }
  if (st == GHB_OK) {
    for (auto& sl : s->slots) sl->th = std::thread(slot_loop, s, sl.get());
    *out = s;
    return GHB_OK;
  }
  ghb_server_destroy(s);
  return st;
}

extern "C" int32_t ghb_server_add_join_table(ghb_server* s, const ghb_column* build_key,
                                             const ghb_column* payload, int32_t npayload, float load_factor,
                                             int32_t* table_id) {
  if (!s || !build_key || !table_id) return GHB_ERR_INVALID;
  cudaSetDevice(s->device);
  ghb_join_cfg cfg{};
  cfg.load_factor = load_factor;
  Table t;
  int32_t st = ghb_join_build(s->table_ctx, build_key, payload, npayload, &cfg, &t.t, s->table_stream);
  if (st == GHB_OK) st = ghb_sync(s->table_ctx, s->table_stream);
  int64_t rows = 0, dup = 0, slots = 0;
  if (st == GHB_OK) st = ghb_join_table_info(s->table_ctx, t.t, &rows, &dup, &slots);
  if (st) {
    std::string e = ghb_last_error(s->table_ctx);
    if (t.t) ghb_join_table_free(s->table_ctx, t.t);
    return srv_error(s, st, e);
  }
  t.max_dup = std::max<int64_t>(1, dup);
  for (int j = 0; j < npayload; j++) {
    t.pay_types.push_back(payload[j].type);
    t.pay_nulls.push_back(payload[j].null_mode != GHB_NULLS_NONE);
  }
  std::lock_guard<std::mutex> g(s->mu);
  s->tables.push_back(t);
  *table_id = (int32_t)s->tables.size() - 1;
  return GHB_OK;
}

extern "C" int32_t ghb_server_submit(ghb_server* s, const ghb_request* r, uint64_t* ticket) {
  if (!s || !r || !ticket) return GHB_ERR_INVALID;
  auto q = std::make_unique<Req>();
  q->op = r->op;
  if (r->ncols < 0 || r->ncols > kMaxCols || (r->ncols > 0 && !r->cols))
    return srv_error(s, GHB_ERR_INVALID, "bad column list");
  q->cols.assign(r->cols, r->cols + r->ncols);
  q->n = r->ncols ? r->cols[0].n : 0;
  if (r->pred && r->pred->n_nodes > 0) {
    if (r->pred->n_nodes > GHB_MAX_PRED_NODES || !r->pred->nodes)
      return srv_error(s, GHB_ERR_INVALID, "bad predicate");
    q->nodes.assign(r->pred->nodes, r->pred->nodes + r->pred->n_nodes);
    q->pred = *r->pred;
    q->pred.nodes = q->nodes.data();
    q->has_pred = true;
  }
  if (r->idx && r->nidx > 0) q->idx.assign(r->idx, r->idx + r->nidx);
  if (r->aggs && r->naggs > 0) q->aggs.assign(r->aggs, r->aggs + r->naggs);
  q->max_groups = r->max_groups;
  q->table = r->table;
  q->join_type = r->join_type;
  q->nkeys = r->nkeys;
  q->want_rowid = r->want_rowid;
  if (r->op == GHB_OP_SORT && r->nkeys > 0) {
    if (r->orders) q->orders.assign(r->orders, r->orders + r->nkeys);
    if (r->null_orders) q->null_orders.assign(r->null_orders, r->null_orders + r->nkeys);
  }
  std::string err;
  int32_t st;
  {
    std::lock_guard<std::mutex> g(s->mu);
    st = plan_outputs(s, q.get(), &err);
    if (st) {
      s->last_error = err;
      return st;
    }
    q->ticket = s->next_ticket++;
    q->res.submit_ns = now_ns();
    *ticket = q->ticket;
    Req* raw = q.release();
    s->reqs[raw->ticket] = raw;
    s->queue.push_back(raw);
    try_admit(s);
  }
  return GHB_OK;
}

extern "C" int32_t ghb_server_wait(ghb_server* s, uint64_t ticket, ghb_result* out) {
  if (!s || !out) return GHB_ERR_INVALID;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->reqs.find(ticket);
  if (it == s->reqs.end()) {
    s->last_error = "unknown ticket";
    return GHB_ERR_INVALID;
  }
  Req* q = it->second;
  s->cv_done.wait(lk, [&] { return q->done; });
  *out = q->res;
  return q->res.status;
}

extern "C" int32_t ghb_server_release(ghb_server* s, uint64_t ticket) {
  if (!s) return GHB_ERR_INVALID;
  Req* q = nullptr;
  {
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) {
      s->last_error = "unknown ticket";
      return GHB_ERR_INVALID;
    }
    q = it->second;
    s->cv_done.wait(lk, [&] { return q->done; });
    s->reqs.erase(it);
    s->admitted_bytes -= (int64_t)q->out_bytes;
    try_admit(s);
  }
  if (q->block) {
    cudaSetDevice(s->device);
    // the request is done: free on the idle stream, reusable immediately
    cudaFreeAsync(q->block, s->free_stream);
  }
  delete q;
  return GHB_OK;
}

extern "C" int32_t ghb_server_stats(ghb_server* s, int64_t* completed, int64_t* running, int64_t* queued,
                                    int64_t* bytes_admitted) {
  if (!s) return GHB_ERR_INVALID;
  std::lock_guard<std::mutex> g(s->mu);
  if (completed) *completed = s->completed;
  if (running) *running = s->running;
  if (queued) *queued = (int64_t)s->queue.size();
  if (bytes_admitted) *bytes_admitted = s->admitted_bytes;
  return GHB_OK;
}

extern "C" const char* ghb_server_last_error(ghb_server* s) {
  if (!s) return "null server";
  std::lock_guard<std::mutex> g(s->mu);
  return s->last_error.c_str();
}

extern "C" int32_t ghb_server_destroy(ghb_server* s) {
  if (!s) return GHB_OK;
  {
    std::unique_lock<std::mutex> lk(s->mu);
    // queued requests never run: finish them with an error so waiters return
    for (Req* q : s->queue) {
      q->res.status = GHB_ERR_INVALID;
      q->done = true;
    }
    s->queue.clear();
    s->cv_done.notify_all();
    // running requests finish first
    s->cv_done.wait(lk, [&] { return s->running == 0; });
    s->stop = true;
    for (auto& sl : s->slots) sl->cv.notify_all();
  }
  for (auto& sl : s->slots)
    if (sl->th.joinable()) sl->th.join();
  cudaSetDevice(s->device);
  cudaDeviceSynchronize();
  for (auto& kv : s->reqs) {
    if (kv.second->block) cudaFree(kv.second->block);
    delete kv.second;
  }
  for (Table& t : s->tables)
    if (t.t) ghb_join_table_free(s->table_ctx, t.t);
  for (auto& sl : s->slots) {
    if (sl->pinned) cudaFreeHost(sl->pinned);
    if (sl->stream) cudaStreamDestroy(sl->stream);
    if (sl->ctx) ghb_ctx_destroy(sl->ctx);
  }
  if (s->table_stream) cudaStreamDestroy(s->table_stream);
  if (s->free_stream) cudaStreamDestroy(s->free_stream);
  if (s->table_ctx) ghb_ctx_destroy(s->table_ctx);
  cudaDeviceSynchronize();
  if (s->pool) cudaMemPoolDestroy(s->pool);
  delete s;
  return GHB_OK;
}
