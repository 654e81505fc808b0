// ghb_host_api.cu — operator calls on HOST columns (the end-to-end path).
//
// One call does what one GHive operator call did on host `Column`s
// (FilterPredicate.cu:173 device_vector(h_ptr...), GroupByPredicate.cu:39-91
// cudaMalloc+cudaMemcpy per column, SinkOperator.cu:153-232): copy the
// inputs to the device, run the operator, copy the result back.  Here the
// copies are cudaMemcpyAsync on the context's stream (DMA straight from
// pinned memory, staged by the driver from pageable memory), the device
// buffers come from the context's scratch arena (no cudaMalloc per call once
// the arena has grown), and only the result rows travel back.
#include <algorithm>
#include <vector>

#include "ghb_ctx.hpp"
#include "ghb_log.hpp"

namespace ghb {

int32_t filter_impl(ghb_ctx*, const ghb_predicate*, const ghb_column*, int32_t, const int32_t*,
                    int32_t, ghb_out_column*, int64_t, int64_t*, cudaStream_t);
int32_t filter_groupby_impl(ghb_ctx*, const ghb_predicate*, const ghb_column*, int32_t,
                            const int32_t*, int32_t, const ghb_agg_desc*, int32_t, ghb_out_column*,
                            int64_t, int64_t*, const ghb_groupby_cfg*, cudaStream_t, void*, size_t);
int32_t join_build_impl(ghb_ctx*, const ghb_column*, const ghb_column*, int32_t,
                        const ghb_join_cfg*, ghb_join_table**, cudaStream_t);
int32_t join_probe_impl(ghb_ctx*, const ghb_join_table*, const ghb_column*, int32_t,
                        ghb_out_column*, const ghb_column*, int32_t, ghb_out_column*, int32_t*,
                        int32_t*, int64_t, int64_t*, cudaStream_t, int32_t);
int32_t sort_impl(ghb_ctx*, const ghb_column*, const int32_t*, const int32_t*, int32_t,
                  const ghb_column*, int32_t, ghb_out_column*, ghb_out_column*, int32_t*,
                  const ghb_sort_cfg*, cudaStream_t);
size_t sort_scratch_bytes(int64_t n);
size_t join_probe_scratch_bytes(int64_t n);

namespace {

size_t col_bytes(const ghb_column& c) { return (size_t)c.n * type_width(c.type); }
size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }
size_t in_bytes(const ghb_column& c) {
  return align256(col_bytes(c)) + (c.null_mode == GHB_NULLS_BYTEMAP ? align256((size_t)c.n) : 0);
}
size_t out_bytes(const ghb_out_column& o, int64_t cap) {
  return align256((size_t)cap * type_width(o.type)) + (o.is_null ? align256((size_t)cap) : 0);
}

// Copies host columns into scratch and returns device descriptors.
int32_t stage_in(ghb_ctx* ctx, const ghb_column* h, int32_t n, std::vector<ghb_column>& d,
                 cudaStream_t s) {
  d.assign(h, h + n);
  std::vector<CopyTask> copies;
  for (int i = 0; i < n; i++) {
    if (h[i].type == GHB_STRING)
      return set_error(ctx, GHB_ERR_UNSUPPORTED, "STRING columns are not on the device path");
    void* p = nullptr;
    int32_t st = scratch_alloc(ctx, std::max<size_t>(col_bytes(h[i]), 16), &p, s);
    if (st) return st;
    if (h[i].n > 0) {
      if (!h[i].data) return set_error(ctx, GHB_ERR_INVALID, "column %d: data is NULL", i);
      copies.push_back({p, h[i].data, col_bytes(h[i])});
    }
    d[i].data = p;
    if (h[i].null_mode == GHB_NULLS_BYTEMAP && h[i].n > 0) {
      if (!h[i].is_null) return set_error(ctx, GHB_ERR_INVALID, "column %d: is_null is NULL", i);
      void* q = nullptr;
      st = scratch_alloc(ctx, (size_t)h[i].n, &q, s);
      if (st) return st;
      copies.push_back({q, h[i].is_null, (size_t)h[i].n});
      d[i].is_null = (const uint8_t*)q;
    }
  }
  return copy_h2d_many(ctx, copies, s);
}

int32_t stage_out(ghb_ctx* ctx, const ghb_out_column* h, int32_t n, int64_t cap,
                  std::vector<ghb_out_column>& d, cudaStream_t s) {
  d.assign(h, h + n);
  for (int i = 0; i < n; i++) {
    void* p = nullptr;
    int32_t st = scratch_alloc(ctx, std::max<size_t>((size_t)cap * type_width(h[i].type), 16), &p, s);
    if (st) return st;
    d[i].data = p;
    if (h[i].is_null) {
      void* q = nullptr;
      st = scratch_alloc(ctx, std::max<size_t>((size_t)cap, 16), &q, s);
      if (st) return st;
      d[i].is_null = (uint8_t*)q;
    }
  }
  return GHB_OK;
}

// The first `rows` rows of the device outputs into the caller's host outputs
// (pageable ones through the staging lanes); returns when they are there.
int32_t copy_back(ghb_ctx* ctx, const ghb_out_column* h, const std::vector<ghb_out_column>& d,
                  int64_t rows, cudaStream_t s) {
  std::vector<CopyTask> copies;
  for (size_t i = 0; i < d.size() && rows > 0; i++) {
    copies.push_back({h[i].data, d[i].data, (size_t)rows * type_width(h[i].type)});
    if (h[i].is_null) copies.push_back({h[i].is_null, d[i].is_null, (size_t)rows});
  }
  return copy_d2h_many(ctx, copies, s);
}

// Reads a device int64 counter and the device status after the stream drains.
int32_t read_count(ghb_ctx* ctx, const int64_t* d_count, int64_t* out, cudaStream_t s) {
  int64_t v = 0;
  GHB_CUDA_TRY(ctx, cudaMemcpyAsync(&v, d_count, sizeof(v), cudaMemcpyDeviceToHost, s));
  int32_t st = ghb_sync(ctx, s);
  *out = v;
  return st;
}

// The context's three host-path streams (copy in, kernels, copy out) and
// their per-buffer events, made on first use.
int32_t host_streams(ghb_ctx* ctx) {
  for (int i = 0; i < 3; i++)
    if (!ctx->hstream[i]) GHB_CUDA_TRY(ctx, cudaStreamCreateWithFlags(&ctx->hstream[i], cudaStreamNonBlocking));
  for (auto& row : ctx->hev)
    for (cudaEvent_t& e : row)
      if (!e) GHB_CUDA_TRY(ctx, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  return GHB_OK;
}

// At least `bytes` of pinned host memory at ctx->pinned.
int32_t ensure_pinned(ghb_ctx* ctx, size_t bytes) {
  if (ctx->pinned_bytes >= bytes) return GHB_OK;
  if (ctx->pinned) cudaFreeHost(ctx->pinned);
  ctx->pinned = nullptr;
  ctx->pinned_bytes = 0;
  if (cudaMallocHost(&ctx->pinned, std::max<size_t>(bytes, 4096)) != cudaSuccess) {
    cudaGetLastError();
    return set_error(ctx, GHB_ERR_OOM, "cannot allocate pinned host memory");
  }
  ctx->pinned_bytes = std::max<size_t>(bytes, 4096);
  return GHB_OK;
}

// Rows of one chunk of the pipelined filter: about a twelfth of the input
// (so the first chunk's copy, which nothing overlaps, is short), in whole
// 2048-row tiles, between 512Ki and 8Mi rows.
int64_t filter_chunk_rows(int64_t n) {
  const int64_t c = std::min<int64_t>(8 << 20, std::max<int64_t>(512 << 10, (n + 11) / 12));
  return (c + 2047) / 2048 * 2048;
}

// True when every buffer the filter reads or writes on the host is pinned,
// so its copies can run asynchronously chunk by chunk.
bool filter_host_pinned(const ghb_column* cols, int32_t ncols, const ghb_out_column* out, int32_t nproj) {
  for (int i = 0; i < ncols; i++) {
    if (!cols[i].data || !host_pinned(cols[i].data)) return false;
    if (cols[i].null_mode == GHB_NULLS_BYTEMAP && (!cols[i].is_null || !host_pinned(cols[i].is_null))) return false;
  }
  for (int j = 0; j < nproj; j++) {
    if (!out[j].data || !host_pinned(out[j].data)) return false;
    if (out[j].is_null && !host_pinned(out[j].is_null)) return false;
  }
  return true;
}
// The filter over pinned host columns, in chunks of rows through three
// streams: a chunk's columns are copied in while the one before is filtered
// and the one before that is copied out, so the copies in both directions
// overlap each other and the kernels.  Each chunk is filtered into one of
// two device output buffers (a chunk's output is at most its rows); its row
// count comes back before its copy-out is issued, and the chunks' outputs
// are appended in chunk order, which is the filter's row order.
int32_t filter_host_chunked(ghb_ctx* ctx, const ghb_predicate* pred, const ghb_column* cols, int32_t ncols,
                            const int32_t* proj, int32_t nproj, ghb_out_column* out, int64_t out_capacity,
                            int64_t n, int64_t* out_rows) {
  int32_t st = host_streams(ctx);
  if (st) return st;
  cudaStream_t s_in = ctx->hstream[0], s_k = ctx->hstream[1], s_out = ctx->hstream[2];
  // the calling thread's legacy default stream may hold work on these buffers
  GHB_CUDA_TRY(ctx, cudaStreamSynchronize(0));
  const int64_t chunk = filter_chunk_rows(n);
  const int64_t nchunks = (n + chunk - 1) / chunk;
  size_t need = 4096;
  for (int i = 0; i < ncols; i++) {
    need += 2 * (align256((size_t)chunk * type_width(cols[i].type)) + 256);
    if (cols[i].null_mode == GHB_NULLS_BYTEMAP) need += 2 * (align256((size_t)chunk) + 256);
  }
  for (int j = 0; j < nproj; j++) need += 2 * (out_bytes(out[j], chunk) + 512);
  if ((st = scratch_reserve(ctx, need, s_in))) return st;
  if ((st = ensure_pinned(ctx, (size_t)nchunks * 8))) return st;
  int64_t* h_rows = (int64_t*)ctx->pinned;   // each chunk's row count
  struct Slot {
    std::vector<ghb_column> in;
    std::vector<ghb_out_column> out;
    int64_t* d_rows = nullptr;
  } slot[2];
  for (int b = 0; b < 2; b++) {
    Slot& sl = slot[b];
    sl.in.assign(cols, cols + ncols);
    for (int i = 0; i < ncols; i++) {
      void* q = nullptr;
      if ((st = scratch_alloc(ctx, std::max<size_t>((size_t)chunk * type_width(cols[i].type), 16), &q, s_in)))
        return st;
      sl.in[i].data = q;
      if (cols[i].null_mode == GHB_NULLS_BYTEMAP) {
        if ((st = scratch_alloc(ctx, std::max<size_t>((size_t)chunk, 16), &q, s_in))) return st;
        sl.in[i].is_null = (const uint8_t*)q;
      }
    }
    if ((st = stage_out(ctx, out, nproj, chunk, sl.out, s_in))) return st;
    if ((st = scratch_alloc(ctx, 8, (void**)&sl.d_rows, s_in))) return st;
  }
  cudaEvent_t* ev_in = ctx->hev[0];     // chunk copied in (per buffer)
  cudaEvent_t* ev_filt = ctx->hev[1];   // chunk filtered: its input buffer is free
  cudaEvent_t* ev_rows = ctx->hev[2];   // chunk's row count on the host side
  cudaEvent_t* ev_out = ctx->hev[3];    // chunk copied out: its output buffer is free
  auto fail = [&](int32_t code) {
    cudaStreamSynchronize(s_in);
    cudaStreamSynchronize(s_k);
    cudaStreamSynchronize(s_out);
    return code;
  };
  int64_t total = 0, written = 0;
  auto copy_out = [&](int64_t c) -> int32_t {
    const int b = (int)(c & 1);
    const Slot& sl = slot[b];
    GHB_CUDA_TRY(ctx, cudaEventSynchronize(ev_rows[b]));
    const int64_t rows = h_rows[c];
    total += rows;
    const int64_t r = std::max<int64_t>(0, std::min<int64_t>(rows, out_capacity - written));
    GHB_CUDA_TRY(ctx, cudaStreamWaitEvent(s_out, ev_rows[b], 0));
    for (int j = 0; j < nproj && r > 0; j++) {
      const size_t w = type_width(out[j].type);
      GHB_CUDA_TRY(ctx, cudaMemcpyAsync((char*)out[j].data + written * w, sl.out[j].data, r * w,
                                        cudaMemcpyDeviceToHost, s_out));
      if (out[j].is_null)
        GHB_CUDA_TRY(ctx, cudaMemcpyAsync(out[j].is_null + written, sl.out[j].is_null, r, cudaMemcpyDeviceToHost,
                                          s_out));
    }
    written += r;
    GHB_CUDA_TRY(ctx, cudaEventRecord(ev_out[b], s_out));
    return GHB_OK;
  };
  for (int64_t c = 0; c < nchunks; c++) {
    const int b = (int)(c & 1);
    Slot& sl = slot[b];
    const int64_t r0 = c * chunk, rows = std::min<int64_t>(chunk, n - r0);
    // copy in, once the filter of chunk c - 2 has read this buffer
    if (c >= 2) GHB_CUDA_TRY(ctx, cudaStreamWaitEvent(s_in, ev_filt[b], 0));
    for (int i = 0; i < ncols; i++) {
      const size_t w = type_width(cols[i].type);
      sl.in[i].n = rows;
      GHB_CUDA_TRY(ctx, cudaMemcpyAsync((void*)sl.in[i].data, (const char*)cols[i].data + r0 * w, rows * w,
                                        cudaMemcpyHostToDevice, s_in));
      if (cols[i].null_mode == GHB_NULLS_BYTEMAP)
        GHB_CUDA_TRY(ctx, cudaMemcpyAsync((void*)sl.in[i].is_null, cols[i].is_null + r0, rows,
                                          cudaMemcpyHostToDevice, s_in));
    }
    GHB_CUDA_TRY(ctx, cudaEventRecord(ev_in[b], s_in));
    // filter, once the chunk is in and chunk c - 2's output has been copied out
    GHB_CUDA_TRY(ctx, cudaStreamWaitEvent(s_k, ev_in[b], 0));
    if (c >= 2) GHB_CUDA_TRY(ctx, cudaStreamWaitEvent(s_k, ev_out[b], 0));
    st = filter_impl(ctx, pred, sl.in.data(), ncols, proj, nproj, sl.out.data(), rows, sl.d_rows, s_k);
    if (st) return fail(st);
    GHB_CUDA_TRY(ctx, cudaEventRecord(ev_filt[b], s_k));
    GHB_CUDA_TRY(ctx, cudaMemcpyAsync(&h_rows[c], sl.d_rows, 8, cudaMemcpyDeviceToHost, s_k));
    GHB_CUDA_TRY(ctx, cudaEventRecord(ev_rows[b], s_k));
    // the previous chunk's output goes out while this one is filtered
    if (c >= 1 && (st = copy_out(c - 1))) return fail(st);
  }
  if (nchunks >= 1 && (st = copy_out(nchunks - 1))) return fail(st);
  GHB_CUDA_TRY(ctx, cudaStreamSynchronize(s_out));
  GHB_CUDA_TRY(ctx, cudaStreamSynchronize(s_in));
  st = ghb_sync(ctx, s_k);   // device status of every chunk's kernel
  *out_rows = total;
  if (st) return st;
  if (total > out_capacity) return set_error(ctx, GHB_ERR_CAPACITY, "output or table capacity exceeded");
  return GHB_OK;
}

}  // namespace
}  // namespace ghb

using namespace ghb;

extern "C" {

static int32_t ghb_filter_host_body(ghb_ctx* ctx, const ghb_predicate* pred, const ghb_column* cols,
                        int32_t ncols, const int32_t* proj, int32_t nproj, ghb_out_column* out,
                        int64_t out_capacity, int64_t* out_rows) {
  if (!ctx || !out_rows) return GHB_ERR_INVALID;
  cudaStream_t s = 0;
  scratch_reset(ctx);
  int64_t n = 0;
  int32_t st = validate_columns(ctx, cols, ncols, &n);
  if (st) return st;
  if (nproj < 0 || nproj > kMaxCols || (nproj > 0 && (!proj || !out)))
    return set_error(ctx, GHB_ERR_INVALID, "bad projection list");
  if (out_capacity < 0) return set_error(ctx, GHB_ERR_INVALID, "negative out_capacity");
  for (int j = 0; j < nproj; j++)
    if (proj[j] < 0 || proj[j] >= ncols) return set_error(ctx, GHB_ERR_INVALID, "projection %d out of range", j);
  if (n >= 2 * filter_chunk_rows(n) && filter_host_pinned(cols, ncols, out, nproj))
    return filter_host_chunked(ctx, pred, cols, ncols, proj, nproj, out, out_capacity, n, out_rows);
  size_t need = 4096 + align256(8);
  for (int i = 0; i < ncols; i++) need += in_bytes(cols[i]) + 256;
  for (int j = 0; j < nproj; j++) need += out_bytes(out[j], out_capacity) + 512;
  st = scratch_reserve(ctx, need, s);
  if (st) return st;
  std::vector<ghb_column> dc;
  std::vector<ghb_out_column> dout;
  int64_t* d_rows = nullptr;
  if ((st = scratch_alloc(ctx, 8, (void**)&d_rows, s))) return st;
  if ((st = stage_in(ctx, cols, ncols, dc, s))) return st;
  if ((st = stage_out(ctx, out, nproj, out_capacity, dout, s))) return st;
  st = filter_impl(ctx, pred, dc.data(), ncols, proj, nproj, dout.data(), out_capacity, d_rows, s);
  if (st) return st;
  int64_t rows = 0;
  st = read_count(ctx, d_rows, &rows, s);
  *out_rows = rows;
  if (st) return st;
  if ((st = copy_back(ctx, out, dout, std::min(rows, out_capacity), s))) return st;
  GHB_CUDA_TRY(ctx, cudaStreamSynchronize(s));
  return GHB_OK;
}

int32_t ghb_filter_host(ghb_ctx* ctx, const ghb_predicate* pred, const ghb_column* cols, int32_t ncols,
                        const int32_t* proj, int32_t nproj, ghb_out_column* out, int64_t out_capacity,
                        int64_t* out_rows) {
  CallScope cs(ctx, "filter_host", 0, true);
  cs.rows(ncols > 0 && cols ? cols[0].n : 0);
  cs.bytes(cols_bytes(cols, ncols));
  return cs.done(ghb_filter_host_body(ctx, pred, cols, ncols, proj, nproj, out, out_capacity, out_rows));
}

static int32_t ghb_filter_groupby_host_body(ghb_ctx* ctx, const ghb_predicate* pred, const ghb_column* cols,
                                int32_t ncols, const int32_t* key_cols, int32_t nkeys,
                                const ghb_agg_desc* aggs, int32_t naggs, ghb_out_column* out,
                                int64_t out_capacity, int64_t* out_groups,
                                const ghb_groupby_cfg* cfg) {
  if (!ctx || !out_groups) return GHB_ERR_INVALID;
  cudaStream_t s = 0;
  scratch_reset(ctx);
  int64_t n = 0;
  int32_t st = validate_columns(ctx, cols, ncols, &n);
  if (st) return st;
  if (nkeys < 0 || naggs < 0 || nkeys + naggs > 2 * kMaxCols || (nkeys + naggs > 0 && !out))
    return set_error(ctx, GHB_ERR_INVALID, "bad key/aggregate lists");
  size_t need = 4096;
  for (int i = 0; i < ncols; i++) need += in_bytes(cols[i]) + 256;
  for (int j = 0; j < nkeys + naggs; j++) need += out_bytes(out[j], out_capacity) + 512;
  if (nkeys > 1) need += keypack_scratch_bytes(n, out_capacity);
  st = scratch_reserve(ctx, need, s);
  if (st) return st;
  std::vector<ghb_column> dc;
  std::vector<ghb_out_column> dout;
  int64_t* d_groups = nullptr;
  if ((st = scratch_alloc(ctx, 8, (void**)&d_groups, s))) return st;
  if ((st = stage_in(ctx, cols, ncols, dc, s))) return st;
  if ((st = stage_out(ctx, out, nkeys + naggs, out_capacity, dout, s))) return st;
  st = filter_groupby_impl(ctx, pred, dc.data(), ncols, key_cols, nkeys, aggs, naggs, dout.data(),
                           out_capacity, d_groups, cfg, s, nullptr, 0);
  if (st) return st;
  int64_t g = 0;
  st = read_count(ctx, d_groups, &g, s);
  *out_groups = g;
  if (st) return st;
  if ((st = copy_back(ctx, out, dout, std::min(g, out_capacity), s))) return st;
  GHB_CUDA_TRY(ctx, cudaStreamSynchronize(s));
  return GHB_OK;
}

int32_t ghb_filter_groupby_host(ghb_ctx* ctx, const ghb_predicate* pred, const ghb_column* cols, int32_t ncols,
                                const int32_t* key_cols, int32_t nkeys, const ghb_agg_desc* aggs, int32_t naggs,
                                ghb_out_column* out, int64_t out_capacity, int64_t* out_groups,
                                const ghb_groupby_cfg* cfg) {
  CallScope cs(ctx, "filter_groupby_host", 0, true);
  cs.rows(ncols > 0 && cols ? cols[0].n : 0);
  cs.bytes(cols_bytes(cols, ncols));
  return cs.done(ghb_filter_groupby_host_body(ctx, pred, cols, ncols, key_cols, nkeys, aggs, naggs, out,
                                              out_capacity, out_groups, cfg));
}

static int32_t ghb_hash_join_host_body(ghb_ctx* ctx, const ghb_column* build_key, const ghb_column* probe_key,
                           int32_t join_type, const ghb_column* build_payload, int32_t nbp,
                           ghb_out_column* out_build, const ghb_column* probe_payload, int32_t npp,
                           ghb_out_column* out_probe, int32_t* out_probe_rowid,
                           int32_t* out_build_rowid, int64_t out_capacity, int64_t* out_rows,
                           const ghb_join_cfg* cfg) {
  if (!ctx || !out_rows || !build_key || !probe_key) return GHB_ERR_INVALID;
  if (nbp < 0 || nbp > GHB_MAX_JOIN_PAYLOAD || npp < 0 || npp > GHB_MAX_JOIN_PAYLOAD)
    return set_error(ctx, GHB_ERR_INVALID, "payload counts");
  if ((nbp > 0 && (!build_payload || !out_build)) || (npp > 0 && (!probe_payload || !out_probe)))
    return set_error(ctx, GHB_ERR_INVALID, "payload columns or their outputs are NULL");
  if (out_capacity < 0) return set_error(ctx, GHB_ERR_INVALID, "negative out_capacity");
  *out_rows = 0;
  scratch_reset(ctx);
  const int64_t n = probe_key->n;
  for (int j = 0; j < npp; j++)
    if (probe_payload[j].n != n)
      return set_error(ctx, GHB_ERR_INVALID, "probe payload %d row count differs from the key", j);
  if (n >= (int64_t)INT32_MAX) return set_error(ctx, GHB_ERR_UNSUPPORTED, "probe of 2^31 rows or more");
  int32_t st = host_streams(ctx);
  if (st) return st;
  cudaStream_t s_in = ctx->hstream[0], s_k = ctx->hstream[1], s_out = ctx->hstream[2];
  // the calling thread's legacy default stream may hold work on these
  // buffers: start after it
  GHB_CUDA_TRY(ctx, cudaStreamSynchronize(0));

  // The probe runs in chunks of rows, each through three streams: its key
  // (and payload) chunk is copied in while the previous chunk is probed and
  // the one before is copied out, so the copies in both directions overlap
  // each other and the kernels.  A chunk's output goes to one of two device
  // buffers; its row count comes back before its copy-out is issued.
  const int64_t kChunkRows = 8 << 20;
  const int64_t chunk = std::min<int64_t>(std::max<int64_t>(n, 1), kChunkRows);
  const int64_t nchunks = n == 0 ? 0 : (n + chunk - 1) / chunk;

  size_t need = 8192 + in_bytes(*build_key) + join_probe_scratch_bytes(n) + (size_t)nchunks * 256 * 2;
  for (int j = 0; j < nbp; j++) need += in_bytes(build_payload[j]) + 256;
  auto chunk_in = [&](int64_t rows) {
    size_t b = align256((size_t)rows * type_width(probe_key->type)) + 256;
    if (probe_key->null_mode == GHB_NULLS_BYTEMAP) b += align256((size_t)rows) + 256;
    for (int j = 0; j < npp; j++) {
      b += align256((size_t)rows * type_width(probe_payload[j].type)) + 256;
      if (probe_payload[j].null_mode == GHB_NULLS_BYTEMAP) b += align256((size_t)rows) + 256;
    }
    return b;
  };
  auto chunk_out = [&](int64_t rows) {
    size_t b = 0;
    for (int j = 0; j < nbp; j++) b += out_bytes(out_build[j], rows) + 256;
    for (int j = 0; j < npp; j++) b += out_bytes(out_probe[j], rows) + 256;
    if (out_probe_rowid) b += align256((size_t)rows * 4) + 256;
    if (out_build_rowid) b += align256((size_t)rows * 4) + 256;
    return b;
  };
  std::vector<ghb_column> dbk, dbp;
  if ((st = scratch_reserve(ctx, need + 2 * chunk_in(chunk), s_in))) return st;
  if ((st = stage_in(ctx, build_key, 1, dbk, s_in))) return st;
  if ((st = stage_in(ctx, build_payload, nbp, dbp, s_in))) return st;
  GHB_CUDA_TRY(ctx, cudaEventRecord(ctx->hev[0][0], s_in));
  GHB_CUDA_TRY(ctx, cudaStreamWaitEvent(s_k, ctx->hev[0][0], 0));
  ghb_join_table* t = nullptr;
  if ((st = join_build_impl(ctx, dbk.data(), dbp.data(), nbp, cfg, &t, s_k))) return st;
  // the output rows a chunk can make: its rows times the most build rows of
  // one key (one for a semi join, at least one for an outer join)
  int64_t max_dup = 1;
  {
    unsigned long long stats[2] = {0, 0};
    st = GHB_OK;
    if (cudaMemcpyAsync(stats, t->d_stats, sizeof(stats), cudaMemcpyDeviceToHost, s_k) != cudaSuccess ||
        cudaStreamSynchronize(s_k) != cudaSuccess)
      st = set_error(ctx, GHB_ERR_CUDA, "reading the join table's statistics failed");
    max_dup = std::max<int64_t>(1, (int64_t)stats[1]);
    if (join_type == GHB_LEFT_SEMI_JOIN) max_dup = 1;
    if (st) {
      ghb_join_table_free(ctx, t);
      return st;
    }
  }
  const int64_t out_chunk = std::min<int64_t>(chunk * max_dup, std::max<int64_t>(out_capacity, 1));
  struct Slot {
    std::vector<ghb_column> pk, pp;
    std::vector<ghb_out_column> ob, op;
    int32_t *prow = nullptr, *brow = nullptr;
    int64_t* d_rows = nullptr;
  } slot[2];
  int64_t* h_rows = nullptr;   // pinned: each chunk's row count
  if ((st = ensure_pinned(ctx, (size_t)std::max<int64_t>(nchunks, 1) * 8))) {
    ghb_join_table_free(ctx, t);
    return st;
  }
  h_rows = (int64_t*)ctx->pinned;
  auto fail = [&](int32_t code) {
    cudaStreamSynchronize(s_in);
    cudaStreamSynchronize(s_k);
    cudaStreamSynchronize(s_out);
    ghb_join_table_free(ctx, t);
    return code;
  };
  // room for the chunk buffers beside what is already in the arena: the
  // arena cannot grow inside a call, so a short arena is an error here
  {
    size_t more = 2 * chunk_out(out_chunk) + 4096;
    if (ctx->scratch_used + more + join_probe_scratch_bytes(n) + (size_t)nchunks * 1024 > ctx->scratch_bytes) {
      // grow once more: nothing of this call's arena content is in flight
      // except the build, so wait for it and start the arena over
      cudaStreamSynchronize(s_k);
      ghb_join_table_free(ctx, t);
      size_t want = need + 2 * chunk_in(chunk) + more + (size_t)nchunks * 1024;
      if ((st = scratch_reserve(ctx, want, s_in))) return st;
      return ghb_hash_join_host(ctx, build_key, probe_key, join_type, build_payload, nbp, out_build,
                                probe_payload, npp, out_probe, out_probe_rowid, out_build_rowid,
                                out_capacity, out_rows, cfg);
    }
  }
  for (int b = 0; b < 2; b++) {
    Slot& sl = slot[b];
    sl.pk.assign(probe_key, probe_key + 1);
    sl.pp.assign(probe_payload, probe_payload + npp);
    auto dev_col = [&](ghb_column& c) {
      void* q = nullptr;
      int32_t r = scratch_alloc(ctx, std::max<size_t>((size_t)chunk * type_width(c.type), 16), &q, s_in);
      if (r) return r;
      c.data = q;
      if (c.null_mode == GHB_NULLS_BYTEMAP) {
        if ((r = scratch_alloc(ctx, std::max<size_t>((size_t)chunk, 16), &q, s_in))) return r;
        c.is_null = (const uint8_t*)q;
      }
      return (int32_t)GHB_OK;
    };
    if ((st = dev_col(sl.pk[0]))) return fail(st);
    for (int j = 0; j < npp; j++)
      if ((st = dev_col(sl.pp[j]))) return fail(st);
    if ((st = stage_out(ctx, out_build, nbp, out_chunk, sl.ob, s_in))) return fail(st);
    if ((st = stage_out(ctx, out_probe, npp, out_chunk, sl.op, s_in))) return fail(st);
    if (out_probe_rowid && (st = scratch_alloc(ctx, (size_t)out_chunk * 4 + 16, (void**)&sl.prow, s_in)))
      return fail(st);
    if (out_build_rowid && (st = scratch_alloc(ctx, (size_t)out_chunk * 4 + 16, (void**)&sl.brow, s_in)))
      return fail(st);
    if ((st = scratch_alloc(ctx, 8, (void**)&sl.d_rows, s_in))) return fail(st);
  }
  cudaEvent_t* ev_in = ctx->hev[0];     // chunk copied in (per buffer)
  cudaEvent_t* ev_probe = ctx->hev[1];  // chunk probed: its input buffer is free
  cudaEvent_t* ev_rows = ctx->hev[2];   // chunk's row count on the host side
  cudaEvent_t* ev_out = ctx->hev[3];    // chunk copied out: its output buffer is free
  int64_t total = 0, written = 0;
  auto copy_out = [&](int64_t c) -> int32_t {
    const int b = (int)(c & 1);
    Slot& sl = slot[b];
    GHB_CUDA_TRY(ctx, cudaEventSynchronize(ev_rows[b]));
    const int64_t rows = h_rows[c];
    total += rows;
    const int64_t r = std::max<int64_t>(0, std::min<int64_t>(rows, out_capacity - written));
    GHB_CUDA_TRY(ctx, cudaStreamWaitEvent(s_out, ev_rows[b], 0));
    if (r > 0) {
      for (int j = 0; j < nbp; j++) {
        const size_t w = type_width(out_build[j].type);
        GHB_CUDA_TRY(ctx, cudaMemcpyAsync((char*)out_build[j].data + written * w, sl.ob[j].data, r * w,
                                          cudaMemcpyDeviceToHost, s_out));
        if (out_build[j].is_null)
          GHB_CUDA_TRY(ctx, cudaMemcpyAsync(out_build[j].is_null + written, sl.ob[j].is_null, r,
                                            cudaMemcpyDeviceToHost, s_out));
      }
      for (int j = 0; j < npp; j++) {
        const size_t w = type_width(out_probe[j].type);
        GHB_CUDA_TRY(ctx, cudaMemcpyAsync((char*)out_probe[j].data + written * w, sl.op[j].data, r * w,
                                          cudaMemcpyDeviceToHost, s_out));
        if (out_probe[j].is_null)
          GHB_CUDA_TRY(ctx, cudaMemcpyAsync(out_probe[j].is_null + written, sl.op[j].is_null, r,
                                            cudaMemcpyDeviceToHost, s_out));
      }
      if (sl.prow)
        GHB_CUDA_TRY(ctx, cudaMemcpyAsync(out_probe_rowid + written, sl.prow, r * 4, cudaMemcpyDeviceToHost,
                                          s_out));
      if (sl.brow)
        GHB_CUDA_TRY(ctx, cudaMemcpyAsync(out_build_rowid + written, sl.brow, r * 4, cudaMemcpyDeviceToHost,
                                          s_out));
    }
    written += r;
    GHB_CUDA_TRY(ctx, cudaEventRecord(ev_out[b], s_out));
    return GHB_OK;
  };
  for (int64_t c = 0; c < nchunks; c++) {
    const int b = (int)(c & 1);
    Slot& sl = slot[b];
    const int64_t r0 = c * chunk, rows = std::min<int64_t>(chunk, n - r0);
    // copy in, once the probe of chunk c - 2 has read this buffer
    if (c >= 2) GHB_CUDA_TRY(ctx, cudaStreamWaitEvent(s_in, ev_probe[b], 0));
    auto copy_in = [&](const ghb_column& h, ghb_column& d) -> int32_t {
      const size_t w = type_width(h.type);
      d.n = rows;
      if (rows > 0 && !h.data) return set_error(ctx, GHB_ERR_INVALID, "probe column data is NULL");
      GHB_CUDA_TRY(ctx, cudaMemcpyAsync((void*)d.data, (const char*)h.data + r0 * w, rows * w,
                                        cudaMemcpyHostToDevice, s_in));
      if (h.null_mode == GHB_NULLS_BYTEMAP) {
        if (!h.is_null) return set_error(ctx, GHB_ERR_INVALID, "probe column is_null is NULL");
        GHB_CUDA_TRY(ctx, cudaMemcpyAsync((void*)d.is_null, h.is_null + r0, rows, cudaMemcpyHostToDevice, s_in));
      }
      return (int32_t)GHB_OK;
    };
    if ((st = copy_in(*probe_key, sl.pk[0]))) return fail(st);
    for (int j = 0; j < npp; j++)
      if ((st = copy_in(probe_payload[j], sl.pp[j]))) return fail(st);
    GHB_CUDA_TRY(ctx, cudaEventRecord(ev_in[b], s_in));
    // probe, once the chunk is in and chunk c - 2's output has been copied out
    GHB_CUDA_TRY(ctx, cudaStreamWaitEvent(s_k, ev_in[b], 0));
    if (c >= 2) GHB_CUDA_TRY(ctx, cudaStreamWaitEvent(s_k, ev_out[b], 0));
    st = join_probe_impl(ctx, t, sl.pk.data(), join_type, sl.ob.data(), sl.pp.data(), npp, sl.op.data(),
                         sl.prow, sl.brow, out_chunk, sl.d_rows, s_k, (int32_t)r0);
    if (st) return fail(st);
    GHB_CUDA_TRY(ctx, cudaEventRecord(ev_probe[b], s_k));
    GHB_CUDA_TRY(ctx, cudaMemcpyAsync(&h_rows[c], sl.d_rows, 8, cudaMemcpyDeviceToHost, s_k));
    GHB_CUDA_TRY(ctx, cudaEventRecord(ev_rows[b], s_k));
    // the previous chunk's output goes out while this one is probed
    if (c >= 1 && (st = copy_out(c - 1))) return fail(st);
  }
  if (nchunks >= 1 && (st = copy_out(nchunks - 1))) return fail(st);
  GHB_CUDA_TRY(ctx, cudaStreamSynchronize(s_out));
  GHB_CUDA_TRY(ctx, cudaStreamSynchronize(s_in));
  st = ghb_sync(ctx, s_k);   // device status of every chunk's kernels
  ghb_join_table_free(ctx, t);
  *out_rows = total;
  if (st) return st;
  if (total > out_capacity)
    return set_error(ctx, GHB_ERR_CAPACITY, "join output of %lld rows exceeds out_capacity %lld",
                     (long long)total, (long long)out_capacity);
  return GHB_OK;
}

int32_t ghb_hash_join_host(ghb_ctx* ctx, const ghb_column* build_key, const ghb_column* probe_key,
                           int32_t join_type, const ghb_column* build_payload, int32_t nbp, ghb_out_column* out_build,
                           const ghb_column* probe_payload, int32_t npp, ghb_out_column* out_probe,
                           int32_t* out_probe_rowid, int32_t* out_build_rowid, int64_t out_capacity,
                           int64_t* out_rows, const ghb_join_cfg* cfg) {
  CallScope cs(ctx, "hash_join_host", 0, true);
  cs.rows(probe_key ? probe_key->n : 0);
  cs.bytes(cols_bytes(build_key, build_key ? 1 : 0) + cols_bytes(probe_key, probe_key ? 1 : 0) +
           cols_bytes(build_payload, nbp) + cols_bytes(probe_payload, npp));
  return cs.done(ghb_hash_join_host_body(ctx, build_key, probe_key, join_type, build_payload, nbp, out_build,
                                         probe_payload, npp, out_probe, out_probe_rowid, out_build_rowid,
                                         out_capacity, out_rows, cfg));
}

static int32_t ghb_sort_host_body(ghb_ctx* ctx, const ghb_column* keys, const int32_t* orders,
                      const int32_t* null_orders, int32_t nkeys, const ghb_column* payload,
                      int32_t npayload, ghb_out_column* out_keys, ghb_out_column* out_payload,
                      int32_t* out_rowid, const ghb_sort_cfg* cfg) {
  if (!ctx || !keys || nkeys < 1 || nkeys > kMaxCols || npayload < 0 || npayload > kMaxCols)
    return set_error(ctx, GHB_ERR_INVALID, "bad key/payload lists");
  cudaStream_t s = 0;
  scratch_reset(ctx);
  int64_t n = keys[0].n;
  size_t need = 8192;
  for (int i = 0; i < nkeys; i++) need += in_bytes(keys[i]) + out_bytes(out_keys[i], n) + 1024;
  for (int i = 0; i < npayload; i++) need += in_bytes(payload[i]) + out_bytes(out_payload[i], n) + 1024;
  if (out_rowid) need += align256((size_t)n * 4) + 256;
  need += sort_scratch_bytes(n);
  int32_t st = scratch_reserve(ctx, need, s);
  if (st) return st;
  std::vector<ghb_column> dk, dp;
  std::vector<ghb_out_column> dok, dop;
  int32_t* d_rowid = nullptr;
  if ((st = stage_in(ctx, keys, nkeys, dk, s))) return st;
  if ((st = stage_in(ctx, payload, npayload, dp, s))) return st;
  if ((st = stage_out(ctx, out_keys, nkeys, n, dok, s))) return st;
  if ((st = stage_out(ctx, out_payload, npayload, n, dop, s))) return st;
  if (out_rowid && (st = scratch_alloc(ctx, (size_t)n * 4 + 16, (void**)&d_rowid, s))) return st;
  // the sort's own scratch comes after the staged buffers in the same arena
  st = sort_impl(ctx, dk.data(), orders, null_orders, nkeys, dp.data(), npayload, dok.data(),
                 dop.data(), d_rowid, cfg, s);
  if (st) return st;
  st = ghb_sync(ctx, s);
  if (st) return st;
  if ((st = copy_back(ctx, out_keys, dok, n, s))) return st;
  if ((st = copy_back(ctx, out_payload, dop, n, s))) return st;
  if (d_rowid && n > 0)
    GHB_CUDA_TRY(ctx, cudaMemcpyAsync(out_rowid, d_rowid, (size_t)n * 4, cudaMemcpyDeviceToHost, s));
  GHB_CUDA_TRY(ctx, cudaStreamSynchronize(s));
  return GHB_OK;
}

int32_t ghb_sort_host(ghb_ctx* ctx, const ghb_column* keys, const int32_t* orders, const int32_t* null_orders,
                      int32_t nkeys, const ghb_column* payload, int32_t npayload, ghb_out_column* out_keys,
                      ghb_out_column* out_payload, int32_t* out_rowid, const ghb_sort_cfg* cfg) {
  CallScope cs(ctx, "sort_host", 0, true);
  cs.rows(keys && nkeys > 0 ? keys[0].n : 0);
  cs.bytes(cols_bytes(keys, nkeys) + cols_bytes(payload, npayload));
  return cs.done(ghb_sort_host_body(ctx, keys, orders, null_orders, nkeys, payload, npayload, out_keys,
                                    out_payload, out_rowid, cfg));
}

}  // extern "C"
