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
                        int32_t*, int64_t, int64_t*, cudaStream_t);
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
  for (int i = 0; i < n; i++) {
    if (h[i].type == GHB_STRING)
      return set_error(ctx, GHB_ERR_UNSUPPORTED, "STRING columns are not on the device path");
    void* p = nullptr;
    int32_t st = scratch_alloc(ctx, std::max<size_t>(col_bytes(h[i]), 16), &p, s);
    if (st) return st;
    if (h[i].n > 0) {
      if (!h[i].data) return set_error(ctx, GHB_ERR_INVALID, "column %d: data is NULL", i);
      GHB_CUDA_TRY(ctx, cudaMemcpyAsync(p, h[i].data, col_bytes(h[i]), cudaMemcpyHostToDevice, s));
    }
    d[i].data = p;
    if (h[i].null_mode == GHB_NULLS_BYTEMAP && h[i].n > 0) {
      if (!h[i].is_null) return set_error(ctx, GHB_ERR_INVALID, "column %d: is_null is NULL", i);
      void* q = nullptr;
      st = scratch_alloc(ctx, (size_t)h[i].n, &q, s);
      if (st) return st;
      GHB_CUDA_TRY(ctx, cudaMemcpyAsync(q, h[i].is_null, (size_t)h[i].n, cudaMemcpyHostToDevice, s));
      d[i].is_null = (const uint8_t*)q;
    }
  }
  return GHB_OK;
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

int32_t copy_back(ghb_ctx* ctx, const ghb_out_column* h, const std::vector<ghb_out_column>& d,
                  int64_t rows, cudaStream_t s) {
  for (size_t i = 0; i < d.size(); i++) {
    if (rows <= 0) break;
    GHB_CUDA_TRY(ctx, cudaMemcpyAsync(h[i].data, d[i].data, (size_t)rows * type_width(h[i].type),
                                      cudaMemcpyDeviceToHost, s));
    if (h[i].is_null)
      GHB_CUDA_TRY(ctx, cudaMemcpyAsync(h[i].is_null, d[i].is_null, (size_t)rows,
                                        cudaMemcpyDeviceToHost, s));
  }
  return GHB_OK;
}

// Reads a device int64 counter and the device status after the stream drains.
int32_t read_count(ghb_ctx* ctx, const int64_t* d_count, int64_t* out, cudaStream_t s) {
  int64_t v = 0;
  GHB_CUDA_TRY(ctx, cudaMemcpyAsync(&v, d_count, sizeof(v), cudaMemcpyDeviceToHost, s));
  int32_t st = ghb_sync(ctx, s);
  *out = v;
  return st;
}

}  // namespace
}  // namespace ghb

using namespace ghb;

extern "C" {

int32_t ghb_filter_host(ghb_ctx* ctx, const ghb_predicate* pred, const ghb_column* cols,
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

int32_t ghb_filter_groupby_host(ghb_ctx* ctx, const ghb_predicate* pred, const ghb_column* cols,
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

int32_t ghb_hash_join_host(ghb_ctx* ctx, const ghb_column* build_key, const ghb_column* probe_key,
                           int32_t join_type, const ghb_column* build_payload, int32_t nbp,
                           ghb_out_column* out_build, const ghb_column* probe_payload, int32_t npp,
                           ghb_out_column* out_probe, int32_t* out_probe_rowid,
                           int32_t* out_build_rowid, int64_t out_capacity, int64_t* out_rows,
                           const ghb_join_cfg* cfg) {
  if (!ctx || !out_rows || !build_key || !probe_key) return GHB_ERR_INVALID;
  if (nbp < 0 || nbp > 8 || npp < 0 || npp > 8) return set_error(ctx, GHB_ERR_INVALID, "payload counts");
  cudaStream_t s = 0;
  scratch_reset(ctx);
  size_t need = 8192 + in_bytes(*build_key) + in_bytes(*probe_key);
  for (int j = 0; j < nbp; j++) need += in_bytes(build_payload[j]) + out_bytes(out_build[j], out_capacity) + 1024;
  for (int j = 0; j < npp; j++) need += in_bytes(probe_payload[j]) + out_bytes(out_probe[j], out_capacity) + 1024;
  if (out_probe_rowid) need += align256((size_t)out_capacity * 4) + 256;
  if (out_build_rowid) need += align256((size_t)out_capacity * 4) + 256;
  need += join_probe_scratch_bytes(probe_key->n);
  int32_t st = scratch_reserve(ctx, need, s);
  if (st) return st;
  std::vector<ghb_column> dbk, dpk, dbp, dpp;
  std::vector<ghb_out_column> dob, dop;
  int64_t* d_rows = nullptr;
  int32_t *d_prow = nullptr, *d_brow = nullptr;
  if ((st = scratch_alloc(ctx, 8, (void**)&d_rows, s))) return st;
  if ((st = stage_in(ctx, build_key, 1, dbk, s))) return st;
  if ((st = stage_in(ctx, probe_key, 1, dpk, s))) return st;
  if ((st = stage_in(ctx, build_payload, nbp, dbp, s))) return st;
  if ((st = stage_in(ctx, probe_payload, npp, dpp, s))) return st;
  if ((st = stage_out(ctx, out_build, nbp, out_capacity, dob, s))) return st;
  if ((st = stage_out(ctx, out_probe, npp, out_capacity, dop, s))) return st;
  if (out_probe_rowid && (st = scratch_alloc(ctx, (size_t)out_capacity * 4 + 16, (void**)&d_prow, s))) return st;
  if (out_build_rowid && (st = scratch_alloc(ctx, (size_t)out_capacity * 4 + 16, (void**)&d_brow, s))) return st;
  ghb_join_table* t = nullptr;
  st = join_build_impl(ctx, dbk.data(), dbp.data(), nbp, cfg, &t, s);
  if (st) return st;
  st = join_probe_impl(ctx, t, dpk.data(), join_type, dob.data(), dpp.data(), npp, dop.data(),
                       d_prow, d_brow, out_capacity, d_rows, s);
  int64_t rows = 0;
  if (!st) st = read_count(ctx, d_rows, &rows, s);
  *out_rows = rows;
  if (!st) {
    int64_t r = std::min(rows, out_capacity);
    st = copy_back(ctx, out_build, dob, r, s);
    if (!st) st = copy_back(ctx, out_probe, dop, r, s);
    if (!st && d_prow && r > 0)
      GHB_CUDA_TRY(ctx, cudaMemcpyAsync(out_probe_rowid, d_prow, r * 4, cudaMemcpyDeviceToHost, s));
    if (!st && d_brow && r > 0)
      GHB_CUDA_TRY(ctx, cudaMemcpyAsync(out_build_rowid, d_brow, r * 4, cudaMemcpyDeviceToHost, s));
    if (!st) GHB_CUDA_TRY(ctx, cudaStreamSynchronize(s));
  }
  ghb_join_table_free(ctx, t);
  return st;
}

int32_t ghb_sort_host(ghb_ctx* ctx, const ghb_column* keys, const int32_t* orders,
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

}  // extern "C"
