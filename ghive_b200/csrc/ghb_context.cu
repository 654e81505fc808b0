// ghb_context.cu — contexts, errors, scratch arena, argument validation.
//
// Replaces the process-global mutable state of the reference
// (SinkOperator::table_map and friends, gpu_impl/src/Parser/Parser.cu:16-20)
// with an explicit context per caller, and its stdout-and-nullptr error
// convention (gpu_impl/src/ghive_JNIInterface.cu:111-118) with status codes.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>

#include "ghb_ctx.hpp"

namespace ghb {

int32_t set_error(ghb_ctx* ctx, int32_t code, const char* fmt, ...) {
  if (ctx) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    ctx->last_error = buf;
  }
  return code;
}

int32_t scratch_reset(ghb_ctx* ctx) {
  ctx->scratch_used = 0;
  return GHB_OK;
}

int32_t regrow(ghb_ctx* ctx, void** buf, size_t* bytes, size_t want, cudaStream_t stream, bool zero) {
  if (ctx->stream_ordered) {
    // the old buffer is only used on this stream: free and allocate in its order
    if (*buf) cudaFreeAsync(*buf, stream);
    *buf = nullptr;
    *bytes = 0;
    cudaError_t e = ctx->pool ? cudaMallocFromPoolAsync(buf, want, ctx->pool, stream)
                              : cudaMallocAsync(buf, want, stream);
    if (e != cudaSuccess) {
      cudaGetLastError();
      *buf = nullptr;
      return set_error(ctx, GHB_ERR_OOM, "cannot allocate %zu bytes of device memory", want);
    }
  } else {
    // the old buffer may still be read by work queued on any stream
    GHB_CUDA_TRY(ctx, cudaDeviceSynchronize());
    if (*buf) cudaFree(*buf);
    *buf = nullptr;
    *bytes = 0;
    if (cudaMalloc(buf, want) != cudaSuccess) {
      cudaGetLastError();
      *buf = nullptr;
      return set_error(ctx, GHB_ERR_OOM, "cannot allocate %zu bytes of device memory", want);
    }
  }
  *bytes = want;
  if (zero) GHB_CUDA_TRY(ctx, cudaMemsetAsync(*buf, 0, want, stream));
  return GHB_OK;
}

int32_t ensure_dyn_smem(ghb_ctx* ctx, const void* fn, size_t bytes) {
  static std::mutex mu;
  static std::map<std::pair<int, const void*>, int> done;
  int dev = 0;
  GHB_CUDA_TRY(ctx, cudaGetDevice(&dev));
  std::lock_guard<std::mutex> g(mu);
  auto key = std::make_pair(dev, fn);
  auto it = done.find(key);
  if (it != done.end() && (size_t)it->second >= bytes) return GHB_OK;
  int optin = 0;
  GHB_CUDA_TRY(ctx, cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  cudaFuncAttributes fa;
  GHB_CUDA_TRY(ctx, cudaFuncGetAttributes(&fa, fn));
  // the dynamic limit is what the opt-in maximum leaves beside the static part
  const int limit = optin - (int)fa.sharedSizeBytes;
  if (bytes > (size_t)limit)
    return set_error(ctx, GHB_ERR_UNSUPPORTED,
                     "kernel needs %zu bytes of dynamic shared memory, at most %d are available", bytes, limit);
  GHB_CUDA_TRY(ctx, cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, limit));
  done[key] = limit;
  return GHB_OK;
}

int32_t scratch_reserve(ghb_ctx* ctx, size_t total, cudaStream_t stream) {
  if (total <= ctx->scratch_bytes) return GHB_OK;
  size_t want = std::max(total, ctx->scratch_bytes * 2);
  return regrow(ctx, (void**)&ctx->scratch, &ctx->scratch_bytes, want, stream, false);
}

int32_t scratch_alloc(ghb_ctx* ctx, size_t bytes, void** out, cudaStream_t stream) {
  size_t off = (ctx->scratch_used + 255) & ~(size_t)255;
  if (off + bytes > ctx->scratch_bytes) {
    if (ctx->scratch_used != 0)
      return set_error(ctx, GHB_ERR_OOM, "scratch arena exhausted inside one call");
    int32_t st = scratch_reserve(ctx, off + bytes, stream);
    if (st) return st;
  }
  *out = ctx->scratch + off;
  ctx->scratch_used = off + bytes;
  return GHB_OK;
}

int32_t lookback_prepare(ghb_ctx* ctx, int64_t tiles, uint32_t* epoch, cudaStream_t stream) {
  if (tiles > ctx->lb_tiles) {
    int64_t want = std::max<int64_t>(tiles, 1 << 16);
    size_t bytes = (size_t)ctx->lb_tiles * sizeof(uint64_t);
    ctx->lb_tiles = 0;
    int32_t st = regrow(ctx, (void**)&ctx->lb_status, &bytes, want * sizeof(uint64_t), stream, true);
    if (st) return st;
    ctx->lb_tiles = want;
    ctx->epoch = 0;
  }
  ctx->epoch = (ctx->epoch + 1) & (uint32_t)kEpochMask;
  if (ctx->epoch == 0) {
    // the 20-bit tag wrapped: clear so no stale word can carry the new tag
    GHB_CUDA_TRY(ctx, cudaMemsetAsync(ctx->lb_status, 0, ctx->lb_tiles * sizeof(uint64_t), stream));
    ctx->epoch = 1;
  }
  *epoch = ctx->epoch;
  return GHB_OK;
}

int32_t validate_columns(ghb_ctx* ctx, const ghb_column* cols, int32_t ncols, int64_t* n, bool allow_string) {
  if (ncols < 0 || ncols > kMaxCols)
    return set_error(ctx, GHB_ERR_INVALID, "ncols=%d outside [0,%d]", ncols, kMaxCols);
  if (ncols > 0 && !cols) return set_error(ctx, GHB_ERR_INVALID, "cols is NULL");
  int64_t rows = -1;
  for (int i = 0; i < ncols; i++) {
    const ghb_column& c = cols[i];
    if (c.type == GHB_STRING) {
      if (!allow_string)
        return set_error(ctx, GHB_ERR_UNSUPPORTED, "column %d: STRING columns are not supported here", i);
      if (c.n > 0 && !c.aux) return set_error(ctx, GHB_ERR_INVALID, "column %d: STRING without its index", i);
      if (rows >= 0 && c.n != rows)
        return set_error(ctx, GHB_ERR_INVALID, "column %d has %lld rows, column 0 has %lld", i,
                         (long long)c.n, (long long)rows);
      rows = c.n;
      continue;
    }
    if (c.type != GHB_LONG && c.type != GHB_DOUBLE && c.type != GHB_INT)
      return set_error(ctx, GHB_ERR_INVALID, "column %d: unknown type %d", i, c.type);
    if (c.null_mode < GHB_NULLS_NONE || c.null_mode > GHB_NULLS_BYTEMAP)
      return set_error(ctx, GHB_ERR_INVALID, "column %d: unknown null_mode %d", i, c.null_mode);
    if (c.null_mode == GHB_NULLS_BYTEMAP && !c.is_null && c.n > 0)
      return set_error(ctx, GHB_ERR_INVALID, "column %d: BYTEMAP nulls without is_null", i);
    if (c.n < 0) return set_error(ctx, GHB_ERR_INVALID, "column %d: negative row count", i);
    if (c.n > 0 && !c.data) return set_error(ctx, GHB_ERR_INVALID, "column %d: data is NULL", i);
    if (rows >= 0 && c.n != rows)
      return set_error(ctx, GHB_ERR_INVALID, "column %d has %lld rows, column 0 has %lld", i,
                       (long long)c.n, (long long)rows);
    rows = c.n;
  }
  if (n) *n = rows < 0 ? 0 : rows;
  return GHB_OK;
}

// Copies the tree into a post-order program (children before parents), as
// the device evaluator sweeps it forward.  Rejects cycles, bad indices and
// leaves whose mode needs a literal pair that is absent.
int32_t build_pred_prog(ghb_ctx* ctx, const ghb_predicate* pred, const ghb_column* cols, int32_t ncols,
                        PredProg* prog) {
  std::memset(prog, 0, sizeof(*prog));
  if (!pred || pred->n_nodes == 0) return GHB_OK;
  if (pred->n_nodes < 0 || pred->n_nodes > GHB_MAX_PRED_NODES || !pred->nodes)
    return set_error(ctx, GHB_ERR_INVALID, "predicate has %d nodes (max %d)", pred->n_nodes,
                     GHB_MAX_PRED_NODES);
  if (pred->root < 0 || pred->root >= pred->n_nodes)
    return set_error(ctx, GHB_ERR_INVALID, "predicate root %d out of range", pred->root);
  std::vector<int> order, state(pred->n_nodes, 0), remap(pred->n_nodes, -1);
  int32_t strbytes = 0;
  // iterative post-order DFS from the root
  std::vector<std::pair<int, int>> stack{{pred->root, 0}};
  while (!stack.empty()) {
    auto& top = stack.back();
    int id = top.first;
    const ghb_pred_node& nd = pred->nodes[id];
    bool inner = nd.mode == GHB_FILTER_AND || nd.mode == GHB_FILTER_OR;
    if (top.second == 0) {
      if (state[id] == 1)
        return set_error(ctx, GHB_ERR_INVALID, "predicate tree has a cycle at node %d", id);
      if (state[id] == 2) { stack.pop_back(); continue; }
      state[id] = 1;
    }
    if (inner && top.second < 2) {
      int ch = nd.child[top.second++];
      if (ch < 0 || ch >= pred->n_nodes)
        return set_error(ctx, GHB_ERR_INVALID, "node %d: child index %d out of range", id, ch);
      stack.push_back({ch, 0});
      continue;
    }
    state[id] = 2;
    remap[id] = (int)order.size();
    order.push_back(id);
    stack.pop_back();
  }
  for (size_t k = 0; k < order.size(); k++) {
    ghb_pred_node nd = pred->nodes[order[k]];
    if (nd.mode == GHB_FILTER_AND || nd.mode == GHB_FILTER_OR) {
      nd.child[0] = remap[nd.child[0]];
      nd.child[1] = remap[nd.child[1]];
    } else {
      if (nd.mode < GHB_FILTER_EQ || nd.mode > GHB_FILTER_NOT_NULL)
        return set_error(ctx, GHB_ERR_INVALID, "node %d: unknown mode %d", order[k], nd.mode);
      if (nd.col < 0 || nd.col >= ncols)
        return set_error(ctx, GHB_ERR_INVALID, "node %d: column %d out of range", order[k], nd.col);
      if (nd.col2 >= ncols)
        return set_error(ctx, GHB_ERR_INVALID, "node %d: column %d out of range", order[k], nd.col2);
      bool two_lit = nd.mode == GHB_FILTER_RANGE || nd.mode == GHB_FILTER_EQ_RANGE ||
                     nd.mode == GHB_FILTER_NOT_RANGE || nd.mode == GHB_FILTER_NOT_EQ_RANGE;
      if (two_lit && nd.col2 >= 0)
        return set_error(ctx, GHB_ERR_INVALID, "node %d: range modes compare with literals only", order[k]);
      const bool str = cols && cols[nd.col].type == GHB_STRING;
      if (cols && nd.col2 >= 0 && (cols[nd.col2].type == GHB_STRING) != str)
        return set_error(ctx, GHB_ERR_INVALID, "node %d: a STRING column compares with a STRING only",
                         order[k]);
      if (str) {
        if (!cols[nd.col].aux || (nd.col2 >= 0 && !cols[nd.col2].aux))
          return set_error(ctx, GHB_ERR_INVALID, "node %d: STRING column without its index", order[k]);
        prog->has_str = 1;
        // the literals' bytes go into the program (kernel parameter space)
        const int nlit = nd.col2 >= 0 || nd.mode == GHB_FILTER_NOT_NULL ? 0 : (two_lit ? 2 : 1);
        for (int j = 0; j < 2; j++) {
          const int32_t len = j < nlit ? nd.lit_s_len[j] : 0;
          if (len < 0 || (len > 0 && !nd.lit_s[j]))
            return set_error(ctx, GHB_ERR_INVALID, "node %d: string literal %d without bytes", order[k], j);
          if (strbytes + len > GHB_MAX_PRED_STR_BYTES)
            return set_error(ctx, GHB_ERR_UNSUPPORTED, "string literals of more than %d bytes",
                             GHB_MAX_PRED_STR_BYTES);
          if (len) std::memcpy(prog->sbytes + strbytes, nd.lit_s[j], len);
          nd.lit_i[j] = strbytes;
          nd.lit_s_len[j] = len;
          strbytes += len;
        }
      }
      nd.lit_s[0] = nd.lit_s[1] = nullptr;   // host pointers never reach a kernel
    }
    prog->nodes[k] = nd;
  }
  prog->n_nodes = (int32_t)order.size();
  return GHB_OK;
}

}  // namespace ghb

using namespace ghb;

extern "C" {

int32_t ghb_abi_version(void) { return GHB_ABI_VERSION; }

int32_t ghb_ctx_create(int32_t device, int64_t arena_bytes, ghb_ctx** out) {
  if (!out) return GHB_ERR_INVALID;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return GHB_ERR_CUDA;
  }
  if (device < 0 || device >= ndev) return GHB_ERR_INVALID;
  if (cudaSetDevice(device) != cudaSuccess) return GHB_ERR_CUDA;
  ghb_ctx* ctx = new ghb_ctx();
  ctx->device = device;
  cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device);
  if (cudaMalloc((void**)&ctx->d_status, 64) != cudaSuccess ||
      cudaMalloc((void**)&ctx->d_counters, 64 * sizeof(unsigned long long)) != cudaSuccess) {
    ghb_ctx_destroy(ctx);
    return GHB_ERR_OOM;
  }
  // keep freed stream-ordered allocations (join tables) cached in the pool
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  cudaMemset(ctx->d_status, 0, 64);
  cudaMemset(ctx->d_counters, 0, 64 * sizeof(unsigned long long));
  if (arena_bytes > 0 && scratch_reserve(ctx, (size_t)arena_bytes, 0) != GHB_OK) {
    ghb_ctx_destroy(ctx);
    return GHB_ERR_OOM;
  }
  if (cudaDeviceSynchronize() != cudaSuccess) {
    ghb_ctx_destroy(ctx);
    return GHB_ERR_CUDA;
  }
  // the per-call log named by the environment, if any
  if (const char* path = std::getenv("GHB_LOG")) {
    const char* lv = std::getenv("GHB_LOG_LEVEL");
    const char* pk = std::getenv("GHB_LOG_PEAK_GBS");
    if (*path && ghb_ctx_set_log(ctx, path, lv ? std::atoi(lv) : 1, pk ? std::atof(pk) : 0) != GHB_OK) {
      ghb_ctx_destroy(ctx);
      return GHB_ERR_INVALID;
    }
  }
  *out = ctx;
  return GHB_OK;
}

int32_t ghb_ctx_destroy(ghb_ctx* ctx) {
  if (!ctx) return GHB_ERR_INVALID;
  cudaDeviceSynchronize();
  if (ctx->d_status) cudaFree(ctx->d_status);
  if (ctx->d_counters) cudaFree(ctx->d_counters);
  if (ctx->scratch) cudaFree(ctx->scratch);
  if (ctx->lb_status) cudaFree(ctx->lb_status);
  if (ctx->gb_table) cudaFree(ctx->gb_table);
  if (ctx->pinned) cudaFreeHost(ctx->pinned);
  for (int l = 0; l < kStageLanes; l++)
    for (int b = 0; b < 2; b++) {
      if (ctx->stage[l][b]) cudaFreeHost(ctx->stage[l][b]);
      if (ctx->stage_ev[l][b]) cudaEventDestroy(ctx->stage_ev[l][b]);
    }
  for (cudaStream_t& hs : ctx->hstream)
    if (hs) cudaStreamDestroy(hs);
  for (auto& row : ctx->hev)
    for (cudaEvent_t& e : row)
      if (e) cudaEventDestroy(e);
  ghb_ctx_set_log(ctx, nullptr, 0, 0);
  delete ctx;
  return GHB_OK;
}

int32_t ghb_ctx_set_log(ghb_ctx* ctx, const char* path, int32_t level, double peak_gbs) {
  if (!ctx) return GHB_ERR_INVALID;
  if (ctx->log) std::fclose(ctx->log);
  ctx->log = nullptr;
  ctx->log_level = 0;
  for (cudaEvent_t& e : ctx->log_ev)
    if (e) {
      cudaEventDestroy(e);
      e = nullptr;
    }
  if (!path || level <= 0) return GHB_OK;
  ctx->log = std::fopen(path, "a");
  if (!ctx->log) return set_error(ctx, GHB_ERR_INVALID, "cannot open the log file %s", path);
  ctx->log_level = level;
  ctx->log_peak_gbs = peak_gbs > 0 ? peak_gbs : 0;
  if (level >= 2)
    for (cudaEvent_t& e : ctx->log_ev) GHB_CUDA_TRY(ctx, cudaEventCreate(&e));
  return GHB_OK;
}

const char* ghb_last_error(const ghb_ctx* ctx) {
  return ctx ? ctx->last_error.c_str() : "null context";
}

int64_t ghb_kernel_launches(const ghb_ctx* ctx) { return ctx ? ctx->launches : -1; }

int32_t ghb_ctx_set_spin_limit(ghb_ctx* ctx, int32_t polls) {
  if (!ctx) return GHB_ERR_INVALID;
  ctx->spin_limit = polls > 0 ? polls : ghb::kSpinLimit;
  return GHB_OK;
}

int32_t ghb_sync(ghb_ctx* ctx, void* stream) {
  if (!ctx) return GHB_ERR_INVALID;
  cudaStream_t s = (cudaStream_t)stream;
  GHB_CUDA_TRY(ctx, cudaStreamSynchronize(s));
  int32_t st = 0;
  GHB_CUDA_TRY(ctx, cudaMemcpy(&st, ctx->d_status, sizeof(st), cudaMemcpyDeviceToHost));
  if (st != 0) {
    GHB_CUDA_TRY(ctx, cudaMemset(ctx->d_status, 0, sizeof(st)));
    ctx->gb_dirty = true;  // a failed group-by may leave its table partly filled
    if (st == GHB_ERR_TIMEOUT) return set_error(ctx, st, "a device-side wait timed out");
    if (st == GHB_ERR_CAPACITY) return set_error(ctx, st, "output or table capacity exceeded");
    return set_error(ctx, st, "device error %d", st);
  }
  return GHB_OK;
}

}  // extern "C"
