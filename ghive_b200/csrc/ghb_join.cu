// ghb_join.cu — device hash equi-join: build (J1) and probe (J2).
//
// Replaces the reference's join, which sorted both inputs' row indices on the
// GPU and merged them single-threaded on the CPU
// (gpu_impl/src/Operator/SortMergeJoinPredicate.cu:8-461), then gathered the
// retained columns on the host (gpu_impl/src/Operator/BaseJoinPredicate.cu:
// 4-97).  Hive's CPU map-join probes a power-of-two open-addressing table of
// (valueRef, key) slot pairs (VectorMapJoinFastLongHashTable.java:99-254);
// the device table keeps that shape with 16-byte slots:
//
//   slot = { uint64 key image (flip_i64, 0 = empty), int32 head+1, int32 count }
//
// Duplicate build keys chain through next[] (head/next hold row+1, 0 ends the
// chain), pushed with atomicExch so concurrent inserts of one key stay
// consistent.  The key INT64_MIN, whose image is the empty marker, lives in
// a side slot at index `slots`.
//
// The probe is one pass: each CTA claims tiles of probe rows in launch order,
// finds each key's slot with linear probing, counts its output rows (build
// matches for INNER, 0/1 for LEFT SEMI, max(matches,1) for LEFT OUTER), scans
// the counts across the CTA, takes the tile's output offset by decoupled
// look-back, and writes (probe row, build row, gathered payloads) in
// probe-row order.
#include <algorithm>

#include "ghb_ctx.hpp"

namespace ghb {

struct __align__(16) JSlot {
  unsigned long long key;
  int32_t head_p1;
  int32_t count;
};

constexpr int kJThreads = 256;
constexpr int kJItems = 8;
constexpr int kJTile = kJThreads * kJItems;
constexpr int kMaxPay = 8;

struct BuildParams {
  ghb_column key;
  JSlot* slots;
  int32_t* next_p1;
  int64_t mask;
  int64_t side;          // index of the side slot (= number of hashed slots)
  unsigned long long* stats;  // [0] rows stored, [1] max duplicates
  int32_t* status;
};

__global__ void __launch_bounds__(256) join_build_kernel(BuildParams p) {
  unsigned long long stored = 0, maxdup = 0;
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < p.key.n;
       r += (int64_t)gridDim.x * blockDim.x) {
    int64_t raw = ld_raw(p.key, r);
    if (raw_is_null(p.key, raw, r)) continue;   // NULL keys never join
    unsigned long long u = flip_i64(raw);
    int64_t s;
    if (u == 0) {
      s = p.side;
    } else {
      s = (int64_t)(mix64(u) & (uint64_t)p.mask);
      int64_t probes = 0;
      while (true) {
        unsigned long long cur = p.slots[s].key;
        if (cur == u) break;
        if (cur == 0) {
          unsigned long long prev = atomicCAS(&p.slots[s].key, 0ull, u);
          if (prev == 0 || prev == u) break;
        }
        s = (s + 1) & p.mask;
        if (++probes > p.mask) {   // table full: cannot happen with load factor < 1
          raise_status(p.status, kDevCapacity);
          s = -1;
          break;
        }
      }
      if (s < 0) continue;
    }
    int old = atomicAdd(&p.slots[s].count, 1);
    int prev = atomicExch(&p.slots[s].head_p1, (int)(r + 1));
    p.next_p1[r] = prev;
    stored++;
    maxdup = max(maxdup, (unsigned long long)(old + 1));
  }
  // one atomic per warp for the statistics
  for (int o = 16; o > 0; o >>= 1) {
    stored += __shfl_down_sync(0xffffffffu, stored, o);
    maxdup = max(maxdup, __shfl_down_sync(0xffffffffu, maxdup, o));
  }
  if ((threadIdx.x & 31) == 0) {
    if (stored) atomicAdd(&p.stats[0], stored);
    if (maxdup) atomicMax(&p.stats[1], maxdup);
  }
}

struct ProbeParams {
  const JSlot* slots;
  const int32_t* next_p1;
  int64_t mask;
  int64_t side;
  ghb_column pkey;
  int32_t join_type;
  int32_t nbp, npp;
  ghb_column bpay[kMaxPay];
  ghb_out_column obp[kMaxPay];
  ghb_column ppay[kMaxPay];
  ghb_out_column opp[kMaxPay];
  int32_t* out_prow;
  int32_t* out_brow;
  int64_t n, ntiles, cap;
  int64_t* d_out_rows;
  uint64_t* lb;
  uint32_t epoch;
  unsigned long long* counters;
  int32_t* status;
};

__device__ __forceinline__ void put_value(const ghb_column& c, const ghb_out_column& o, int64_t row,
                                          int64_t pos) {
  if (row < 0) {  // outer-join miss: NULL
    if (o.is_null) o.is_null[pos] = 1;
    if (o.type == GHB_INT) ((int32_t*)o.data)[pos] = INT32_MAX;
    else if (o.type == GHB_LONG) ((int64_t*)o.data)[pos] = INT64_MAX;
    else ((long long*)o.data)[pos] = 0x7ff8000000000000ll;
    return;
  }
  int64_t raw = ld_raw(c, row);
  if (c.type == GHB_INT) ((int32_t*)o.data)[pos] = (int32_t)raw;
  else ((long long*)o.data)[pos] = raw;
  if (o.is_null) o.is_null[pos] = (c.null_mode != GHB_NULLS_NONE && raw_is_null(c, raw, row)) ? 1 : 0;
}

__device__ __forceinline__ void emit_pair(const ProbeParams& p, int64_t pos, int64_t prow, int32_t brow) {
  if (p.out_prow) p.out_prow[pos] = (int32_t)prow;
  if (p.out_brow) p.out_brow[pos] = brow;
  for (int j = 0; j < p.nbp; j++) put_value(p.bpay[j], p.obp[j], brow, pos);
  for (int j = 0; j < p.npp; j++) put_value(p.ppay[j], p.opp[j], prow, pos);
}

__global__ void __launch_bounds__(kJThreads) join_probe_kernel(ProbeParams p) {
  __shared__ int64_t s_tile;
  __shared__ uint64_t s_warp_tot[kJThreads / 32];
  __shared__ uint64_t s_warp_excl[kJThreads / 32];
  __shared__ uint64_t s_tile_excl;
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;

  while (true) {
    if (threadIdx.x == 0) s_tile = (int64_t)atomicAdd(&p.counters[0], 1ull);
    __syncthreads();
    const int64_t tile = s_tile;
    if (tile >= p.ntiles) break;
    // each warp owns a contiguous segment of 32 * kJItems probe rows
    const int64_t wbase = tile * kJTile + (int64_t)warp * (32 * kJItems);

    int32_t head[kJItems];
    int32_t mult[kJItems];
    uint32_t excl[kJItems];
    uint64_t running = 0;
#pragma unroll
    for (int k = 0; k < kJItems; k++) {
      int64_t row = wbase + k * 32 + lane;
      int32_t m = 0, h = 0;
      if (row < p.n) {
        int64_t raw = ld_raw(p.pkey, row);
        bool found = false;
        if (!raw_is_null(p.pkey, raw, row)) {
          unsigned long long u = flip_i64(raw);
          int64_t s = u == 0 ? p.side : (int64_t)(mix64(u) & (uint64_t)p.mask);
          while (true) {
            JSlot sl = p.slots[s];
            if (sl.key == u && sl.count > 0) {
              found = true;
              m = sl.count;
              h = sl.head_p1;
              break;
            }
            if (sl.key == 0 || u == 0) break;   // empty slot: no match
            s = (s + 1) & p.mask;
          }
        }
        if (p.join_type == GHB_LEFT_SEMI_JOIN) m = found ? 1 : 0;
        else if (p.join_type == GHB_LEFT_OUTER_JOIN && !found) m = 1;
        if (!found) h = 0;
      }
      head[k] = h;
      mult[k] = m;
      // inclusive warp scan of m (ballot when every lane emits 0 or 1)
      uint32_t incl;
      if (__all_sync(0xffffffffu, m <= 1)) {
        unsigned b = __ballot_sync(0xffffffffu, m == 1);
        incl = __popc(b & ((2u << lane) - 1u));
      } else {
        incl = (uint32_t)m;
        for (int o = 1; o < 32; o <<= 1) {
          uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
          if (lane >= o) incl += t;
        }
      }
      excl[k] = (uint32_t)running + incl - (uint32_t)m;
      running += __shfl_sync(0xffffffffu, incl, 31);
    }
    if (lane == 0) s_warp_tot[warp] = running;
    __syncthreads();
    if (warp == 0) {
      uint64_t v = lane < kJThreads / 32 ? s_warp_tot[lane] : 0;
      uint64_t incl = v;
      for (int o = 1; o < 32; o <<= 1) {
        uint64_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
      }
      if (lane < kJThreads / 32) s_warp_excl[lane] = incl - v;
      uint64_t total = __shfl_sync(0xffffffffu, incl, 31);
      uint64_t ex = lookback_exclusive(p.lb, p.epoch, tile, total, p.status);
      if (lane == 0) {
        s_tile_excl = ex;
        if (tile == p.ntiles - 1) *p.d_out_rows = (int64_t)(ex + total);
      }
    }
    __syncthreads();
    const uint64_t wexcl = s_tile_excl + s_warp_excl[warp];
#pragma unroll
    for (int k = 0; k < kJItems; k++) {
      if (mult[k] == 0) continue;
      int64_t row = wbase + k * 32 + lane;
      int64_t pos = (int64_t)(wexcl + excl[k]);
      if (pos + mult[k] > p.cap) {
        raise_status(p.status, kDevCapacity);
        continue;
      }
      if (head[k] == 0 || p.join_type == GHB_LEFT_SEMI_JOIN) {
        emit_pair(p, pos, row, -1);
        continue;
      }
      int32_t b = head[k] - 1;
      for (int j = 0; j < mult[k]; j++) {
        emit_pair(p, pos + j, row, b);
        if (j + 1 < mult[k]) b = p.next_p1[b] - 1;
      }
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    __threadfence();
    unsigned long long done = atomicAdd(&p.counters[1], 1ull);
    if (done == gridDim.x - 1) {
      p.counters[0] = 0;
      p.counters[1] = 0;
      __threadfence();
    }
  }
}

static int64_t next_pow2(int64_t v) {
  int64_t p = 1;
  while (p < v) p <<= 1;
  return p;
}

int32_t join_build_impl(ghb_ctx* ctx, const ghb_column* build_key, const ghb_join_cfg* cfg,
                        ghb_join_table** out, cudaStream_t stream) {
  if (!out) return set_error(ctx, GHB_ERR_INVALID, "out is NULL");
  *out = nullptr;
  int32_t st = validate_columns(ctx, build_key, 1, nullptr);
  if (st) return st;
  if (build_key->type == GHB_DOUBLE)
    return set_error(ctx, GHB_ERR_UNSUPPORTED, "join keys must be LONG or INT");
  if (build_key->n >= INT32_MAX)
    return set_error(ctx, GHB_ERR_UNSUPPORTED, "build side above 2^31-1 rows");
  float lf = (cfg && cfg->load_factor > 0.f && cfg->load_factor < 0.95f) ? cfg->load_factor : 0.5f;
  int64_t C = next_pow2(std::max<int64_t>(64, (int64_t)((double)build_key->n / lf) + 1));
  ghb_join_table* t = new ghb_join_table();
  t->slots = C;
  t->build_rows = build_key->n;
  t->key_type = build_key->type;
  size_t slot_bytes = (size_t)(C + 1) * sizeof(JSlot);
  size_t next_bytes = ((size_t)std::max<int64_t>(build_key->n, 1) * 4 + 255) & ~(size_t)255;
  size_t bytes = slot_bytes + next_bytes + 256;
  // stream-ordered allocation: no device-wide sync, and the pool keeps the
  // memory for the next build on this device
  t->stream = stream;
  if (cudaMallocAsync(&t->alloc, bytes, stream) != cudaSuccess) {
    cudaGetLastError();
    delete t;
    return set_error(ctx, GHB_ERR_OOM, "cannot allocate a %zu-byte join table", bytes);
  }
  t->alloc_bytes = bytes;
  t->keys = (uint64_t*)t->alloc;
  t->next = (int32_t*)((char*)t->alloc + slot_bytes);
  t->d_stats = (unsigned long long*)((char*)t->alloc + slot_bytes + next_bytes);
  if (cudaMemsetAsync(t->alloc, 0, slot_bytes, stream) != cudaSuccess ||
      cudaMemsetAsync(t->d_stats, 0, 256, stream) != cudaSuccess) {
    cudaFreeAsync(t->alloc, stream);
    delete t;
    return set_error(ctx, GHB_ERR_CUDA, "memset of the join table failed");
  }
  BuildParams p;
  p.key = *build_key;
  p.slots = (JSlot*)t->alloc;
  p.next_p1 = t->next;
  p.mask = C - 1;
  p.side = C;
  p.stats = t->d_stats;
  p.status = ctx->d_status;
  if (build_key->n > 0) {
    int grid = (int)std::min<int64_t>((build_key->n + 255) / 256, (int64_t)ctx->num_sms * 8);
    join_build_kernel<<<grid, 256, 0, stream>>>(p);
    ctx->launches++;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
      cudaFreeAsync(t->alloc, stream);
      delete t;
      return set_error(ctx, GHB_ERR_CUDA, "join build launch failed: %s", cudaGetErrorString(e));
    }
  }
  if (cfg && cfg->l2_persist) {
    int max_persist = 0;
    cudaDeviceGetAttribute(&max_persist, cudaDevAttrMaxPersistingL2CacheSize, ctx->device);
    if (max_persist > 0) {
      cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, (size_t)max_persist);
      cudaStreamAttrValue attr;
      std::memset(&attr, 0, sizeof(attr));
      attr.accessPolicyWindow.base_ptr = t->alloc;
      attr.accessPolicyWindow.num_bytes = std::min(slot_bytes, (size_t)max_persist);
      attr.accessPolicyWindow.hitRatio = 1.0f;
      attr.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
      attr.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
      cudaStreamSetAttribute(stream, cudaStreamAttributeAccessPolicyWindow, &attr);
      t->l2_window = true;
    }
  }
  *out = t;
  return GHB_OK;
}

int32_t join_probe_impl(ghb_ctx* ctx, const ghb_join_table* t, const ghb_column* probe_key,
                        int32_t join_type, const ghb_column* build_payload, int32_t nbp,
                        ghb_out_column* out_build, const ghb_column* probe_payload, int32_t npp,
                        ghb_out_column* out_probe, int32_t* out_probe_rowid,
                        int32_t* out_build_rowid, int64_t out_capacity, int64_t* d_out_rows,
                        cudaStream_t stream) {
  if (!t) return set_error(ctx, GHB_ERR_INVALID, "table is NULL");
  int32_t st = validate_columns(ctx, probe_key, 1, nullptr);
  if (st) return st;
  if (probe_key->type == GHB_DOUBLE)
    return set_error(ctx, GHB_ERR_UNSUPPORTED, "join keys must be LONG or INT");
  if (probe_key->n >= INT32_MAX)
    return set_error(ctx, GHB_ERR_UNSUPPORTED, "probe side above 2^31-1 rows per call");
  if (join_type != GHB_INNER_JOIN && join_type != GHB_LEFT_SEMI_JOIN && join_type != GHB_LEFT_OUTER_JOIN)
    return set_error(ctx, GHB_ERR_UNSUPPORTED, "join type %d", join_type);
  if (nbp < 0 || nbp > kMaxPay || npp < 0 || npp > kMaxPay)
    return set_error(ctx, GHB_ERR_INVALID, "payload counts %d/%d outside [0,%d]", nbp, npp, kMaxPay);
  if (!d_out_rows) return set_error(ctx, GHB_ERR_INVALID, "d_out_rows is NULL");
  ProbeParams p;
  std::memset(&p, 0, sizeof(p));
  for (int j = 0; j < nbp; j++) {
    st = validate_columns(ctx, &build_payload[j], 1, nullptr);
    if (st) return st;
    if (build_payload[j].n != t->build_rows)
      return set_error(ctx, GHB_ERR_INVALID, "build payload %d has %lld rows, table has %lld", j,
                       (long long)build_payload[j].n, (long long)t->build_rows);
    if (out_build[j].type != build_payload[j].type || !out_build[j].data)
      return set_error(ctx, GHB_ERR_INVALID, "build payload output %d: bad type or data", j);
    p.bpay[j] = build_payload[j];
    p.obp[j] = out_build[j];
  }
  for (int j = 0; j < npp; j++) {
    st = validate_columns(ctx, &probe_payload[j], 1, nullptr);
    if (st) return st;
    if (probe_payload[j].n != probe_key->n)
      return set_error(ctx, GHB_ERR_INVALID, "probe payload %d row count differs from the key", j);
    if (out_probe[j].type != probe_payload[j].type || !out_probe[j].data)
      return set_error(ctx, GHB_ERR_INVALID, "probe payload output %d: bad type or data", j);
    p.ppay[j] = probe_payload[j];
    p.opp[j] = out_probe[j];
  }
  p.slots = (const JSlot*)t->alloc;
  p.next_p1 = t->next;
  p.mask = t->slots - 1;
  p.side = t->slots;
  p.pkey = *probe_key;
  p.join_type = join_type;
  p.nbp = nbp;
  p.npp = npp;
  p.out_prow = out_probe_rowid;
  p.out_brow = out_build_rowid;
  p.n = probe_key->n;
  p.ntiles = (p.n + kJTile - 1) / kJTile;
  p.cap = out_capacity;
  p.d_out_rows = d_out_rows;
  p.counters = ctx->d_counters;
  p.status = ctx->d_status;
  if (p.ntiles == 0) {
    GHB_CUDA_TRY(ctx, cudaMemsetAsync(d_out_rows, 0, sizeof(int64_t), stream));
    return GHB_OK;
  }
  st = lookback_prepare(ctx, p.ntiles, &p.epoch, stream);
  if (st) return st;
  p.lb = ctx->lb_status;
  int per_sm = 0;
  GHB_CUDA_TRY(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, join_probe_kernel, kJThreads, 0));
  int grid = (int)std::min<int64_t>(p.ntiles, (int64_t)ctx->num_sms * std::max(1, per_sm));
  join_probe_kernel<<<grid, kJThreads, 0, stream>>>(p);
  GHB_LAUNCH_CHECK(ctx);
  return GHB_OK;
}

}  // namespace ghb

using namespace ghb;

extern "C" {

int32_t ghb_join_build(ghb_ctx* ctx, const ghb_column* build_key, const ghb_join_cfg* cfg,
                       ghb_join_table** out, void* stream) {
  if (!ctx) return GHB_ERR_INVALID;
  return join_build_impl(ctx, build_key, cfg, out, (cudaStream_t)stream);
}

int32_t ghb_join_table_free(ghb_ctx* ctx, ghb_join_table* table) {
  if (!ctx || !table) return GHB_ERR_INVALID;
  if (table->l2_window) {
    cudaStreamSynchronize(table->stream);
    cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, 0);
    cudaCtxResetPersistingL2Cache();
  }
  // released in the order of the build stream: probes issued on that stream
  // before this call finish first; probes on other streams must be ordered
  // before it by the caller
  if (table->alloc) cudaFreeAsync(table->alloc, table->stream);
  delete table;
  return GHB_OK;
}

int32_t ghb_join_table_info(ghb_ctx* ctx, const ghb_join_table* table, int64_t* rows,
                            int64_t* max_dup, int64_t* slots) {
  if (!ctx || !table) return GHB_ERR_INVALID;
  unsigned long long st[2] = {0, 0};
  GHB_CUDA_TRY(ctx, cudaMemcpy(st, table->d_stats, sizeof(st), cudaMemcpyDeviceToHost));
  if (rows) *rows = (int64_t)st[0];
  if (max_dup) *max_dup = (int64_t)st[1];
  if (slots) *slots = table->slots;
  return GHB_OK;
}

int32_t ghb_join_probe(ghb_ctx* ctx, const ghb_join_table* table, const ghb_column* probe_key,
                       int32_t join_type, const ghb_column* build_payload, int32_t n_build_payload,
                       ghb_out_column* out_build, const ghb_column* probe_payload,
                       int32_t n_probe_payload, ghb_out_column* out_probe, int32_t* out_probe_rowid,
                       int32_t* out_build_rowid, int64_t out_capacity, int64_t* d_out_rows,
                       void* stream) {
  if (!ctx) return GHB_ERR_INVALID;
  scratch_reset(ctx);
  return join_probe_impl(ctx, table, probe_key, join_type, build_payload, n_build_payload, out_build,
                         probe_payload, n_probe_payload, out_probe, out_probe_rowid, out_build_rowid,
                         out_capacity, d_out_rows, (cudaStream_t)stream);
}

}  // extern "C"
