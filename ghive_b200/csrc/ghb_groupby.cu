// ghb_groupby.cu — fused filter + hash group-by aggregation (G1 + G2).
//
// Replaces GroupByPredicate::gpu_execute (gpu_impl/src/Operator/
// GroupByPredicate.cu:19-359), which sorted row indices with a comparison
// sort and then ran one H2D + reduce_by_key + D2H pass per aggregate
// (:506-720).  Here one pass over the rows evaluates the filter predicate and
// folds every aggregate of the row into a hash table:
//
//   G1  persistent CTAs; each streams 2048-row tiles of the columns it needs
//       into shared memory with bulk copies (cp.async.bulk, completing on an
//       mbarrier, two stages so the next tile loads while this one is
//       folded), evaluates the predicate from shared memory, and folds each
//       passing row into a shared-memory open-addressing table (keys + one
//       64-bit accumulator per aggregate state); rows whose key does not fit
//       go straight to the global table; at the end the CTA merges its shared
//       table into the global one.
//   G2  finalize: walks the global table, emits one output row per group
//       (COUNT, SUM, AVG = sum/count, MIN, MAX with Hive's NULL rules) and
//       zeroes every slot it read, so the next call needs no memset.
//
// Semantics follow Hive's UDAFs (VectorUDAFSum.txt:59-71, VectorUDAFAvg.txt:
// 56-71, VectorUDAFMinMax.txt:65-72): SUM over integers wraps silently, SUM
// and AVG over doubles are double sums, an aggregate that saw only NULLs is
// NULL, COUNT(*) counts rows, COUNT(col) counts non-NULL values.  Double sums
// are accumulated with an error-free transformation: every atomicAdd returns
// the old value, so the adding thread knows the exact rounding error of that
// addition (Knuth's TwoSum) and adds it to a companion compensation word;
// sum + compensation is then accurate to ~1 ulp whatever the order.
#include <algorithm>

#include "ghb_ctx.hpp"

namespace ghb {

enum AccKind : int8_t {
  A_CNT_STAR = 0,  // rows in the group (always accumulator 0: also the "slot used" flag)
  A_CNT_NN = 1,    // non-NULL values of a column
  A_SUM_I = 2,     // int64 wrapping sum
  A_SUM_F = 3,     // double sum; accumulator a+1 is its compensation
  A_COMP_F = 4,
  A_MAX_O = 5,     // atomicMax of the order-preserving unsigned image
  A_MIN_O = 6,     // atomicMax of the complemented image
};
constexpr int kMaxAcc = 16;
constexpr int kMaxAggs = 16;
constexpr int kGbThreads = 1024;
constexpr int kGbRows = 2;     // tile rows per thread at most (tile = 1024 or 2048 rows)

struct AccPlan {
  int32_t n_acc;
  int8_t kind[kMaxAcc];
  int8_t col[kMaxAcc];
};

struct OutAgg {
  int8_t type;       // GHB_AGG_*
  int8_t in_type;    // input column type
  int8_t acc_val;
  int8_t acc_cnt;    // accumulator that says "saw a non-NULL value"
};

struct GbParams {
  ColSet cols;
  PredProg pred;
  AccPlan acc;
  int32_t key_col;       // -1: global aggregate (all rows in one group)
  int32_t smem_slots;    // power of two, 0 = no shared stage
  int32_t warp_agg;      // combine equal keys within a warp before the atomics
  int64_t n;
  uint64_t* gkeys;       // [C + 2] stored keys (flip_i64 of the raw key), 0 = empty
  uint64_t* gacc;        // [n_acc][C + 2]
  int64_t C;             // power of two
  int32_t gshift;        // 64 - log2(C)
  int32_t gprobe;        // probe limit in the global table
  int32_t* status;
  int64_t* d_out_groups;
  // column tiles in shared memory
  int32_t tile_rows;     // rows per tile (multiple of the block size and of 4)
  int64_t ntiles;
  int32_t stage_bytes;   // bytes of one stage (128-byte multiple)
  int32_t tx_bytes;      // bytes the bulk copies of one full tile deliver
  int32_t col_off[kMaxCols];   // byte offset of a used column's tile in a stage, -1 unused
  int32_t null_off[kMaxCols];  // byte offset of a BYTEMAP column's null bytes, -1 none
  int32_t bulk;          // column bases are 16-byte aligned: full tiles arrive by bulk copy
};

struct FinParams {
  const uint64_t* gkeys_ro;
  uint64_t* gkeys;
  uint64_t* gacc;
  int64_t C;
  int32_t n_acc;
  int32_t key_type;      // -1: global aggregate
  ghb_out_column key_out;
  int32_t naggs;
  OutAgg agg[kMaxAggs];
  ghb_out_column out[kMaxAggs];
  int64_t cap;
  int64_t* d_out_groups;
  int32_t* status;
};

// ---------------------------------------------------------------- device
__device__ __forceinline__ double two_sum_err(double a, double b, double s) {
  double bb = __dsub_rn(s, a);
  return __dadd_rn(__dsub_rn(a, __dsub_rn(s, bb)), __dsub_rn(b, bb));
}

// Compensated atomic add of x into (sum, comp).
__device__ __forceinline__ void atomic_add_comp(uint64_t* sum, uint64_t* comp, double x) {
  if (x == 0.0) return;
  double old = atomicAdd((double*)sum, x);
  double e = two_sum_err(old, x, __dadd_rn(old, x));
  if (e != 0.0) atomicAdd((double*)comp, e);
}

__device__ __forceinline__ uint64_t order_image(int type, int64_t raw) {
  return type == GHB_DOUBLE ? flip_f64_bits((uint64_t)raw) : flip_i64(raw);
}

// Slot of a key image in a table of 2^(64 - shift) slots: Fibonacci hashing.
__device__ __forceinline__ int64_t hslot(uint64_t u, int shift) {
  return (int64_t)((u * 0x9E3779B97F4A7C15ull) >> shift);
}

// Open-addressing find-or-insert of a non-zero stored key.  Linear probing;
// returns the slot or -1 after max_probe probes.
__device__ __forceinline__ int64_t table_insert(uint64_t* keys, int64_t mask, int shift, uint64_t u,
                                                int max_probe) {
  int64_t h = hslot(u, shift);
  for (int p = 0; p < max_probe; p++) {
    uint64_t cur = keys[h];
    if (cur == u) return h;
    if (cur == 0) {
      unsigned long long prev = atomicCAS((unsigned long long*)&keys[h], 0ull, (unsigned long long)u);
      if (prev == 0 || prev == u) return h;
    }
    h = (h + 1) & mask;
  }
  return -1;
}

// One row of the current tile, read from shared memory.
struct TileRow {
  const GbParams* p;
  const unsigned char* stage;
  int r;
  __device__ __forceinline__ int64_t raw(int c) const {
    const unsigned char* b = stage + p->col_off[c];
    return p->cols.c[c].type == GHB_INT ? (int64_t)((const int32_t*)b)[r] : ((const long long*)b)[r];
  }
  __device__ __forceinline__ bool null(int c, int64_t v) const {
    const ghb_column& col = p->cols.c[c];
    if (col.null_mode == GHB_NULLS_NONE) return false;
    if (col.null_mode == GHB_NULLS_BYTEMAP) return stage[p->null_off[c] + r] != 0;
    if (col.type == GHB_INT) return v == (int64_t)INT32_MAX;
    if (col.type == GHB_LONG) return v == INT64_MAX;
    double d = __longlong_as_double(v);
    return d != d;
  }
};

__device__ __forceinline__ bool leaf_tile(const ghb_pred_node& nd, const TileRow& t) {
  const int type = t.p->cols.c[nd.col].type;
  int64_t x = t.raw(nd.col);
  if (t.null(nd.col, x)) return false;
  if (nd.mode == GHB_FILTER_NOT_NULL) return true;
  if (nd.col2 >= 0) {
    const int type2 = t.p->cols.c[nd.col2].type;
    int64_t y = t.raw(nd.col2);
    if (t.null(nd.col2, y)) return false;
    if (type == GHB_DOUBLE || type2 == GHB_DOUBLE)
      return cmp_mode<double>(nd.mode, raw_to_f64(type, x), raw_to_f64(type2, y), 0.0);
    return cmp_mode<int64_t>(nd.mode, x, y, 0);
  }
  if (type == GHB_DOUBLE || nd.lit_is_double) {
    double a = nd.lit_is_double ? nd.lit_d[0] : (double)nd.lit_i[0];
    double b = nd.lit_is_double ? nd.lit_d[1] : (double)nd.lit_i[1];
    return cmp_mode<double>(nd.mode, raw_to_f64(type, x), a, b);
  }
  return cmp_mode<int64_t>(nd.mode, x, nd.lit_i[0], nd.lit_i[1]);
}

__device__ __forceinline__ bool pred_tile(const PredProg& pp, const TileRow& t) {
  if (pp.n_nodes == 0) return true;
  if (pp.n_nodes == 1) return leaf_tile(pp.nodes[0], t);
  uint32_t bits = 0;
  for (int k = 0; k < pp.n_nodes; k++) {
    const ghb_pred_node& nd = pp.nodes[k];
    bool r;
    if (nd.mode == GHB_FILTER_AND)
      r = ((bits >> nd.child[0]) & (bits >> nd.child[1]) & 1u) != 0;
    else if (nd.mode == GHB_FILTER_OR)
      r = (((bits >> nd.child[0]) | (bits >> nd.child[1])) & 1u) != 0;
    else
      r = leaf_tile(nd, t);
    bits |= (uint32_t)r << k;
  }
  return (bits >> (pp.n_nodes - 1)) & 1u;
}

// Merges one partial accumulator word `w` (and its compensation `wc`) into a cell.
__device__ __forceinline__ void acc_merge(int8_t kind, uint64_t* cell, int64_t stride, uint64_t w,
                                          uint64_t wc) {
  switch (kind) {
    case A_CNT_STAR:
    case A_CNT_NN:
    case A_SUM_I:
      if (w) atomicAdd((unsigned long long*)cell, (unsigned long long)w);
      break;
    case A_SUM_F:
      atomic_add_comp(cell, cell + stride, __longlong_as_double(w));
      if (wc && __longlong_as_double(wc) != 0.0) atomicAdd((double*)(cell + stride), __longlong_as_double(wc));
      break;
    case A_MAX_O:
    case A_MIN_O:
      if (w) atomicMax((unsigned long long*)cell, (unsigned long long)w);
      break;
    default: break;
  }
}

// Loads tile `tile` into the stage at `stage` with plain loads by all
// threads (a partial last tile, or unaligned columns).  Ends with a barrier.
__device__ __forceinline__ void load_tile_plain(const GbParams& p, unsigned char* stage, int64_t tile) {
  const int64_t base = tile * p.tile_rows;
  const int rows = (int)min((int64_t)p.tile_rows, p.n - base);
  for (int c = 0; c < p.cols.n; c++) {
    if (p.col_off[c] < 0) continue;
    const ghb_column& col = p.cols.c[c];
    if (col.type == GHB_INT) {
      int32_t* d = (int32_t*)(stage + p.col_off[c]);
      for (int r = threadIdx.x; r < rows; r += blockDim.x) d[r] = __ldcs((const int*)col.data + base + r);
    } else {
      long long* d = (long long*)(stage + p.col_off[c]);
      for (int r = threadIdx.x; r < rows; r += blockDim.x) d[r] = __ldcs((const long long*)col.data + base + r);
    }
    if (p.null_off[c] >= 0)
      for (int r = threadIdx.x; r < rows; r += blockDim.x) stage[p.null_off[c] + r] = col.is_null[base + r];
  }
  __syncthreads();
}

// Thread 0: issues the bulk copies of full tile `tile` into `stage`.
__device__ __forceinline__ void load_tile_bulk(const GbParams& p, unsigned char* stage, int64_t tile,
                                               uint64_t* bar) {
  const int64_t base = tile * p.tile_rows;
  mbar_expect_tx(bar, (uint32_t)p.tx_bytes);
  for (int c = 0; c < p.cols.n; c++) {
    if (p.col_off[c] < 0) continue;
    const ghb_column& col = p.cols.c[c];
    const int w = col.type == GHB_INT ? 4 : 8;
    bulk_g2s(stage + p.col_off[c], (const unsigned char*)col.data + base * w, (uint32_t)(p.tile_rows * w), bar);
    if (p.null_off[c] >= 0)
      bulk_g2s(stage + p.null_off[c], col.is_null + base, (uint32_t)p.tile_rows, bar);
  }
}

template <bool KEYED, bool NULLABLE>
__global__ void __launch_bounds__(kGbThreads) gb_fold_kernel(GbParams p) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int S = p.smem_slots;
  const int64_t sstride = S + 2;
  // layout: [stage 0][stage 1][mbarriers][hash keys + accumulators][warp staging]
  // stage s starts at smem_raw + s * stage_bytes
  uint64_t* bars = (uint64_t*)(smem_raw + 2 * (size_t)p.stage_bytes);
  uint64_t* skeys = bars + 2;
  uint64_t* sacc = skeys + sstride;
  uint64_t* wstage = sacc + (int64_t)p.acc.n_acc * sstride + (threadIdx.x >> 5) * 32;
  const int64_t gstride = p.C + 2;
  const int smask_shift = S > 0 ? 64 - __ffs(S) + 1 : 0;   // 64 - log2(S)

  for (int64_t i = threadIdx.x; i < sstride * (1 + p.acc.n_acc); i += blockDim.x) skeys[i] = 0;
  if (threadIdx.x == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    mbar_fence_init();
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) *p.d_out_groups = 0;
  __syncthreads();

  // stage s holds tile blockIdx.x + i * gridDim.x for the i with i % 2 == s
  auto full = [&](int64_t tile) { return (tile + 1) * p.tile_rows <= p.n; };
  uint32_t pending = 0, phase = 0;   // per stage s: bit s = a bulk copy is in flight / its parity
  bool failed = false;
  for (int s = 0; s < 2; s++) {
    int64_t tile = blockIdx.x + (int64_t)s * gridDim.x;
    if (tile >= p.ntiles) break;
    if (p.bulk && full(tile)) {
      if (threadIdx.x == 0) load_tile_bulk(p, smem_raw + s * p.stage_bytes, tile, &bars[s]);
      pending |= 1u << s;
    } else {
      load_tile_plain(p, smem_raw + s * p.stage_bytes, tile);
    }
  }

  for (int64_t it = 0;; it++) {
    const int64_t tile = blockIdx.x + it * gridDim.x;
    if (tile >= p.ntiles) break;
    const int s = (int)(it & 1);
    if ((pending >> s) & 1u) {
      bool ok = mbar_wait(&bars[s], (phase >> s) & 1u, p.status);
      // one decision for the whole CTA: every thread leaves or none does
      if (__syncthreads_or(!ok)) {
        failed = true;
        break;
      }
      phase ^= 1u << s;
      pending &= ~(1u << s);
    }
    const unsigned char* stage = smem_raw + s * p.stage_bytes;
    const int rows = (int)min((int64_t)p.tile_rows, p.n - tile * p.tile_rows);
    // Phase A, per row: predicate, key, slot (shared table, else global).
    // The trip counts are warp-uniform so the warp-cooperative path can use
    // all lanes.
    const int rpt = p.tile_rows / (int)blockDim.x;   // 1 or 2
    int64_t slot[kGbRows];
    bool live[kGbRows], in_s[kGbRows];
    unsigned peers[kGbRows];
#pragma unroll
    for (int j = 0; j < kGbRows; j++) {
      live[j] = in_s[j] = false;
      slot[j] = -1;
      peers[j] = 0;
      if (j >= rpt) continue;
      const int r = j * blockDim.x + threadIdx.x;
      TileRow t{&p, stage, r};
      bool lv = r < rows && pred_tile(p.pred, t);
      uint64_t u = 0;
      int side = -1;  // 0: key INT64_MIN, 1: NULL key / global aggregate
      if (lv) {
        if (KEYED) {
          int64_t raw = t.raw(p.key_col);
          if (NULLABLE && t.null(p.key_col, raw)) side = 1;
          else {
            u = flip_i64(raw);
            if (u == 0) side = 0;
          }
        } else {
          side = 1;
        }
      }
      int64_t ss = -1;
      if (lv && S > 0) ss = side >= 0 ? S + side : table_insert(skeys, S - 1, smask_shift, u, 8);
      if (lv && ss < 0) {
        int64_t g = side >= 0 ? p.C + side : table_insert(p.gkeys, p.C - 1, p.gshift, u, p.gprobe);
        if (g < 0) {
          raise_status(p.status, kDevCapacity);
          lv = false;
        }
        slot[j] = g;
      } else {
        slot[j] = ss;
      }
      live[j] = lv;
      in_s[j] = lv && ss >= 0;
      if (p.warp_agg) peers[j] = __match_any_sync(0xffffffffu, in_s[j] ? ss : -1);
    }
    // Phase B, per accumulator: its kind and column type are the same for
    // every row, so the branches are uniform; each row adds its contribution.
    for (int a = 0; a < p.acc.n_acc; a++) {
      const int8_t kind = p.acc.kind[a];
      if (kind == A_COMP_F) continue;
      const int c = p.acc.col[a];
      const int type = kind == A_CNT_STAR ? GHB_LONG : p.cols.c[c].type;
      const unsigned char* cb = kind == A_CNT_STAR ? stage : stage + p.col_off[c];
#pragma unroll
      for (int j = 0; j < kGbRows; j++) {
        if (j >= rpt) continue;
        const int r = j * blockDim.x + threadIdx.x;
        uint64_t w = 0;
        if (live[j]) {
          if (kind == A_CNT_STAR) {
            w = 1;
          } else {
            int64_t v = type == GHB_INT ? (int64_t)((const int32_t*)cb)[r] : ((const long long*)cb)[r];
            TileRow t{&p, stage, r};
            if (!(NULLABLE && t.null(c, v))) {
              switch (kind) {
                case A_CNT_NN: w = 1; break;
                case A_SUM_I: w = (uint64_t)v; break;
                case A_SUM_F: w = (uint64_t)__double_as_longlong(raw_to_f64(type, v)); break;
                case A_MAX_O: w = order_image(type, v); break;
                default: w = ~order_image(type, v); break;  // A_MIN_O
              }
            }
          }
        }
        if (p.warp_agg) {
          // lanes of one shared slot combine first; the lowest applies it
          wstage[threadIdx.x & 31] = in_s[j] ? w : 0;
          __syncwarp();
          if (in_s[j] && (threadIdx.x & 31) == __ffs(peers[j]) - 1) {
            uint64_t tot = 0, comp = 0;
            double sf = 0.0, cf = 0.0;
            for (unsigned m = peers[j]; m; m &= m - 1) {
              uint64_t x = wstage[__ffs(m) - 1];
              if (kind == A_SUM_F) {
                double xv = __longlong_as_double(x);
                double tt = __dadd_rn(sf, xv);
                cf = __dadd_rn(cf, two_sum_err(sf, xv, tt));
                sf = tt;
              } else if (kind == A_MAX_O || kind == A_MIN_O) {
                tot = max(tot, x);
              } else {
                tot += x;
              }
            }
            if (kind == A_SUM_F) {
              tot = (uint64_t)__double_as_longlong(sf);
              comp = (uint64_t)__double_as_longlong(cf);
            }
            acc_merge(kind, sacc + a * sstride + slot[j], sstride, tot, comp);
          }
          __syncwarp();
          if (live[j] && !in_s[j]) acc_merge(kind, p.gacc + a * gstride + slot[j], gstride, w, 0);
        } else if (live[j]) {
          uint64_t* cell = in_s[j] ? sacc + a * sstride + slot[j] : p.gacc + a * gstride + slot[j];
          acc_merge(kind, cell, in_s[j] ? sstride : gstride, w, 0);
        }
      }
    }
    __syncthreads();  // every thread is done with this stage
    const int64_t next = tile + 2 * (int64_t)gridDim.x;
    if (next < p.ntiles) {
      if (p.bulk && full(next)) {
        if (threadIdx.x == 0) {
          fence_proxy_async_smem();
          load_tile_bulk(p, smem_raw + s * p.stage_bytes, next, &bars[s]);
        }
        pending |= 1u << s;
      } else {
        load_tile_plain(p, smem_raw + s * p.stage_bytes, next);
      }
    }
  }
  if (failed) {
    // a bulk copy never completed: wait (bounded) for the other stage's copy
    // before the CTA's shared memory goes away
    for (int s = 0; s < 2; s++)
      if ((pending >> s) & 1u) mbar_wait(&bars[s], (phase >> s) & 1u, p.status);
    return;
  }
  __syncthreads();

  // merge the shared table into the global one
  for (int64_t s = threadIdx.x; s < sstride && S > 0; s += blockDim.x) {
    if (sacc[s] == 0) continue;  // accumulator 0 is COUNT(*): empty slot
    int64_t g;
    if (s < S) {
      g = table_insert(p.gkeys, p.C - 1, p.gshift, skeys[s], p.gprobe);
      if (g < 0) {
        raise_status(p.status, kDevCapacity);
        continue;
      }
    } else {
      g = p.C + (s - S);
    }
    for (int a = 0; a < p.acc.n_acc; a++) {
      int8_t kind = p.acc.kind[a];
      if (kind == A_COMP_F) continue;
      uint64_t w = sacc[a * sstride + s];
      uint64_t wc = kind == A_SUM_F ? sacc[(a + 1) * sstride + s] : 0;
      acc_merge(kind, p.gacc + a * gstride + g, gstride, w, wc);
    }
  }
}

__device__ __forceinline__ void write_out(const ghb_out_column& o, int64_t row, bool null,
                                          int64_t iv, double dv) {
  if (o.is_null) o.is_null[row] = null ? 1 : 0;
  switch (o.type) {
    case GHB_LONG: ((int64_t*)o.data)[row] = null ? INT64_MAX : iv; break;
    case GHB_INT: ((int32_t*)o.data)[row] = null ? INT32_MAX : (int32_t)iv; break;
    case GHB_DOUBLE: ((double*)o.data)[row] = null ? __longlong_as_double(0x7ff8000000000000ll) : dv; break;
  }
}

__device__ __forceinline__ int64_t decode_order(int type, uint64_t img) {
  return type == GHB_DOUBLE ? (int64_t)unflip_f64_bits(img) : (int64_t)(img ^ 0x8000000000000000ull);
}

__global__ void gb_finalize_kernel(FinParams f) {
  const int64_t stride = f.C + 2;
  for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < stride;
       s += (int64_t)gridDim.x * blockDim.x) {
    uint64_t cnt = f.gacc[s];
    bool emit = cnt != 0 || (f.key_type < 0 && s == f.C + 1);
    if (emit && (f.key_type >= 0 || s == f.C + 1)) {
      int64_t row = (int64_t)atomicAdd((unsigned long long*)f.d_out_groups, 1ull);
      if (row < f.cap) {
        if (f.key_type >= 0) {
          bool knull = s == f.C + 1;
          int64_t raw = s == f.C ? INT64_MIN : (int64_t)(f.gkeys_ro[s] ^ 0x8000000000000000ull);
          write_out(f.key_out, row, knull, raw, __longlong_as_double(raw));
        }
        for (int a = 0; a < f.naggs; a++) {
          const OutAgg& d = f.agg[a];
          uint64_t v = f.gacc[d.acc_val * stride + s];
          bool null = f.gacc[d.acc_cnt * stride + s] == 0;
          int64_t iv = 0;
          double dv = 0.0;
          switch (d.type) {
            case GHB_AGG_CNT: null = false; iv = (int64_t)v; break;
            case GHB_AGG_SUM:
              if (d.in_type == GHB_DOUBLE)
                dv = __longlong_as_double(v) + __longlong_as_double(f.gacc[(d.acc_val + 1) * stride + s]);
              else
                iv = (int64_t)v;
              break;
            case GHB_AGG_AVG: {
              double sum = __longlong_as_double(v) + __longlong_as_double(f.gacc[(d.acc_val + 1) * stride + s]);
              uint64_t c = f.gacc[d.acc_cnt * stride + s];
              dv = c ? sum / (double)c : 0.0;
              break;
            }
            case GHB_AGG_MIN:
            case GHB_AGG_MAX: {
              uint64_t img = d.type == GHB_AGG_MIN ? ~v : v;
              iv = decode_order(d.in_type, img);
              dv = __longlong_as_double(iv);
              break;
            }
          }
          write_out(f.out[a], row, null, iv, dv);
        }
      } else {
        raise_status(f.status, kDevCapacity);
      }
    }
    // leave the slot zeroed for the next call
    if (cnt != 0 || s >= f.C) {
      f.gkeys[s] = 0;
      for (int a = 0; a < f.n_acc; a++) f.gacc[a * stride + s] = 0;
    } else if (f.gkeys[s] != 0) {
      f.gkeys[s] = 0;
    }
  }
}

// ---------------------------------------------------------------- host
struct GbPlan {
  AccPlan acc;
  FinParams fin;
};

// Index of accumulator (k, col), adding it (and its compensation word for a
// double sum) when absent; -1 when the plan has no room left.
static int add_acc(AccPlan& ap, AccKind k, int col) {
  for (int a = 0; a < ap.n_acc; a++)
    if (ap.kind[a] == k && ap.col[a] == col) return a;
  if (ap.n_acc + (k == A_SUM_F ? 2 : 1) > kMaxAcc) return -1;
  int a = ap.n_acc++;
  ap.kind[a] = k;
  ap.col[a] = (int8_t)col;
  if (k == A_SUM_F) {
    ap.kind[ap.n_acc] = A_COMP_F;
    ap.col[ap.n_acc] = (int8_t)col;
    ap.n_acc++;
  }
  return a;
}

static int32_t plan_aggs(ghb_ctx* ctx, const ghb_column* cols, int32_t ncols,
                         const ghb_agg_desc* aggs, int32_t naggs, const ghb_out_column* out,
                         int32_t nkeys, GbPlan* plan) {
  if (naggs < 0 || naggs > kMaxAggs)
    return set_error(ctx, GHB_ERR_INVALID, "naggs=%d outside [0,%d]", naggs, kMaxAggs);
  AccPlan& ap = plan->acc;
  ap.n_acc = 0;
  add_acc(ap, A_CNT_STAR, -1);
  for (int i = 0; i < naggs; i++) {
    const ghb_agg_desc& d = aggs[i];
    OutAgg& o = plan->fin.agg[i];
    o.type = (int8_t)d.type;
    bool star = d.type == GHB_AGG_CNT && d.col < 0;
    if (!star && (d.col < 0 || d.col >= ncols))
      return set_error(ctx, GHB_ERR_INVALID, "aggregate %d: column %d out of range", i, d.col);
    const ghb_column* c = star ? nullptr : &cols[d.col];
    o.in_type = (int8_t)(c ? c->type : GHB_LONG);
    int cnt = 0;
    if (c && c->null_mode != GHB_NULLS_NONE) cnt = add_acc(ap, A_CNT_NN, d.col);
    o.acc_cnt = (int8_t)cnt;
    int32_t want_out;
    switch (d.type) {
      case GHB_AGG_CNT:
        o.acc_val = (int8_t)cnt;
        want_out = GHB_LONG;
        break;
      case GHB_AGG_SUM:
        if (c->type == GHB_DOUBLE) {
          o.acc_val = (int8_t)add_acc(ap, A_SUM_F, d.col);
          want_out = GHB_DOUBLE;
        } else {
          o.acc_val = (int8_t)add_acc(ap, A_SUM_I, d.col);
          want_out = GHB_LONG;
        }
        break;
      case GHB_AGG_AVG:
        o.acc_val = (int8_t)add_acc(ap, A_SUM_F, d.col);
        want_out = GHB_DOUBLE;
        break;
      case GHB_AGG_MIN:
        o.acc_val = (int8_t)add_acc(ap, A_MIN_O, d.col);
        want_out = c->type;
        break;
      case GHB_AGG_MAX:
        o.acc_val = (int8_t)add_acc(ap, A_MAX_O, d.col);
        want_out = c->type;
        break;
      default:
        return set_error(ctx, GHB_ERR_UNSUPPORTED, "aggregate %d: type %d not supported", i, d.type);
    }
    if (cnt < 0 || o.acc_val < 0)
      return set_error(ctx, GHB_ERR_UNSUPPORTED, "more than %d accumulator words per group", kMaxAcc);
    const ghb_out_column& oc = out[nkeys + i];
    if (oc.type != want_out)
      return set_error(ctx, GHB_ERR_INVALID, "aggregate %d: output column type %d, expected %d", i,
                       oc.type, want_out);
    if (!oc.data) return set_error(ctx, GHB_ERR_INVALID, "aggregate %d: output data is NULL", i);
    plan->fin.out[i] = oc;
  }
  plan->fin.naggs = naggs;
  plan->fin.n_acc = ap.n_acc;
  return GHB_OK;
}

static int64_t next_pow2(int64_t v) {
  int64_t p = 1;
  while (p < v) p <<= 1;
  return p;
}

static int log2_exact(int64_t v) {
  int l = 0;
  while ((1ll << l) < v) l++;
  return l;
}

// Shared implementation; `fixed_table` (nullable) replaces the context's table.
int32_t filter_groupby_impl(ghb_ctx* ctx, const ghb_predicate* pred, const ghb_column* cols,
                            int32_t ncols, const int32_t* key_cols, int32_t nkeys,
                            const ghb_agg_desc* aggs, int32_t naggs, ghb_out_column* out,
                            int64_t out_capacity, int64_t* d_out_groups,
                            const ghb_groupby_cfg* cfg, cudaStream_t stream,
                            void* fixed_table, size_t fixed_table_bytes) {
  if (!ctx) return GHB_ERR_INVALID;
  int64_t n = 0;
  int32_t st = validate_columns(ctx, cols, ncols, &n);
  if (st) return st;
  if (nkeys < 0 || nkeys > 1)
    return set_error(ctx, GHB_ERR_UNSUPPORTED, "nkeys=%d: the device group-by takes 0 or 1 key column", nkeys);
  if (nkeys == 1 && (!key_cols || key_cols[0] < 0 || key_cols[0] >= ncols))
    return set_error(ctx, GHB_ERR_INVALID, "key column out of range");
  if (naggs > 0 && !aggs) return set_error(ctx, GHB_ERR_INVALID, "aggs is NULL");
  if ((nkeys + naggs) > 0 && !out) return set_error(ctx, GHB_ERR_INVALID, "out is NULL");
  if (!d_out_groups) return set_error(ctx, GHB_ERR_INVALID, "d_out_groups is NULL");
  if (out_capacity < 1) return set_error(ctx, GHB_ERR_INVALID, "out_capacity must be >= 1");

  GbParams p;
  std::memset(&p, 0, sizeof(p));
  GbPlan plan;
  std::memset(&plan, 0, sizeof(plan));
  st = plan_aggs(ctx, cols, ncols, aggs, naggs, out, nkeys, &plan);
  if (st) return st;
  st = build_pred_prog(ctx, pred, ncols, &p.pred);
  if (st) return st;
  for (int i = 0; i < ncols; i++) p.cols.c[i] = cols[i];
  p.cols.n = ncols;
  p.acc = plan.acc;
  p.n = n;
  p.key_col = nkeys ? key_cols[0] : -1;
  if (nkeys) {
    if (out[0].type != cols[key_cols[0]].type)
      return set_error(ctx, GHB_ERR_INVALID, "key output column type %d, expected %d", out[0].type,
                       cols[key_cols[0]].type);
    if (!out[0].data) return set_error(ctx, GHB_ERR_INVALID, "key output data is NULL");
  }

  // columns the kernel reads: predicate leaves, the key, aggregate inputs
  bool used[kMaxCols] = {false};
  for (int k = 0; k < p.pred.n_nodes; k++) {
    const ghb_pred_node& nd = p.pred.nodes[k];
    if (nd.mode == GHB_FILTER_AND || nd.mode == GHB_FILTER_OR) continue;
    used[nd.col] = true;
    if (nd.col2 >= 0) used[nd.col2] = true;
  }
  if (nkeys) used[key_cols[0]] = true;
  for (int a = 0; a < p.acc.n_acc; a++)
    if (p.acc.col[a] >= 0) used[p.acc.col[a]] = true;

  int64_t max_groups = (cfg && cfg->max_groups > 0) ? cfg->max_groups : out_capacity;
  if (nkeys == 0) max_groups = 1;
  max_groups = std::min<int64_t>(max_groups, std::max<int64_t>(n, 1));
  int64_t C = (cfg && cfg->global_slots_log2 > 0) ? (1ll << cfg->global_slots_log2)
                                                   : next_pow2(std::max<int64_t>(2 * max_groups, 64));
  int S;
  if (cfg && cfg->smem_slots < 0) S = 0;
  else if (cfg && cfg->smem_slots > 0) S = (int)next_pow2(cfg->smem_slots);
  else S = (int)std::min<int64_t>(4096, next_pow2(std::max<int64_t>(2 * max_groups, 64)));
  if (nkeys == 0) S = 64;
  const int threads = kGbThreads;

  // tile rows: as large as shared memory allows next to the hash table
  size_t row_bytes = 0;
  for (int c = 0; c < ncols; c++)
    if (used[c]) row_bytes += type_width(cols[c].type) + (cols[c].null_mode == GHB_NULLS_BYTEMAP ? 1 : 0);
  const size_t smem_cap = 225 * 1024;
  auto table_bytes_smem = [&](int s) {
    return (size_t)(s + 2) * 8 * (1 + p.acc.n_acc) + (size_t)(threads / 32) * 32 * 8 + 64;
  };
  int tile_rows = 2048;
  while (S > 64 && table_bytes_smem(S) + 2 * row_bytes * 1024 > smem_cap) S /= 2;
  while (tile_rows > threads && table_bytes_smem(S) + 2 * row_bytes * tile_rows > smem_cap) tile_rows /= 2;
  if (table_bytes_smem(S) + 2 * row_bytes * tile_rows > smem_cap)
    return set_error(ctx, GHB_ERR_UNSUPPORTED, "rows of %zu bytes do not fit a shared-memory tile", row_bytes);
  p.smem_slots = S;
  p.warp_agg = (nkeys == 0 || max_groups <= 64) ? 1 : 0;
  p.tile_rows = tile_rows;
  p.ntiles = (n + tile_rows - 1) / tile_rows;
  int32_t off = 0;
  bool aligned = true;
  for (int c = 0; c < kMaxCols; c++) {
    p.col_off[c] = -1;
    p.null_off[c] = -1;
  }
  for (int c = 0; c < ncols; c++) {
    if (!used[c]) continue;
    p.col_off[c] = off;
    off += (int32_t)(tile_rows * type_width(cols[c].type));
    if ((uintptr_t)cols[c].data % 16) aligned = false;
    if (cols[c].null_mode == GHB_NULLS_BYTEMAP) {
      p.null_off[c] = off;
      off += tile_rows;
      if ((uintptr_t)cols[c].is_null % 16) aligned = false;
    }
  }
  p.stage_bytes = (off + 127) & ~127;
  p.tx_bytes = off;
  p.bulk = aligned ? 1 : 0;
  size_t smem = 2 * (size_t)p.stage_bytes + table_bytes_smem(S);

  size_t table_bytes = (size_t)(C + 2) * 8 * (1 + p.acc.n_acc);
  if (fixed_table) {
    if (table_bytes > fixed_table_bytes)
      return set_error(ctx, GHB_ERR_CAPACITY, "group-by table needs %zu bytes, %zu available",
                       table_bytes, fixed_table_bytes);
    // a caller-provided table may hold anything: clear the part this call uses
    GHB_CUDA_TRY(ctx, cudaMemsetAsync(fixed_table, 0, table_bytes, stream));
    p.gkeys = (uint64_t*)fixed_table;
  } else {
    if (table_bytes > ctx->gb_bytes || ctx->gb_dirty || !ctx->gb_table) {
      if (table_bytes > ctx->gb_bytes) {
        GHB_CUDA_TRY(ctx, cudaStreamSynchronize(stream));
        if (ctx->gb_table) cudaFree(ctx->gb_table);
        ctx->gb_table = nullptr;
        ctx->gb_bytes = 0;
        size_t want = std::max(table_bytes, (size_t)1 << 20);
        if (cudaMalloc(&ctx->gb_table, want) != cudaSuccess) {
          cudaGetLastError();
          return set_error(ctx, GHB_ERR_OOM, "cannot allocate a %zu-byte group-by table", want);
        }
        ctx->gb_bytes = want;
      }
      GHB_CUDA_TRY(ctx, cudaMemsetAsync(ctx->gb_table, 0, ctx->gb_bytes, stream));
      ctx->gb_dirty = false;
    }
    p.gkeys = (uint64_t*)ctx->gb_table;
  }
  p.gacc = p.gkeys + (C + 2);
  p.C = C;
  p.gshift = 64 - log2_exact(C);
  p.gprobe = (int32_t)std::min<int64_t>(C, 1 << 20);
  p.status = ctx->d_status;
  p.d_out_groups = d_out_groups;

  int blocks_per_sm = 0;
  bool nullable = false;
  for (int c = 0; c < ncols; c++) nullable |= used[c] && cols[c].null_mode != GHB_NULLS_NONE;
  auto kfn = nkeys ? (nullable ? gb_fold_kernel<true, true> : gb_fold_kernel<true, false>)
                   : (nullable ? gb_fold_kernel<false, true> : gb_fold_kernel<false, false>);
  GHB_CUDA_TRY(ctx, cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  GHB_CUDA_TRY(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, kfn, threads, smem));
  blocks_per_sm = std::max(1, blocks_per_sm);
  if (cfg && cfg->ctas_per_sm > 0) blocks_per_sm = std::min(blocks_per_sm, cfg->ctas_per_sm);
  int grid = (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)ctx->num_sms * blocks_per_sm, p.ntiles));
  kfn<<<grid, threads, smem, stream>>>(p);
  GHB_LAUNCH_CHECK(ctx);

  FinParams& f = plan.fin;
  f.gkeys_ro = p.gkeys;
  f.gkeys = p.gkeys;
  f.gacc = p.gacc;
  f.C = C;
  f.key_type = nkeys ? cols[key_cols[0]].type : -1;
  if (nkeys) f.key_out = out[0];
  f.cap = out_capacity;
  f.d_out_groups = d_out_groups;
  f.status = ctx->d_status;
  int fthreads = 256;
  int fgrid = (int)std::min<int64_t>((C + 2 + fthreads - 1) / fthreads, (int64_t)ctx->num_sms * 8);
  gb_finalize_kernel<<<fgrid, fthreads, 0, stream>>>(f);
  GHB_LAUNCH_CHECK(ctx);
  return GHB_OK;
}

}  // namespace ghb

using namespace ghb;

extern "C" int32_t ghb_filter_groupby(ghb_ctx* ctx, const ghb_predicate* pred, const ghb_column* cols,
                                      int32_t ncols, const int32_t* key_cols, int32_t nkeys,
                                      const ghb_agg_desc* aggs, int32_t naggs, ghb_out_column* out,
                                      int64_t out_capacity, int64_t* d_out_groups,
                                      const ghb_groupby_cfg* cfg, void* stream) {
  if (!ctx) return GHB_ERR_INVALID;
  scratch_reset(ctx);
  return filter_groupby_impl(ctx, pred, cols, ncols, key_cols, nkeys, aggs, naggs, out, out_capacity,
                             d_out_groups, cfg, (cudaStream_t)stream, nullptr, 0);
}
