// ghb_groupby.cuh — the group-by fold and finalize code shared by the
// single-call operator (ghb_groupby.cu) and the batched one (ghb_batch.cu).
//
// Semantics follow Hive's UDAFs (VectorUDAFSum.txt:59-71, VectorUDAFAvg.txt:
// 56-71, VectorUDAFMinMax.txt:65-72): SUM over integers wraps silently, SUM
// and AVG over doubles are double sums, an aggregate that saw only NULLs is
// NULL, COUNT(*) counts rows, COUNT(col) counts non-NULL values.  Double sums
// are accumulated with an error-free transformation: every atomicAdd returns
// the old value, so the adding thread knows the exact rounding error of that
// addition (Knuth's TwoSum) and adds it to a companion compensation word;
// sum + compensation is then accurate to ~1 ulp whatever the order.
//
// Global table (one per operator instance, in HBM):
//   records  [(C + 2) * R] uint64: record s = stored key (flip_i64 of the raw
//            key, 0 = empty), then the R - 1 accumulators of the group, so all
//            the atomics of one row land in one or two cache lines.  Record C
//            holds the key INT64_MIN (whose image is the empty marker), record
//            C + 1 the NULL key, or the single group of a global aggregate.
//   growc    uint64: output rows handed out by the finalize
//   done     uint64: finalize CTAs finished (the last one resets the counters)
//   bits     [C / 32] uint32: a bit per hashed slot, set when the slot is
//            claimed, so the finalize visits the groups and not the table
// Everything is zero between calls: the finalize zeroes each record it emits
// and each bitmap word it reads.
#pragma once

#ifndef __CUDACC_RTC__
#include "ghb_ctx.hpp"
#else
#include "ghb_internal.cuh"
#endif

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
constexpr int kGbThreads = 1024;  // largest CTA of the fold kernels
constexpr int kGbRows = 4;        // tile rows per thread at most
constexpr int kGbMaxSlots = 8192; // shared-memory slots per CTA at most
constexpr int kGbMaxStages = 8;    // tile stages of the single-call fold at most
constexpr int kGbCtrlBytes = 256;  // fold kernels' control words (mbarriers, counters) in shared memory

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

// Everything the fold needs for one operator instance.
struct GbParams {
  ColSet cols;
  PredProg pred;
  AccPlan acc;
  int32_t key_col;       // -1: global aggregate (all rows in one group)
  int32_t smem_slots;    // power of two, 0 = no shared stage
  int32_t warp_agg;      // combine equal keys within a warp before the atomics
  int32_t R;             // words per global record (1 + n_acc)
  int64_t n;
  uint64_t* grec;        // [(C + 2) * R]
  uint32_t* gbits;       // [C / 32]
  int64_t C;             // power of two, >= 64
  int32_t gshift;        // 64 - log2(C)
  int32_t gprobe;        // probe limit in the global table
  int32_t* status;
  // column tiles in shared memory
  int32_t tile_rows;     // rows per tile: the block size times 1, 2 or 4
  int32_t stage_bytes;   // bytes of one stage (128-byte multiple)
  int64_t ntiles;
  int32_t tx_bytes;      // bytes the bulk copies of one full tile deliver
  int32_t bulk;          // column bases are 16-byte aligned: full tiles arrive by bulk copy
  int32_t col_off[kMaxCols];   // byte offset of a used column's tile in a stage, -1 unused
  int32_t null_off[kMaxCols];  // byte offset of a BYTEMAP column's null bytes, -1 none
  int32_t nstages;       // shared-memory stages of the single-call fold (2..kGbMaxStages)
  int32_t table_words;   // 64-bit words of shared memory reserved for the shared table
};

static_assert(sizeof(GbParams) % 8 == 0, "the batched fold copies GbParams as 64-bit words");

// Everything the finalize needs for one operator instance.
struct FinParams {
  uint64_t* grec;
  uint32_t* gbits;
  unsigned long long* growc;
  unsigned long long* done;
  int64_t C;
  int32_t R;
  int32_t key_type;      // -1: global aggregate
  ghb_out_column key_out;
  int32_t naggs;
  OutAgg agg[kMaxAggs];
  ghb_out_column out[kMaxAggs];
  int64_t cap;
  int64_t* d_out_groups;
  int32_t* status;
};

#ifndef __CUDACC_RTC__
// Bytes of the global table of C hashed slots and R words per record.
inline size_t gb_table_bytes(int64_t C, int32_t R) {
  return (size_t)(C + 2) * R * 8 + 16 + (size_t)(C / 32) * 4;
}

// Points p/f at a zeroed table of gb_table_bytes(C, R) bytes at `base`.
inline void gb_table_bind(void* base, int64_t C, int32_t R, GbParams* p, FinParams* f) {
  uint64_t* rec = (uint64_t*)base;
  unsigned long long* ctr = (unsigned long long*)(rec + (size_t)(C + 2) * R);
  p->grec = rec;
  p->gbits = (uint32_t*)(ctr + 2);
  f->grec = rec;
  f->gbits = p->gbits;
  f->growc = ctr;
  f->done = ctr + 1;
  f->C = C;
  f->R = R;
}

#endif

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

// Find-or-insert of a non-zero key image in the shared table (linear
// probing); the slot, or -1 after max_probe probes.
__device__ __forceinline__ int smem_insert(uint64_t* keys, int mask, int shift, uint64_t u, int max_probe) {
  int h = (int)hslot(u, shift);
  for (int q = 0; q < max_probe; q++) {
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

// Find-or-insert in the global table; a slot that this call claims gets its
// bit in the claimed-slot bitmap.  -1 when the probe limit is reached.
__device__ __forceinline__ int64_t gtable_insert(const GbParams& p, uint64_t u) {
  const int64_t mask = p.C - 1;
  int64_t h = hslot(u, p.gshift);
  for (int q = 0; q < p.gprobe; q++) {
    unsigned long long* kp = (unsigned long long*)(p.grec + h * p.R);
    uint64_t cur = *kp;
    if (cur == u) return h;
    if (cur == 0) {
      unsigned long long prev = atomicCAS(kp, 0ull, (unsigned long long)u);
      if (prev == 0) {
        atomicOr(&p.gbits[h >> 5], 1u << (h & 31));
        return h;
      }
      if (prev == u) return h;
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

// Merges one partial accumulator word `w` (and its compensation `wc`) into a
// cell; a double sum's compensation word sits `stride` words after it.
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

// Shared table of one CTA: S slots (+ 2 side slots) of keys, then n_acc
// arrays of S + 2 accumulators.
__device__ __forceinline__ void smem_table_clear(const GbParams& p, uint64_t* skeys) {
  const int64_t words = (int64_t)(p.smem_slots + 2) * (1 + p.acc.n_acc);
  for (int64_t i = threadIdx.x; i < words; i += blockDim.x) skeys[i] = 0;
}

// Folds the `rows` rows of the tile in `stage` into the shared table (or the
// global one), in two phases:
//   A  per row: predicate, key, slot (shared table, else global);
//   B  per accumulator: its kind and column type are the same for every row,
//      so the branches are uniform; each row adds its contribution.
// `wstage` is this warp's 32 words of staging for the warp-combine path.
template <bool KEYED, bool NULLABLE>
__device__ __forceinline__ void fold_tile(const GbParams& p, const unsigned char* stage, int rows,
                                          uint64_t* skeys, uint64_t* wstage) {
  const int S = p.smem_slots;
  const int64_t sstride = S + 2;
  uint64_t* sacc = skeys + sstride;
  const int smask_shift = S > 0 ? 64 - __ffs(S) + 1 : 0;   // 64 - log2(S)
  const int R = p.R;
  // the trip counts are warp-uniform so the warp-cooperative path can use all lanes
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
    if (lv && S > 0) ss = side >= 0 ? S + side : smem_insert(skeys, S - 1, smask_shift, u, 8);
    if (lv && ss < 0) {
      int64_t g = side >= 0 ? p.C + side : gtable_insert(p, u);
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
        if (live[j] && !in_s[j]) acc_merge(kind, p.grec + slot[j] * R + 1 + a, 1, w, 0);
      } else if (live[j]) {
        if (in_s[j]) acc_merge(kind, sacc + a * sstride + slot[j], sstride, w, 0);
        else acc_merge(kind, p.grec + slot[j] * R + 1 + a, 1, w, 0);
      }
    }
  }
}

// Merges the CTA's shared table into the global one (all threads; the caller
// syncs before and after).
__device__ __forceinline__ void flush_smem_table(const GbParams& p, const uint64_t* skeys) {
  const int S = p.smem_slots;
  const int64_t sstride = S + 2;
  const uint64_t* sacc = skeys + sstride;
  for (int64_t s = threadIdx.x; s < sstride && S > 0; s += blockDim.x) {
    if (sacc[s] == 0) continue;  // accumulator 0 is COUNT(*): empty slot
    int64_t g;
    if (s < S) {
      g = gtable_insert(p, skeys[s]);
      if (g < 0) {
        raise_status(p.status, kDevCapacity);
        continue;
      }
    } else {
      g = p.C + (s - S);
    }
    uint64_t* rec = p.grec + g * p.R + 1;
    for (int a = 0; a < p.acc.n_acc; a++) {
      int8_t kind = p.acc.kind[a];
      if (kind == A_COMP_F) continue;
      uint64_t w = sacc[a * sstride + s];
      uint64_t wc = kind == A_SUM_F ? sacc[(a + 1) * sstride + s] : 0;
      acc_merge(kind, rec + a, 1, w, wc);
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

// Writes the group of record `s` as output row `row` (when it fits) and
// zeroes the record.  `rb` is this thread's row of kMaxAcc + 1 words in
// shared memory: the record's words are all loaded (independent loads, one
// round trip) and parked there before the outputs are computed.
__device__ __forceinline__ void emit_group(const FinParams& f, int64_t s, int64_t row, uint64_t* rb) {
  uint64_t* rec = f.grec + s * f.R;
  uint64_t w[kMaxAcc + 1];
#pragma unroll
  for (int i = 0; i <= kMaxAcc; i++)
    if (i < f.R) w[i] = rec[i];
#pragma unroll
  for (int i = 0; i <= kMaxAcc; i++)
    if (i < f.R) {
      rb[i] = w[i];
      rec[i] = 0;
    }
  const uint64_t* acc = rb + 1;
  if (row < f.cap) {
    if (f.key_type >= 0) {
      bool knull = s == f.C + 1;
      int64_t raw = s == f.C ? INT64_MIN : (int64_t)(rb[0] ^ 0x8000000000000000ull);
      write_out(f.key_out, row, knull, raw, __longlong_as_double(raw));
    }
    for (int a = 0; a < f.naggs; a++) {
      const OutAgg& d = f.agg[a];
      uint64_t v = acc[d.acc_val];
      bool null = acc[d.acc_cnt] == 0;
      int64_t iv = 0;
      double dv = 0.0;
      switch (d.type) {
        case GHB_AGG_CNT: null = false; iv = (int64_t)v; break;
        case GHB_AGG_SUM:
          if (d.in_type == GHB_DOUBLE)
            dv = __longlong_as_double(v) + __longlong_as_double(acc[d.acc_val + 1]);
          else
            iv = (int64_t)v;
          break;
        case GHB_AGG_AVG: {
          double sum = __longlong_as_double(v) + __longlong_as_double(acc[d.acc_val + 1]);
          uint64_t c = acc[d.acc_cnt];
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

// Slots per finalize unit: one CTA of kFinThreads threads, a thread per slot.
constexpr int kFinThreads = 256;
__host__ __device__ inline int64_t fin_units(int64_t C) { return (C + kFinThreads - 1) / kFinThreads; }

// Called by all kFinThreads threads of a CTA for unit `unit` of the table:
// each warp covers one bitmap word (ballot), the CTA takes one block of
// output rows for the unit's claimed slots (one atomic per CTA: per warp,
// a large table's warps would serialise on the counter), each warp clears its
// word, and each lane with a claimed slot emits its group.  `rb` is the CTA's
// record buffer, [kFinThreads][kMaxAcc + 1] words.
__device__ __forceinline__ void finalize_unit(const FinParams& f, int64_t unit, uint64_t* rb) {
  __shared__ uint32_t s_cnt[kFinThreads / 32];
  __shared__ unsigned long long s_base;
  const int64_t s = unit * kFinThreads + threadIdx.x;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t word = s < f.C ? f.gbits[s >> 5] : 0u;   // the same word for the whole warp
  const bool has = (word >> lane) & 1u;
  const unsigned m = __ballot_sync(0xffffffffu, has);
  if (lane == 0) {
    s_cnt[warp] = __popc(m);
    if (m) f.gbits[s >> 5] = 0;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t run = 0;
    for (int w = 0; w < kFinThreads / 32; w++) {
      const uint32_t c = s_cnt[w];
      s_cnt[w] = run;
      run += c;
    }
    s_base = run ? atomicAdd(f.growc, (unsigned long long)run) : 0ull;
  }
  __syncthreads();
  const int64_t row = (int64_t)s_base + s_cnt[warp] + __popc(m & ((1u << lane) - 1u));
  if (has) emit_group(f, s, row, rb + threadIdx.x * (kMaxAcc + 1));
  __syncthreads();   // s_cnt and s_base are reused by the next unit
}

// One thread: the two side records (key INT64_MIN, NULL key); a global
// aggregate always emits its one group.
__device__ __forceinline__ void finalize_sides(const FinParams& f, uint64_t* rb) {
  for (int k = 0; k < 2; k++) {
    const int64_t s = f.C + k;
    const bool emit = f.key_type < 0 ? k == 1 : f.grec[s * f.R + 1] != 0;
    if (emit) emit_group(f, s, (int64_t)atomicAdd(f.growc, 1ull), rb);
  }
}

// The generic folder: fold_tile interprets the predicate program, the key
// and the accumulator plan for every row.
template <bool KEYED, bool NULLABLE>
struct GenericFolder {
  static constexpr bool kNarrow = false;   // 64-bit shared counters: no flush guard
  struct State {};                          // nothing kept per thread between tiles
  __device__ __forceinline__ static void fold(const GbParams& p, const unsigned char* stage, int rows,
                                              uint64_t* skeys, uint64_t* wstage, State&) {
    fold_tile<KEYED, NULLABLE>(p, stage, rows, skeys, wstage);
  }
  __device__ __forceinline__ static void drain(const GbParams&, uint64_t*, State&) {}
  // The shared table of p fits the words the launch reserved.
  __device__ __forceinline__ static bool fits(const GbParams& p) {
    return (int64_t)(p.smem_slots + 2) * (1 + p.acc.n_acc) <= p.table_words;
  }
  __device__ __forceinline__ static void clear(const GbParams& p, uint64_t* skeys) { smem_table_clear(p, skeys); }
  __device__ __forceinline__ static void flush(const GbParams& p, const uint64_t* skeys) {
    flush_smem_table(p, skeys);
  }
};

// A folder whose shared counters are 32-bit (kNarrow) has its table flushed
// and cleared before the rows folded since the last clear could reach 2^32.
constexpr uint64_t kNarrowRowLimit = 0xFFFFFFFFull;

// Body of the single-call fold kernel.  A persistent CTA owns tiles
// blockIdx.x, blockIdx.x + gridDim.x, ...; full tiles stream through
// p.nstages shared-memory stages by bulk copies (cp.async.bulk completing on
// the stage's mbarrier), so up to nstages - 1 tiles are in flight while one
// is folded.  There is no CTA-wide barrier per tile: each warp folds its rows
// of a stage as soon as the stage is full and moves on; the last warp to
// finish a stage issues the copy of the stage's next tile.  A partial last
// tile, or every tile when a column is not 16-byte aligned, is read with plain
// loads after the pipeline.  Folder::fold folds one tile.
template <class Folder>
__device__ __forceinline__ void fold_kernel_body(const GbParams& p) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  // layout: [nstages stages][control][shared table][warp staging]
  const int NS = p.nstages;
  unsigned char* ctrl = smem_raw + (size_t)NS * p.stage_bytes;
  uint64_t* full = (uint64_t*)ctrl;                    // [kGbMaxStages] stage s holds a tile
  uint32_t* done = (uint32_t*)(ctrl + 64);             // [kGbMaxStages] warps done with stage s
  uint32_t* issued = (uint32_t*)(ctrl + 96);           // [kGbMaxStages] copies issued into stage s
  int32_t* gave_up = (int32_t*)(ctrl + 128);           // a wait ran out
  uint64_t* skeys = (uint64_t*)(ctrl + kGbCtrlBytes);
  uint64_t* wstage = skeys + p.table_words + (threadIdx.x >> 5) * 32;
  if (!Folder::fits(p) || NS < 2 || NS > kGbMaxStages) {   // a layout the host did not reserve
    if (threadIdx.x == 0) raise_status(p.status, GHB_ERR_INVALID);
    return;
  }

  Folder::clear(p, skeys);
  typename Folder::State st{};   // per-thread partial aggregates of the folder, if it keeps any
  if (threadIdx.x < kGbMaxStages) {
    done[threadIdx.x] = 0;
    issued[threadIdx.x] = 0;
  }
  if (threadIdx.x == 0) {
    for (int s = 0; s < NS; s++) mbar_init(&full[s], 1);
    *gave_up = 0;
    mbar_fence_init();
  }
  __syncthreads();

  auto stage = [&](int s) { return smem_raw + (size_t)s * p.stage_bytes; };
  auto tile_of = [&](int64_t i) { return (int64_t)blockIdx.x + i * (int64_t)gridDim.x; };
  const int64_t mine = p.ntiles > (int64_t)blockIdx.x ? (p.ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  int64_t nfull = p.bulk ? mine : 0;
  if (nfull > 0 && tile_of(nfull - 1) == p.ntiles - 1 && p.n % p.tile_rows != 0) nfull--;

  if (threadIdx.x == 0)
    for (int s = 0; s < NS && s < nfull; s++) {
      load_tile_bulk(p, stage(s), tile_of(s), &full[s]);
      issued[s] = 1;
    }

  const int lane = threadIdx.x & 31;
  const uint32_t nwarps = blockDim.x >> 5;
  int s = 0;          // stage of tile i: i % NS
  uint32_t par = 0;   // parity of its fill: (i / NS) & 1
  for (int64_t i = 0; i < nfull; i++, s = s + 1 == NS ? 0 : s + 1, par ^= s == 0 ? 1u : 0u) {
    bool ok = !__any_sync(0xffffffffu, *(volatile int32_t*)gave_up != 0);
    if (ok) ok = __all_sync(0xffffffffu, mbar_wait(&full[s], par, p.status));
    if (!ok) {
      if (lane == 0) atomicExch(gave_up, 1);
      break;
    }
    Folder::fold(p, stage(s), p.tile_rows, skeys, wstage, st);
    // Every value the warp read from the stage has been consumed by the fold
    // (in-order issue waits for a load's result at its first use), so after
    // __syncwarp the warp's reads are complete.  No memory fence here: one
    // would also wait for the warp's global-table atomics still in flight.
    __syncwarp();
    if (lane == 0 && atomicAdd(&done[s], 1u) == nwarps - 1) {
      // every warp is done with stage s: refill it
      atomicExch(&done[s], 0u);
      if (i + NS < nfull && *(volatile int32_t*)gave_up == 0) {
        fence_proxy_async_smem();
        load_tile_bulk(p, stage(s), tile_of(i + NS), &full[s]);
        issued[s]++;
      }
    }
  }
  __syncthreads();
  if (*(volatile int32_t*)gave_up) {
    // wait (bounded) for the copies in flight before the CTA's shared memory goes away
    if (threadIdx.x == 0)
      for (int s = 0; s < NS; s++)
        if (issued[s]) mbar_wait(&full[s], (issued[s] - 1) & 1u, p.status);
    return;
  }
  for (int64_t i = nfull; i < mine; i++) {
    const int64_t tile = tile_of(i);
    load_tile_plain(p, stage(0), tile);
    Folder::fold(p, stage(0), (int)min((int64_t)p.tile_rows, p.n - tile * p.tile_rows), skeys, wstage, st);
    __syncthreads();
  }
  Folder::drain(p, skeys, st);
  __syncthreads();
  Folder::flush(p, skeys);
}


struct BatchChunk {
  int32_t inst;
  int32_t ntiles;
  int64_t tile0;
};

struct BatchParams {
  const GbParams* insts;
  const BatchChunk* chunks;
  int64_t nchunks;
  unsigned long long* claim;   // next chunk to hand out (reset by the finalize)
  int32_t stage_bytes;         // the same for every instance
  int32_t table_words;         // shared-table words reserved per CTA
};

// Shared bytes the batched fold adds to the single-call layout: its
// mbarriers, the active instance's parameters and the claimed chunk.
inline __host__ __device__ constexpr size_t batch_extra_smem() { return sizeof(GbParams) + 32; }

// Body of the batched fold kernel: persistent CTAs claim chunks (a run of
// tiles of one instance) from a global counter; a CTA keeps the current
// instance's parameters and shared table in shared memory and flushes the
// table when the instance changes; two stages, a CTA barrier per tile (a
// per-warp pipeline as in the single-call fold measured slower here: the
// batches' instance switches need the CTA barriers anyway).  Folder::fold
// folds one tile.
template <class Folder>
__device__ __forceinline__ void batch_fold_body(const BatchParams& bp) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  // layout: [stage 0][stage 1][mbarriers][instance params][claim][table][warp staging]
  uint64_t* bars = (uint64_t*)(smem_raw + 2 * (size_t)bp.stage_bytes);
  GbParams* sp = (GbParams*)(bars + 2);
  long long* sclaim = (long long*)(sp + 1);
  uint64_t* skeys = (uint64_t*)(sclaim + 2);
  uint64_t* wstage = skeys + bp.table_words + (threadIdx.x >> 5) * 32;

  if (threadIdx.x == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    mbar_fence_init();
  }
  __syncthreads();

  // The CTA's tile stream: the tiles of the chunk it claimed last.  Every
  // thread holds the same state, so the barriers inside are uniform.
  int32_t c_inst = -1;
  int64_t c_next = 0, c_end = 0;
  bool exhausted = false;
  auto next_tile = [&](int32_t* inst, int64_t* tile) -> bool {
    if (c_next >= c_end) {
      if (exhausted) return false;
      if (threadIdx.x == 0) *sclaim = (long long)atomicAdd(bp.claim, 1ull);
      __syncthreads();
      const long long c = *sclaim;
      __syncthreads();
      if (c >= bp.nchunks) {
        exhausted = true;
        return false;
      }
      const BatchChunk ch = bp.chunks[c];
      c_inst = ch.inst;
      c_next = ch.tile0;
      c_end = ch.tile0 + ch.ntiles;
    }
    *inst = c_inst;
    *tile = c_next++;
    return true;
  };
  // Starts loading a tile into stage s; true when it arrives by bulk copy.
  auto issue = [&](int s, int32_t inst, int64_t tile) -> bool {
    const GbParams& gp = bp.insts[inst];
    unsigned char* stage = smem_raw + s * (size_t)bp.stage_bytes;
    if (gp.bulk && (tile + 1) * gp.tile_rows <= gp.n) {
      if (threadIdx.x == 0) {
        fence_proxy_async_smem();
        load_tile_bulk(gp, stage, tile, &bars[s]);
      }
      return true;
    }
    load_tile_plain(gp, stage, tile);
    return false;
  };

  int32_t q_inst[2] = {-1, -1};
  int64_t q_tile[2] = {0, 0};
  uint32_t valid = 0, pending = 0, phase = 0;
  for (int s = 0; s < 2; s++) {
    if (!next_tile(&q_inst[s], &q_tile[s])) break;
    valid |= 1u << s;
    if (issue(s, q_inst[s], q_tile[s])) pending |= 1u << s;
  }

  int32_t active = -1;
  bool failed = false;
  uint64_t since = 0;   // rows of `active` folded since its shared table was last cleared
  typename Folder::State st{};   // per-thread partial aggregates of the folder, if it keeps any
  for (int64_t it = 0;; it++) {
    const int s = (int)(it & 1);
    if (!((valid >> s) & 1u)) break;
    const int32_t inst = s ? q_inst[1] : q_inst[0];
    const int64_t tile = s ? q_tile[1] : q_tile[0];
    if (inst != active) {
      if (active >= 0) {
        Folder::drain(*sp, skeys, st);
        __syncthreads();
        Folder::flush(*sp, skeys);
        __syncthreads();
      }
      const uint64_t* src = (const uint64_t*)&bp.insts[inst];
      for (int k = threadIdx.x; k < (int)(sizeof(GbParams) / 8); k += blockDim.x)
        ((uint64_t*)sp)[k] = src[k];
      __syncthreads();
      Folder::clear(*sp, skeys);
      __syncthreads();
      active = inst;
      since = 0;
    }
    if ((pending >> s) & 1u) {
      bool ok = mbar_wait(&bars[s], (phase >> s) & 1u, sp->status);
      if (__syncthreads_or(!ok)) {
        failed = true;
        break;
      }
      phase ^= 1u << s;
      pending &= ~(1u << s);
    }
    const unsigned char* stage = smem_raw + s * (size_t)bp.stage_bytes;
    const int rows = (int)min((int64_t)sp->tile_rows, sp->n - tile * sp->tile_rows);
    Folder::fold(*sp, stage, rows, skeys, wstage, st);
    __syncthreads();  // every thread is done with this stage
    if constexpr (Folder::kNarrow) {
      since += (uint64_t)rows;
      if (since + (uint64_t)sp->tile_rows > kNarrowRowLimit) {
        Folder::drain(*sp, skeys, st);
        __syncthreads();
        Folder::flush(*sp, skeys);
        __syncthreads();
        Folder::clear(*sp, skeys);
        __syncthreads();
        since = 0;
      }
    }
    valid &= ~(1u << s);
    int32_t ni;
    int64_t nt;
    if (next_tile(&ni, &nt)) {
      if (s) {
        q_inst[1] = ni;
        q_tile[1] = nt;
      } else {
        q_inst[0] = ni;
        q_tile[0] = nt;
      }
      valid |= 1u << s;
      if (issue(s, ni, nt)) pending |= 1u << s;
    }
  }
  if (failed) {
    for (int s = 0; s < 2; s++)
      if ((pending >> s) & 1u) mbar_wait(&bars[s], (phase >> s) & 1u, sp->status);
    return;
  }
  __syncthreads();
  if (active >= 0) {
    Folder::drain(*sp, skeys, st);
    __syncthreads();
    Folder::flush(*sp, skeys);
  }
}


#ifndef __CUDACC_RTC__
// ---------------------------------------------------------------- host
struct GbSetup {
  int64_t max_groups;   // table sizing: groups expected (0 = out_capacity)
  int32_t smem_slots;   // -1 none, 0 auto, else power of two
  float load_factor;    // hashed slots = next_pow2(groups / load_factor); 0 = 0.5
  int32_t threads;      // CTA size of the fold (512 or 1024)
  int32_t tile_rows;    // 0 = as large as shared memory allows (threads times 1, 2 or 4)
  int32_t smem_table_slots; // shared-memory slots the layout reserves (0 = smem_slots)
  int32_t warp_agg;     // -1 auto, else 0 / 1
  int32_t extra_smem;   // shared bytes the kernel needs beyond stages, table and staging
  int32_t narrow;       // 1: shared table in the specialised folds' narrow layout
  int32_t nstages;      // tile stages; 0 = as many as useful (single call), the batch uses 2
};

// Validates one instance and fills p and f, except the table pointers (see
// gb_table_bind); *table_bytes is the size of its global table and *smem the
// dynamic shared memory the fold kernel needs.
int32_t gb_setup(ghb_ctx* ctx, const ghb_predicate* pred, const ghb_column* cols, int32_t ncols,
                 const int32_t* key_cols, int32_t nkeys, const ghb_agg_desc* aggs, int32_t naggs,
                 const ghb_out_column* out, int64_t out_capacity, int64_t* d_out_groups,
                 const GbSetup& su, GbParams* p, FinParams* f, size_t* table_bytes, size_t* smem);

int64_t next_pow2_i64(int64_t v);

#endif

}  // namespace ghb
