// ghb_join.cu — device hash equi-join: build (J1) and probe (J2).
//
// Replaces the reference's join, which sorted both inputs' row indices on the
// GPU and merged them single-threaded on the CPU
// (gpu_impl/src/Operator/SortMergeJoinPredicate.cu:8-461), then gathered the
// retained columns on the host (gpu_impl/src/Operator/BaseJoinPredicate.cu:
// 4-97).  Hive's CPU map-join probes a power-of-two open-addressing table
// whose value store holds each build row's retained columns
// (VectorMapJoinFastLongHashTable.java:99-254, VectorMapJoinFastLongHashMap.
// java:71-84).  The device table keeps, per slot, the key, the (first row,
// count) of the rows with that key and the first row's payload words, in
// three arrays (below), under one of two layouts the build chooses on the
// device from the keys' range (join_layout):
//
//   direct  dense keys (a range below twice the rows, the surrogate key of a
//           dimension table): slot = key - min; the probe loads the slot's
//           count, no key array, no bucket scan;
//   hashed  4-slot buckets, Fibonacci-hashed bucket index; slots fill in order
//           inside a bucket and spill to the next bucket (linear probing by
//           buckets), so one 32-byte load of the bucket's keys settles almost
//           every probe.  The key INT64_MIN, whose image is the empty marker,
//           lives in slot 0 of an extra side bucket.
//
// A key that occurs more than once in the build chains its later rows through
// chain[slot] / next[row] (row + 1, 0 ends the chain; pushed with atomicExch)
// and their payloads are read from the build columns.  The default load
// factor is 0.5, below Hive's hive.hashtable.loadfactor (0.75): at 0.75 more
// full buckets send a probe on to the next bucket, and the 60M-row probe
// measured 7% slower.  Keys and results stream with evict-first loads and
// stores.
//
// The probe counts, then writes (two passes over fixed chunks of probe rows,
// no ordering dependency between CTAs):
//   J2a  count: each CTA takes a chunk, loads its keys, issues the table
//        loads of all its rows together, stores each row's slot (-1 = no
//        match) and each warp's output-row count (a warp covers consecutive
//        rows of the chunk);
//   J2b  scan: the warp counts become output offsets (a multi-CTA look-back
//        scan);
//   J2c  write: each warp re-reads its rows' slots, loads each matching
//        slot's payload words, scans its rows' output counts and writes
//        (probe row, build row, payloads) at its offset, in probe-row order.
// Neither pass takes a CTA barrier per chunk.
#include <algorithm>
#include <map>
#include <mutex>

#include "ghb_ctx.hpp"
#include "ghb_log.hpp"

namespace ghb {

// Slot s = bucket * 4 + index (a direct table: key - min).  The slots' fields
// live in three arrays, so each probe pass reads one dense array: the hashed
// count pass only keys (4 per bucket = one 32-byte sector), the direct one
// only the counts, the write pass the payload words and, when it needs them,
// the (first row, count) pairs.
//   key[s]   uint64 key image (flip_i64 of the key, 0 = empty)
//   meta[s]  int2 {first build row + 1, build rows with this key}
//   pay[s]   ulonglong2, the first build row's inline payload words

constexpr int kJThreads = 256;
constexpr int kJItems = 4;
constexpr int kChunk = kJThreads * kJItems;   // probe rows per chunk
constexpr int kMaxPay = GHB_MAX_JOIN_PAYLOAD;
constexpr int kInline = 2;

// Bucket of a key image: Fibonacci (multiplicative) hashing, the top bits of
// u * 2^64/phi.  One 64-bit multiply; consecutive keys land far apart.
__device__ __forceinline__ int64_t bucket_of(unsigned long long u, int shift) {
  return (int64_t)((u * 0x9E3779B97F4A7C15ull) >> shift);
}

struct BuildParams {
  ghb_column key;
  int32_t n_inline;
  ghb_column pay[kInline];
  unsigned long long* kimg;   // key[s] of the layout above
  int2* meta;
  ulonglong2* payw;
  int32_t* chain_p1;     // [slots]
  int32_t* next_p1;      // [build rows]
  int64_t bmask;         // hashed buckets - 1
  int32_t hshift;        // 64 - log2(hashed buckets)
  int64_t side;          // index of the side bucket
  unsigned long long* stats;  // [0] rows stored, [1] max duplicates
  int32_t* status;
  int64_t slots;         // hashed slots allocated (a direct table fits in them)
};

// The table's layout, decided on the device from the build keys' range
// (stats[2] non-NULL keys, stats[3] max of the complemented order images,
// stats[4] max of the order images): dense keys (a range below twice the
// rows and within the allocated slots, the common surrogate key of a
// dimension table) get a direct table, slot = key - min, with no key array
// and no bucket scan on probe; other keys the hashed buckets.  Every thread
// of the build and probe kernels computes the same answer from the same
// words, so no host round trip is needed.
struct JoinLayout {
  bool direct;
  int64_t dmin;
  int64_t drange;
};

__host__ __device__ inline JoinLayout join_layout(const unsigned long long* stats, int64_t build_rows,
                                                  int64_t slots) {
  JoinLayout L{false, 0, 0};
  if (stats[2] == 0) return L;
  const unsigned long long umin = ~stats[3], umax = stats[4];
  const unsigned long long span = umax - umin;   // the images keep the keys' order and distances
  if (span < 2ull * (unsigned long long)build_rows && span < (unsigned long long)slots && span < (1ull << 30)) {
    L.direct = true;
    L.dmin = (int64_t)(umin ^ 0x8000000000000000ull);
    L.drange = (int64_t)span + 1;
  }
  return L;
}

// The build keys' range into stats[2..4] (zeroed with the table).
__global__ void __launch_bounds__(256) join_key_range_kernel(ghb_column key, unsigned long long* stats) {
  unsigned long long cmin = 0, umax = 0, cnt = 0;   // cmin: max of ~image = ~(min image)
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < key.n;
       r += (int64_t)gridDim.x * blockDim.x) {
    const int64_t raw = ld_raw(key, r);
    if (raw_is_null(key, raw, r)) continue;
    const unsigned long long u = flip_i64(raw);
    cmin = max(cmin, ~u);
    umax = max(umax, u);
    cnt++;
  }
  for (int o = 16; o > 0; o >>= 1) {
    cmin = max(cmin, __shfl_down_sync(0xffffffffu, cmin, o));
    umax = max(umax, __shfl_down_sync(0xffffffffu, umax, o));
    cnt += __shfl_down_sync(0xffffffffu, cnt, o);
  }
  // one set of atomics per CTA (the same three words from every warp would
  // serialise at L2)
  __shared__ unsigned long long s_red[3][8];
  const int warp = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    s_red[0][warp] = cmin;
    s_red[1][warp] = umax;
    s_red[2][warp] = cnt;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); w++) {
      cmin = max(cmin, s_red[0][w]);
      umax = max(umax, s_red[1][w]);
      cnt += s_red[2][w];
    }
    if (cnt) {
      atomicMax(&stats[3], cmin);
      atomicMax(&stats[4], umax);
      atomicAdd(&stats[2], cnt);
    }
  }
}

__global__ void __launch_bounds__(256) join_build_kernel(BuildParams p) {
  const JoinLayout L = join_layout(p.stats, p.key.n, p.slots);
  unsigned long long stored = 0, maxdup = 0;
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < p.key.n;
       r += (int64_t)gridDim.x * blockDim.x) {
    int64_t raw = ld_raw(p.key, r);
    if (raw_is_null(p.key, raw, r)) continue;   // NULL keys never join
    unsigned long long u = flip_i64(raw);
    int64_t bk, j = -1;
    if (L.direct) {   // slot = key - dmin: bucket * 4 + j
      const unsigned long long d = (unsigned long long)raw - (unsigned long long)L.dmin;
      bk = (int64_t)(d >> 2);
      j = (int64_t)(d & 3);
    } else if (u == 0) {
      bk = p.side;
      j = 0;
    } else {
      bk = bucket_of(u, p.hshift);
      for (int64_t probes = 0; probes <= p.bmask && j < 0; probes++) {
        for (int q = 0; q < 4; q++) {
          unsigned long long cur = p.kimg[bk * 4 + q];
          if (cur == 0) {
            unsigned long long prev = atomicCAS(&p.kimg[bk * 4 + q], 0ull, u);
            if (prev == 0 || prev == u) { j = q; break; }
            cur = prev;
          }
          if (cur == u) { j = q; break; }
        }
        if (j < 0) bk = (bk + 1) & p.bmask;
      }
      if (j < 0) {   // table full: cannot happen with load factor < 1
        raise_status(p.status, kDevCapacity);
        continue;
      }
    }
    const int64_t slot = bk * 4 + j;
    int old = atomicAdd(&p.meta[slot].y, 1);
    if (old == 0) {
      p.meta[slot].x = (int32_t)(r + 1);
      if (p.n_inline > 0) p.payw[slot].x = (unsigned long long)ld_raw(p.pay[0], r);
      if (p.n_inline > 1) p.payw[slot].y = (unsigned long long)ld_raw(p.pay[1], r);
    } else {
      p.next_p1[r] = atomicExch(&p.chain_p1[slot], (int)(r + 1));
    }
    stored++;
    maxdup = max(maxdup, (unsigned long long)(old + 1));
  }
  // one atomic per CTA for the statistics (per warp, thousands of warps'
  // atomics on two words would serialise at L2)
  for (int o = 16; o > 0; o >>= 1) {
    stored += __shfl_down_sync(0xffffffffu, stored, o);
    maxdup = max(maxdup, __shfl_down_sync(0xffffffffu, maxdup, o));
  }
  __shared__ unsigned long long s_red[2][8];
  const int warp = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    s_red[0][warp] = stored;
    s_red[1][warp] = maxdup;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); w++) {
      stored += s_red[0][w];
      maxdup = max(maxdup, s_red[1][w]);
    }
    if (stored) atomicAdd(&p.stats[0], stored);
    if (maxdup) atomicMax(&p.stats[1], maxdup);
  }
}

// ------------------------------------------------------------------ probe
struct ProbeParams {
  const unsigned long long* kimg;
  const int2* meta;
  const ulonglong2* payw;
  const int32_t* chain_p1;
  const int32_t* next_p1;
  const unsigned long long* stats;
  int64_t bmask;
  int32_t hshift;
  int64_t side;
  ghb_column pkey;
  int32_t join_type;
  int32_t nbp, npp, n_inline;
  int32_t lean;            // INNER, no probe payloads, every build payload inline and non-NULL
  ghb_column bpay[kMaxPay];
  ghb_out_column obp[kMaxPay];
  ghb_column ppay[kMaxPay];
  ghb_out_column opp[kMaxPay];
  int32_t* out_prow;
  int32_t* out_brow;
  int32_t prow_base;       // added to every probe row id written (a chunk of a longer probe)
  int64_t n, nchunks, cap;
  int32_t* slot_of_row;    // [n] slot (bucket * 4 + index) of the row's key, -1 = no match
  int64_t* chunk_count;    // [nchunks * warps per CTA] output rows of each warp's rows of a
                           // chunk (a warp covers 32 * IT consecutive rows), then their offset
  int64_t* d_out_rows;
  int32_t* status;
  int64_t build_rows;      // with slots: the table's layout (join_layout of stats)
  int64_t slots;
};

// Output rows a probe row produces, from its slot's count (0 = no match).
__device__ __forceinline__ int32_t out_rows_of(int join_type, int32_t count) {
  if (join_type == GHB_LEFT_SEMI_JOIN) return count > 0 ? 1 : 0;
  if (join_type == GHB_LEFT_OUTER_JOIN) return count > 0 ? count : 1;
  return count;
}

__device__ __forceinline__ void load_keys(const unsigned long long* kimg, int64_t bk,
                                          unsigned long long k[4]) {
  const ulonglong2* s = (const ulonglong2*)(kimg + bk * 4);
  ulonglong2 x = s[0], y = s[1];
  k[0] = x.x;
  k[1] = x.y;
  k[2] = y.x;
  k[3] = y.y;
}

// Index (0..3) of `u` among the bucket's keys, -1 when an empty slot ends
// the search, -2 when the bucket is full of other keys.
__device__ __forceinline__ int find_in(const unsigned long long k[4], unsigned long long u) {
#pragma unroll
  for (int q = 0; q < 4; q++) {
    if (k[q] == u) return q;
    if (k[q] == 0) return -1;
  }
  return -2;
}

// The count pass over a direct table: one load of the slot's row count per
// probe row, nothing else, so a thread keeps little and many CTAs fit on an
// SM.  It runs beside the hashed count pass; the build's key range chooses
// which of the two does the work and the other returns at once.
template <int TH, int IT, bool KEY_INT, bool NULLABLE>
__global__ void __launch_bounds__(TH) join_count_direct_kernel(ProbeParams p) {
  static_assert(TH * IT == kChunk, "a CTA iteration covers one chunk");
  const JoinLayout L = join_layout(p.stats, p.build_rows, p.slots);
  if (!L.direct) return;
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const bool unique = p.stats[1] <= 1;
  // every key of [min, max] present once (a dense surrogate key): a probe key
  // in the range matches, with no table load
  const bool full = unique && p.stats[2] == (unsigned long long)L.drange;
  // the lean write pass recomputes a direct table's slot from the key, so
  // this pass writes no slots for it
  const bool keep_slots = !(p.lean && p.out_brow == nullptr && unique);
  const int woff = warp * (32 * IT) + lane;
  auto load_chunk_keys = [&](int64_t c, long long* raw) {
    const int64_t cbase = c * kChunk;
    const int left = (int)min((int64_t)kChunk, p.n - cbase);
#pragma unroll
    for (int k = 0; k < IT; k++) {
      const int off = woff + k * 32;
      raw[k] = 0;
      if (c < p.nchunks && off < left)
        raw[k] = KEY_INT ? (long long)__ldcs((const int*)p.pkey.data + cbase + off)
                         : __ldcs((const long long*)p.pkey.data + cbase + off);
    }
  };
  long long next_raw[IT];
  load_chunk_keys(blockIdx.x, next_raw);
  for (int64_t c = blockIdx.x; c < p.nchunks; c += gridDim.x) {
    const int64_t cbase = c * kChunk;
    const int left = (int)min((int64_t)kChunk, p.n - cbase);
    long long raw[IT];
#pragma unroll
    for (int k = 0; k < IT; k++) raw[k] = next_raw[k];
    load_chunk_keys(c + gridDim.x, next_raw);
    unsigned long long d[IT];
    int32_t cnt[IT];
#pragma unroll
    for (int k = 0; k < IT; k++) {
      const int off = woff + k * 32;
      const bool valid = off < left && !(NULLABLE && raw_is_null(p.pkey, raw[k], cbase + off));
      d[k] = (unsigned long long)raw[k] - (unsigned long long)L.dmin;
      const bool inr = valid && d[k] < (unsigned long long)L.drange;
      cnt[k] = inr ? (full ? 1 : p.meta[d[k]].y) : 0;
    }
    uint64_t m_sum = 0;
#pragma unroll
    for (int k = 0; k < IT; k++) {
      const int off = woff + k * 32;
      if (off < left) {
        if (keep_slots) p.slot_of_row[cbase + off] = cnt[k] > 0 ? (int32_t)d[k] : -1;
        m_sum += (uint64_t)out_rows_of(p.join_type, unique ? (cnt[k] > 0 ? 1 : 0) : cnt[k]);
      }
    }
    for (int o = 16; o > 0; o >>= 1) m_sum += __shfl_down_sync(0xffffffffu, m_sum, o);
    if (lane == 0) p.chunk_count[c * (TH / 32) + warp] = (int64_t)m_sum;
  }
}

// TH threads x IT rows per thread = one chunk (kChunk rows) per iteration.
// Four 256-thread CTAs per SM (64 registers): more key and table loads in flight.
template <int TH, int IT, bool KEY_INT, bool NULLABLE>
__global__ void __launch_bounds__(TH, TH == 512 ? 2 : TH == 256 ? 4 : 1) join_count_kernel(ProbeParams p) {
  constexpr int kJThreads = TH, kJItems = IT;
  static_assert(TH * IT == kChunk, "a CTA iteration covers one chunk");
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const bool unique = p.stats[1] <= 1;   // every key once: a match is one output row
  if (join_layout(p.stats, p.build_rows, p.slots).direct) return;   // join_count_direct_kernel's table
  const int woff = warp * (32 * kJItems) + lane;
  // The keys of the CTA's next chunk are loaded while this chunk probes the
  // table, so the DRAM latency of the key stream overlaps the table loads.
  auto load_chunk_keys = [&](int64_t c, long long* raw) {
    const int64_t cbase = c * kChunk;
    const int left = (int)min((int64_t)kChunk, p.n - cbase);
#pragma unroll
    for (int k = 0; k < kJItems; k++) {
      const int off = woff + k * 32;
      raw[k] = 0;
      if (c < p.nchunks && off < left)
        raw[k] = KEY_INT ? (long long)__ldcs((const int*)p.pkey.data + cbase + off)
                         : __ldcs((const long long*)p.pkey.data + cbase + off);
    }
  };
  long long next_raw[kJItems];
  load_chunk_keys(blockIdx.x, next_raw);
  for (int64_t c = blockIdx.x; c < p.nchunks; c += gridDim.x) {
    const int64_t cbase = c * kChunk;
    // rows of this chunk left (a full chunk unless it is the last one)
    const int left = (int)min((int64_t)kChunk, p.n - cbase);
    long long cur_raw[kJItems];
#pragma unroll
    for (int k = 0; k < kJItems; k++) cur_raw[k] = next_raw[k];
    load_chunk_keys(c + gridDim.x, next_raw);
    unsigned long long u[kJItems];
    bool valid[kJItems];
#pragma unroll
    for (int k = 0; k < kJItems; k++) {
      const int off = woff + k * 32;
      const long long raw = cur_raw[k];
      valid[k] = off < left && !(NULLABLE && raw_is_null(p.pkey, raw, cbase + off));
      u[k] = flip_i64(raw);
    }
    uint64_t m_sum = 0;
    int64_t bk[kJItems];
    unsigned long long keys[kJItems][4];
#pragma unroll
    for (int k = 0; k < kJItems; k++) {
      bk[k] = bucket_of(u[k], p.hshift);
      if (valid[k] && u[k] != 0) load_keys(p.kimg, bk[k], keys[k]);
    }
#pragma unroll
    for (int k = 0; k < kJItems; k++) {
      const int off = woff + k * 32;
      const int64_t row = cbase + off;
      int32_t slot = -1, count = 0;
      if (valid[k]) {
        if (u[k] == 0) {
          int32_t cnt = p.meta[p.side * 4].y;
          if (cnt > 0) { slot = (int32_t)(p.side * 4); count = cnt; }
        } else {
          int q = find_in(keys[k], u[k]);
          while (q == -2) {   // bucket full of other keys: continue in the next one
            bk[k] = (bk[k] + 1) & p.bmask;
            load_keys(p.kimg, bk[k], keys[k]);
            q = find_in(keys[k], u[k]);
          }
          if (q >= 0) {
            slot = (int32_t)(bk[k] * 4 + q);
            count = unique ? 1 : p.meta[slot].y;
          }
        }
      }
      if (off < left) {
        p.slot_of_row[row] = slot;
        m_sum += (uint64_t)out_rows_of(p.join_type, count);
      }
    }
    for (int o = 16; o > 0; o >>= 1) m_sum += __shfl_down_sync(0xffffffffu, m_sum, o);
    if (lane == 0) p.chunk_count[c * (kJThreads / 32) + warp] = (int64_t)m_sum;
  }
}

// Chunk counts -> exclusive offsets in place, many CTAs: each claims a tile
// of 1024 counts in order, scans it, and gets the tile's offset from the tiles
// before it by decoupled look-back; the last tile writes the total.
struct ScanParams {
  int64_t* counts;
  int64_t n;
  int64_t ntiles;
  int64_t* d_total;
  uint64_t* lb;
  uint32_t epoch;
  unsigned long long* counters;
  int32_t* status;
  int32_t spin_limit;   // look-back polls before GHB_ERR_TIMEOUT
};

__global__ void __launch_bounds__(1024) join_scan_lb_kernel(ScanParams p) {
  __shared__ int64_t s_tile;
  __shared__ int64_t s_warp[32];
  __shared__ uint64_t s_excl;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  while (true) {
    claim_tile(&p.counters[0], &s_tile);
    const int64_t tile = s_tile;
    if (tile >= p.ntiles) break;
    const int64_t i = tile * 1024 + threadIdx.x;
    const int64_t v = i < p.n ? p.counts[i] : 0;
    int64_t incl = v;
    for (int o = 1; o < 32; o <<= 1) {
      const int64_t t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    if (warp == 0) {
      const int64_t w = s_warp[lane];
      int64_t wi = w;
      for (int o = 1; o < 32; o <<= 1) {
        const int64_t t = __shfl_up_sync(0xffffffffu, wi, o);
        if (lane >= o) wi += t;
      }
      s_warp[lane] = wi - w;
      const int64_t total = __shfl_sync(0xffffffffu, wi, 31);
      const uint64_t ex = lookback_exclusive(p.lb, p.epoch, tile, (uint64_t)total, p.status,
                                                    p.spin_limit);
      if (lane == 0) {
        s_excl = ex;
        if (tile == p.ntiles - 1) *p.d_total = (int64_t)(ex + total);
      }
    }
    __syncthreads();
    if (i < p.n) p.counts[i] = (int64_t)s_excl + s_warp[warp] + incl - v;
    __syncthreads();
  }
  claim_finish(p.counters);
}

// One CTA: chunk counts -> exclusive offsets in place; the total to d_out_rows.
__global__ void __launch_bounds__(1024) join_scan_kernel(int64_t* counts, int64_t n, int64_t* d_total) {
  __shared__ int64_t s_part[1024];
  const int t = threadIdx.x;
  const int64_t per = (n + 1023) / 1024;
  const int64_t lo = t * per, hi = min(n, lo + per);
  int64_t sum = 0;
  for (int64_t i = lo; i < hi; i++) sum += counts[i];
  s_part[t] = sum;
  __syncthreads();
  for (int o = 1; o < 1024; o <<= 1) {
    int64_t v = t >= o ? s_part[t - o] : 0;
    __syncthreads();
    s_part[t] += v;
    __syncthreads();
  }
  int64_t run = s_part[t] - sum;
  for (int64_t i = lo; i < hi; i++) {
    int64_t c = counts[i];
    counts[i] = run;
    run += c;
  }
  if (t == 1023) *d_total = s_part[1023];
}

__device__ __forceinline__ void put_word(const ghb_out_column& o, int64_t pos, int type, int64_t raw,
                                         bool null) {
  if (null) {
    if (type == GHB_INT) __stcs((int*)o.data + pos, INT32_MAX);
    else if (type == GHB_LONG) __stcs((long long*)o.data + pos, (long long)INT64_MAX);
    else __stcs((long long*)o.data + pos, 0x7ff8000000000000ll);
  } else if (type == GHB_INT) {
    __stcs((int*)o.data + pos, (int)raw);
  } else {
    __stcs((long long*)o.data + pos, (long long)raw);
  }
  if (o.is_null) o.is_null[pos] = null ? 1 : 0;
}

// The payload descriptors and output pointers of a probe, copied to shared
// memory once per CTA for the general emit path below.
struct EmitDesc {
  ghb_column bpay[kMaxPay];
  ghb_out_column obp[kMaxPay];
  ghb_column ppay[kMaxPay];
  ghb_out_column opp[kMaxPay];
  int32_t* out_prow;
  int32_t* out_brow;
  int32_t prow_base;
  int32_t nbp, npp, n_inline;
};

__device__ __forceinline__ void load_emit_desc(const ProbeParams& p, EmitDesc* d) {
  if (threadIdx.x < kMaxPay) {
    const int j = threadIdx.x;
    d->bpay[j] = p.bpay[j];
    d->obp[j] = p.obp[j];
    d->ppay[j] = p.ppay[j];
    d->opp[j] = p.opp[j];
  }
  if (threadIdx.x == 0) {
    d->out_prow = p.out_prow;
    d->out_brow = p.out_brow;
    d->prow_base = p.prow_base;
    d->nbp = p.nbp;
    d->npp = p.npp;
    d->n_inline = p.n_inline;
  }
  __syncthreads();
}

// One output row: probe row `prow`, build row `brow` (-1 for an outer miss /
// semi), with the first-row payload words `w0`, `w1` when `inl` is set.  Out
// of line, reading its descriptors from shared memory: the write kernel's hot
// path is emit_lean, and inlined copies of this general loop would crowd its
// registers.
__device__ __noinline__ void emit_row(const EmitDesc* d, int64_t pos, int64_t prow, int32_t brow, bool inl,
                                      unsigned long long w0, unsigned long long w1) {
  if (d->out_prow) __stcs(d->out_prow + pos, (int)prow + d->prow_base);
  if (d->out_brow) __stcs(d->out_brow + pos, brow);
  for (int j = 0; j < d->nbp; j++) {
    const ghb_column& c = d->bpay[j];
    if (brow < 0) {
      put_word(d->obp[j], pos, c.type, 0, true);
      continue;
    }
    int64_t raw = (inl && j < d->n_inline) ? (int64_t)(j == 0 ? w0 : w1) : ld_raw(c, brow);
    bool null = c.null_mode != GHB_NULLS_NONE && raw_is_null(c, raw, brow);
    put_word(d->obp[j], pos, c.type, raw, null);
  }
  for (int j = 0; j < d->npp; j++) {
    const ghb_column& c = d->ppay[j];
    int64_t raw = ld_raw(c, prow);
    put_word(d->opp[j], pos, c.type, raw, c.null_mode != GHB_NULLS_NONE && raw_is_null(c, raw, prow));
  }
}

// The lean case (INNER, no probe payloads, at most two build payloads, all
// inline and non-NULL): the output descriptors are read once into registers
// and a row is a few stores.  Constant indices keep the descriptors in the
// parameter space; the general emit_row loops over them with a run-time
// index.
struct LeanOut {
  int32_t* prow;
  int32_t* brow;
  int32_t prow_base;
  void* data[kInline];
  uint8_t* nul[kInline];
  bool is_int[kInline];
  int nbp;
};

__device__ __forceinline__ LeanOut lean_out(const ProbeParams& p) {
  LeanOut o;
  o.prow = p.out_prow;
  o.brow = p.out_brow;
  o.prow_base = p.prow_base;
  o.nbp = p.nbp;
#pragma unroll
  for (int j = 0; j < kInline; j++) {
    o.data[j] = p.obp[j].data;
    o.nul[j] = p.obp[j].is_null;
    o.is_int[j] = p.bpay[j].type == GHB_INT;
  }
  return o;
}

__device__ __forceinline__ void emit_lean(const LeanOut& o, int64_t pos, int64_t prow, int32_t brow,
                                          unsigned long long w0, unsigned long long w1) {
  if (o.prow) __stcs(o.prow + pos, (int)prow + o.prow_base);
  if (o.brow) __stcs(o.brow + pos, brow);
#pragma unroll
  for (int j = 0; j < kInline; j++) {
    if (j >= o.nbp) break;
    const unsigned long long w = j == 0 ? w0 : w1;
    if (o.is_int[j]) __stcs((int*)o.data[j] + pos, (int)w);
    else __stcs((unsigned long long*)o.data[j] + pos, w);
    if (o.nul[j]) o.nul[j][pos] = 0;
  }
}

// The write pass of an INNER join on unique build keys whose output is the
// probe row and at most two inline, non-NULL build payloads (p.lean, no
// build row ids): a row's output is its slot's two payload words or nothing,
// so a thread keeps only slots and words and many CTAs fit on an SM.  It runs
// beside the general write pass; the build's statistics (unique keys) choose
// which of the two does the work and the other returns at once.
template <int TH, int IT>
__global__ void __launch_bounds__(TH) join_write_lean_kernel(ProbeParams p) {
  static_assert(TH * IT == kChunk, "a CTA iteration covers one chunk");
  if (!(p.lean && p.out_brow == nullptr && p.stats[1] <= 1)) return;
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  // a direct table: the slot is the key's offset from the minimum, read from
  // the key itself (the count pass wrote no slots); a full one (every key of
  // the range present) needs no check of the slot
  const JoinLayout L = join_layout(p.stats, p.build_rows, p.slots);
  const bool from_keys = L.direct;
  const bool full = from_keys && p.stats[2] == (unsigned long long)L.drange;
  const bool kint = p.pkey.type == GHB_INT;
  const bool knull = p.pkey.null_mode != GHB_NULLS_NONE;
  // a row's next input: its probe key (direct table) or its slot (hashed)
  auto fetch = [&](int64_t row) -> long long {
    if (row >= p.n) return 0;
    if (!from_keys) return (long long)__ldcs(p.slot_of_row + row);
    return kint ? (long long)__ldcs((const int*)p.pkey.data + row) : __ldcs((const long long*)p.pkey.data + row);
  };
  long long next_r[IT];
#pragma unroll
  for (int k = 0; k < IT; k++)
    next_r[k] = fetch((int64_t)blockIdx.x * kChunk + (int64_t)warp * (32 * IT) + k * 32 + lane);
  for (int64_t c = blockIdx.x; c < p.nchunks; c += gridDim.x) {
    const int64_t wbase = c * kChunk + (int64_t)warp * (32 * IT);
    int32_t s[IT];
#pragma unroll
    for (int k = 0; k < IT; k++) {
      const int64_t row = wbase + k * 32 + lane;
      const long long r = next_r[k];
      next_r[k] = fetch(wbase + (int64_t)gridDim.x * kChunk + k * 32 + lane);
      if (!from_keys) {
        s[k] = row < p.n ? (int32_t)r : -1;
      } else {
        const unsigned long long d = (unsigned long long)r - (unsigned long long)L.dmin;
        const bool hit = row < p.n && d < (unsigned long long)L.drange && !(knull && raw_is_null(p.pkey, r, row));
        s[k] = hit ? (int32_t)d : -1;
      }
    }
    if (from_keys && !full) {
#pragma unroll
      for (int k = 0; k < IT; k++)
        if (s[k] >= 0 && p.meta[s[k]].y == 0) s[k] = -1;   // a hole of the key range
    }
    ulonglong2 w[IT];
#pragma unroll
    for (int k = 0; k < IT; k++) w[k] = s[k] >= 0 && p.nbp > 0 ? p.payw[s[k]] : make_ulonglong2(0, 0);
    uint32_t excl[IT];
    uint32_t running = 0;
#pragma unroll
    for (int k = 0; k < IT; k++) {
      const unsigned bal = __ballot_sync(0xffffffffu, s[k] >= 0);
      excl[k] = running + __popc(bal & ((1u << lane) - 1u));
      running += __popc(bal);
    }
    const int64_t wpos = p.chunk_count[c * (TH / 32) + warp];   // this warp's offset
#pragma unroll
    for (int k = 0; k < IT; k++) {
      if (s[k] < 0) continue;
      const int64_t pos = wpos + excl[k];
      if (pos >= p.cap) {
        raise_status(p.status, kDevCapacity);
        continue;
      }
      if (p.out_prow) __stcs(p.out_prow + pos, (int)(wbase + k * 32 + lane) + p.prow_base);
#pragma unroll
      for (int j = 0; j < kInline; j++) {
        if (j >= p.nbp) break;
        const unsigned long long x = j == 0 ? w[k].x : w[k].y;
        if (p.bpay[j].type == GHB_INT) __stcs((int*)p.obp[j].data + pos, (int)x);
        else __stcs((unsigned long long*)p.obp[j].data + pos, x);
        if (p.obp[j].is_null) p.obp[j].is_null[pos] = 0;
      }
    }
  }
}

template <int TH, int IT>
__global__ void __launch_bounds__(TH) join_write_kernel(ProbeParams p) {
  constexpr int kJThreads = TH, kJItems = IT;
  static_assert(TH * IT == kChunk, "a CTA iteration covers one chunk");
  if (p.lean && p.out_brow == nullptr && p.stats[1] <= 1) return;   // join_write_lean_kernel's case
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const bool unique = p.stats[1] <= 1;
  // the row's (first row, count) is needed for duplicates and build row ids
  const bool need_meta = !unique || p.out_brow != nullptr || !p.lean;
  const LeanOut lo = lean_out(p);
  __shared__ EmitDesc s_desc;
  load_emit_desc(p, &s_desc);
  // the next chunk's slots load while this chunk gathers and writes
  int32_t next_s[kJItems];
#pragma unroll
  for (int k = 0; k < kJItems; k++) {
    const int64_t row = (int64_t)blockIdx.x * kChunk + (int64_t)warp * (32 * kJItems) + k * 32 + lane;
    next_s[k] = row < p.n ? __ldcs(p.slot_of_row + row) : -1;
  }
  for (int64_t c = blockIdx.x; c < p.nchunks; c += gridDim.x) {
    const int64_t wbase = c * kChunk + (int64_t)warp * (32 * kJItems);
    int32_t s[kJItems];
#pragma unroll
    for (int k = 0; k < kJItems; k++) {
      s[k] = next_s[k];
      const int64_t nrow = wbase + (int64_t)gridDim.x * kChunk + k * 32 + lane;
      next_s[k] = nrow < p.n ? __ldcs(p.slot_of_row + nrow) : -1;
    }
    ulonglong2 w[kJItems];
    int32_t first[kJItems], cnt[kJItems];
#pragma unroll
    for (int k = 0; k < kJItems; k++) {
      first[k] = 0;
      cnt[k] = s[k] >= 0 ? 1 : 0;
      if (s[k] >= 0) {
        if (p.nbp > 0) w[k] = p.payw[s[k]];
        if (need_meta) {
          const int2 m = p.meta[s[k]];
          first[k] = m.x;
          cnt[k] = m.y;
        }
      }
    }
    int32_t mult[kJItems];
    uint32_t excl[kJItems];
    uint32_t running = 0;
#pragma unroll
    for (int k = 0; k < kJItems; k++) {
      int64_t row = wbase + k * 32 + lane;
      int32_t m = row < p.n ? out_rows_of(p.join_type, cnt[k]) : 0;
      mult[k] = m;
      uint32_t incl;
      if (__all_sync(0xffffffffu, m <= 1)) {
        unsigned bal = __ballot_sync(0xffffffffu, m == 1);
        incl = __popc(bal & ((2u << lane) - 1u));
      } else {
        incl = (uint32_t)m;
        for (int o = 1; o < 32; o <<= 1) {
          uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
          if (lane >= o) incl += t;
        }
      }
      excl[k] = running + incl - (uint32_t)m;
      running += __shfl_sync(0xffffffffu, incl, 31);
    }
    const int64_t wpos = p.chunk_count[c * (kJThreads / 32) + warp];   // this warp's offset
#pragma unroll
    for (int k = 0; k < kJItems; k++) {
      if (mult[k] == 0) continue;
      int64_t row = wbase + k * 32 + lane;
      int64_t pos = wpos + excl[k];
      if (pos + mult[k] > p.cap) {
        raise_status(p.status, kDevCapacity);
        continue;
      }
      if (s[k] < 0 || p.join_type == GHB_LEFT_SEMI_JOIN) {
        emit_row(&s_desc, pos, row, -1, false, 0, 0);
        continue;
      }
      if (p.lean) emit_lean(lo, pos, row, first[k] - 1, p.nbp > 0 ? w[k].x : 0, p.nbp > 0 ? w[k].y : 0);
      else emit_row(&s_desc, pos, row, first[k] - 1, true, p.nbp > 0 ? w[k].x : 0, p.nbp > 0 ? w[k].y : 0);
      if (mult[k] > 1) {
        int32_t b = p.chain_p1[s[k]] - 1;
        for (int j = 1; j < mult[k]; j++) {
          emit_row(&s_desc, pos + j, row, b, false, 0, 0);
          if (j + 1 < mult[k]) b = p.next_p1[b] - 1;
        }
      }
    }
  }
}

static int64_t next_pow2(int64_t v) {
  int64_t p = 1;
  while (p < v) p <<= 1;
  return p;
}

// Tables holding an L2 persistence window, per device (`delta` added under a
// lock; returns the new count).
static int l2_window_count(int device, int delta) {
  static std::mutex mu;
  static std::map<int, int> count;
  std::lock_guard<std::mutex> lock(mu);
  return count[device] += delta;
}

int32_t join_build_impl(ghb_ctx* ctx, const ghb_column* build_key, const ghb_column* build_payload,
                        int32_t nbp, const ghb_join_cfg* cfg, ghb_join_table** out,
                        cudaStream_t stream) {
  if (!out) return set_error(ctx, GHB_ERR_INVALID, "out is NULL");
  *out = nullptr;
  int32_t st = validate_columns(ctx, build_key, 1, nullptr);
  if (st) return st;
  if (build_key->type == GHB_DOUBLE)
    return set_error(ctx, GHB_ERR_UNSUPPORTED, "join keys must be LONG or INT");
  if (build_key->n >= INT32_MAX / 2)
    return set_error(ctx, GHB_ERR_UNSUPPORTED, "build side of 2^30 rows or more");
  if (nbp < 0 || nbp > kMaxPay || (nbp > 0 && !build_payload))
    return set_error(ctx, GHB_ERR_INVALID, "n_build_payload=%d outside [0,%d]", nbp, kMaxPay);
  for (int j = 0; j < nbp; j++) {
    if ((st = validate_columns(ctx, &build_payload[j], 1, nullptr))) return st;
    if (build_payload[j].n != build_key->n)
      return set_error(ctx, GHB_ERR_INVALID, "build payload %d has %lld rows, the key %lld", j,
                       (long long)build_payload[j].n, (long long)build_key->n);
  }
  float lf = (cfg && cfg->load_factor > 0.f && cfg->load_factor < 0.95f) ? cfg->load_factor : 0.5f;
  int64_t nb = next_pow2(std::max<int64_t>(16, (int64_t)((double)build_key->n / (4.0 * lf)) + 1));
  ghb_join_table* t = new ghb_join_table();
  t->slots = nb * 4;
  t->build_rows = build_key->n;
  t->key_type = build_key->type;
  t->nbp = nbp;
  for (int j = 0; j < nbp; j++) t->pay[j] = build_payload[j];
  // payloads copied into the slots: the first two non-BYTEMAP columns
  t->n_inline = 0;
  while (t->n_inline < std::min(nbp, kInline) && build_payload[t->n_inline].null_mode != GHB_NULLS_BYTEMAP)
    t->n_inline++;
  const size_t slots = (size_t)(nb + 1) * 4;   // hashed buckets + the side bucket
  auto a256 = [](size_t b) { return (b + 255) & ~(size_t)255; };
  const size_t key_bytes = a256(slots * 8), meta_bytes = a256(slots * 8), pay_bytes = a256(slots * 16);
  size_t bucket_bytes = key_bytes + meta_bytes + pay_bytes;
  size_t chain_bytes = a256(slots * 4);
  size_t next_bytes = a256((size_t)std::max<int64_t>(build_key->n, 1) * 4);
  size_t bytes = bucket_bytes + chain_bytes + next_bytes + 256;
  // stream-ordered allocation: no device-wide sync, and the pool keeps the
  // memory for the next build on this device
  t->stream = stream;
  if (cfg && cfg->block_threads > 0) t->probe_threads = cfg->block_threads;
  if (cudaMallocAsync(&t->alloc, bytes, stream) != cudaSuccess) {
    cudaGetLastError();
    delete t;
    return set_error(ctx, GHB_ERR_OOM, "cannot allocate a %zu-byte join table", bytes);
  }
  t->alloc_bytes = bytes;
  t->kimg = (unsigned long long*)t->alloc;
  t->meta = (int2*)((char*)t->alloc + key_bytes);
  t->payw = (ulonglong2*)((char*)t->alloc + key_bytes + meta_bytes);
  t->chain = (int32_t*)((char*)t->alloc + bucket_bytes);
  t->next = (int32_t*)((char*)t->alloc + bucket_bytes + chain_bytes);
  t->d_stats = (unsigned long long*)((char*)t->alloc + bucket_bytes + chain_bytes + next_bytes);
  // keys, counts and chain heads start at zero; the payload words are read
  // only in slots a build row filled, so they are not cleared
  if (cudaMemsetAsync(t->alloc, 0, key_bytes + meta_bytes, stream) != cudaSuccess ||
      cudaMemsetAsync(t->chain, 0, chain_bytes, stream) != cudaSuccess ||
      cudaMemsetAsync(t->d_stats, 0, 256, stream) != cudaSuccess) {
    cudaFreeAsync(t->alloc, stream);
    delete t;
    return set_error(ctx, GHB_ERR_CUDA, "memset of the join table failed");
  }
  BuildParams p;
  std::memset(&p, 0, sizeof(p));
  p.key = *build_key;
  p.n_inline = t->n_inline;
  for (int j = 0; j < t->n_inline; j++) p.pay[j] = build_payload[j];
  p.kimg = t->kimg;
  p.meta = t->meta;
  p.payw = t->payw;
  p.chain_p1 = t->chain;
  p.next_p1 = t->next;
  p.bmask = nb - 1;
  p.hshift = 64 - __builtin_ctzll((unsigned long long)nb);
  p.side = nb;
  p.stats = t->d_stats;
  p.status = ctx->d_status;
  p.slots = nb * 4;
  if (build_key->n > 0) {
    int grid = (int)std::min<int64_t>((build_key->n + 255) / 256, (int64_t)ctx->num_sms * 8);
    join_key_range_kernel<<<grid, 256, 0, stream>>>(*build_key, t->d_stats);
    ctx->launches++;
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
      attr.accessPolicyWindow.num_bytes = std::min(bucket_bytes, (size_t)max_persist);
      attr.accessPolicyWindow.hitRatio = 1.0f;
      attr.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
      attr.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
      cudaStreamSetAttribute(stream, cudaStreamAttributeAccessPolicyWindow, &attr);
      t->l2_window = true;
      t->device = ctx->device;
      l2_window_count(ctx->device, +1);
    }
  }
  *out = t;
  return GHB_OK;
}

// Scratch one probe of n rows needs (slot per row, count per chunk).
size_t join_probe_scratch_bytes(int64_t n) {
  int64_t nchunks = (n + kChunk - 1) / kChunk;
  // a count per warp of each chunk: 16 warps at most (512-thread CTAs)
  return (((size_t)std::max<int64_t>(n, 1) * 4 + 255) & ~(size_t)255) +
         (((size_t)std::max<int64_t>(nchunks, 1) * 16 * 8 + 255) & ~(size_t)255) + 512;
}

int32_t scan_counts(ghb_ctx* ctx, int64_t* counts, int64_t n, int64_t* d_total, cudaStream_t stream) {
  if (n <= 4096) {
    join_scan_kernel<<<1, 1024, 0, stream>>>(counts, n, d_total);
  } else {
    ScanParams sp;
    sp.counts = counts;
    sp.n = n;
    sp.ntiles = (n + 1023) / 1024;
    sp.d_total = d_total;
    const int32_t st = lookback_prepare(ctx, sp.ntiles, &sp.epoch, stream);
    if (st) return st;
    sp.lb = ctx->lb_status;
    sp.counters = ctx->d_counters;
    sp.status = ctx->d_status;
    sp.spin_limit = ctx->spin_limit;
    const int sgrid = (int)std::min<int64_t>(sp.ntiles, (int64_t)ctx->num_sms);
    join_scan_lb_kernel<<<sgrid, 1024, 0, stream>>>(sp);
  }
  GHB_LAUNCH_CHECK(ctx);
  return GHB_OK;
}

int32_t join_probe_impl(ghb_ctx* ctx, const ghb_join_table* t, const ghb_column* probe_key,
                        int32_t join_type, ghb_out_column* out_build, const ghb_column* probe_payload,
                        int32_t npp, ghb_out_column* out_probe, int32_t* out_probe_rowid,
                        int32_t* out_build_rowid, int64_t out_capacity, int64_t* d_out_rows,
                        cudaStream_t stream, int32_t prow_base) {
  if (!t) return set_error(ctx, GHB_ERR_INVALID, "table is NULL");
  int32_t st = validate_columns(ctx, probe_key, 1, nullptr);
  if (st) return st;
  if (probe_key->type == GHB_DOUBLE)
    return set_error(ctx, GHB_ERR_UNSUPPORTED, "join keys must be LONG or INT");
  if (probe_key->n >= INT32_MAX)
    return set_error(ctx, GHB_ERR_UNSUPPORTED, "probe side above 2^31-1 rows per call");
  if (join_type != GHB_INNER_JOIN && join_type != GHB_LEFT_SEMI_JOIN && join_type != GHB_LEFT_OUTER_JOIN)
    return set_error(ctx, GHB_ERR_UNSUPPORTED, "join type %d", join_type);
  if (npp < 0 || npp > kMaxPay)
    return set_error(ctx, GHB_ERR_INVALID, "n_probe_payload=%d outside [0,%d]", npp, kMaxPay);
  if (!d_out_rows) return set_error(ctx, GHB_ERR_INVALID, "d_out_rows is NULL");
  if (t->nbp > 0 && !out_build) return set_error(ctx, GHB_ERR_INVALID, "out_build is NULL");
  ProbeParams p;
  std::memset(&p, 0, sizeof(p));
  for (int j = 0; j < t->nbp; j++) {
    if (out_build[j].type != t->pay[j].type || !out_build[j].data)
      return set_error(ctx, GHB_ERR_INVALID, "build payload output %d: bad type or data", j);
    p.bpay[j] = t->pay[j];
    p.obp[j] = out_build[j];
  }
  for (int j = 0; j < npp; j++) {
    if ((st = validate_columns(ctx, &probe_payload[j], 1, nullptr))) return st;
    if (probe_payload[j].n != probe_key->n)
      return set_error(ctx, GHB_ERR_INVALID, "probe payload %d row count differs from the key", j);
    if (out_probe[j].type != probe_payload[j].type || !out_probe[j].data)
      return set_error(ctx, GHB_ERR_INVALID, "probe payload output %d: bad type or data", j);
    p.ppay[j] = probe_payload[j];
    p.opp[j] = out_probe[j];
  }
  p.kimg = t->kimg;
  p.meta = t->meta;
  p.payw = t->payw;
  p.chain_p1 = t->chain;
  p.next_p1 = t->next;
  p.stats = t->d_stats;
  p.bmask = t->slots / 4 - 1;
  p.hshift = 64 - __builtin_ctzll((unsigned long long)(t->slots / 4));
  p.side = t->slots / 4;
  p.build_rows = t->build_rows;
  p.slots = t->slots;
  p.pkey = *probe_key;
  p.join_type = join_type;
  p.nbp = t->nbp;
  p.npp = npp;
  p.n_inline = t->n_inline;
  p.lean = join_type == GHB_INNER_JOIN && npp == 0 && t->nbp == t->n_inline;
  for (int j = 0; j < t->n_inline && p.lean; j++) p.lean = t->pay[j].null_mode == GHB_NULLS_NONE;
  p.out_prow = out_probe_rowid;
  p.out_brow = out_build_rowid;
  p.prow_base = prow_base;
  p.n = probe_key->n;
  p.nchunks = (p.n + kChunk - 1) / kChunk;
  p.cap = out_capacity;
  p.d_out_rows = d_out_rows;
  p.status = ctx->d_status;
  if (p.nchunks == 0) {
    GHB_CUDA_TRY(ctx, cudaMemsetAsync(d_out_rows, 0, sizeof(int64_t), stream));
    return GHB_OK;
  }
  // CTA shape (threads x rows per thread, one 1024-row chunk either way),
  // chosen by the build's ghb_join_cfg.block_threads
  const int threads = t->probe_threads == 128 || t->probe_threads == 512 ? t->probe_threads : 256;
  const int64_t nunits = p.nchunks * (threads / 32);   // a count per warp of each chunk
  if ((st = scratch_alloc(ctx, (size_t)p.n * 4, (void**)&p.slot_of_row, stream))) return st;
  if ((st = scratch_alloc(ctx, (size_t)nunits * 8, (void**)&p.chunk_count, stream))) return st;
  const bool kint = probe_key->type == GHB_INT, knull = probe_key->null_mode != GHB_NULLS_NONE;
  void (*count_kernel)(ProbeParams) = nullptr;
  void (*write_kernel)(ProbeParams) = nullptr;
  void (*write_lean)(ProbeParams) = nullptr;
  void (*count_direct)(ProbeParams) = nullptr;
#define GHB_COUNT(TH, IT)                                                                   \
  count_kernel = kint ? (knull ? join_count_kernel<TH, IT, true, true> : join_count_kernel<TH, IT, true, false>) \
                      : (knull ? join_count_kernel<TH, IT, false, true> : join_count_kernel<TH, IT, false, false>); \
  count_direct = kint ? (knull ? join_count_direct_kernel<TH, IT, true, true> : join_count_direct_kernel<TH, IT, true, false>) \
                      : (knull ? join_count_direct_kernel<TH, IT, false, true> : join_count_direct_kernel<TH, IT, false, false>); \
  write_kernel = join_write_kernel<TH, IT>;                                                  \
  write_lean = join_write_lean_kernel<TH, IT>
  if (threads == 128) { GHB_COUNT(128, 8); }
  else if (threads == 512) { GHB_COUNT(512, 2); }
  else { GHB_COUNT(256, 4); }
#undef GHB_COUNT
  int per_sm = 0;
  GHB_CUDA_TRY(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, count_kernel, threads, 0));
  int grid = (int)std::min<int64_t>(p.nchunks, (int64_t)ctx->num_sms * std::max(1, per_sm));
  count_kernel<<<grid, threads, 0, stream>>>(p);
  GHB_LAUNCH_CHECK(ctx);
  // the count pass of a direct table (the build decided on the device which one works)
  GHB_CUDA_TRY(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, count_direct, threads, 0));
  grid = (int)std::min<int64_t>(p.nchunks, (int64_t)ctx->num_sms * std::max(1, per_sm));
  count_direct<<<grid, threads, 0, stream>>>(p);
  GHB_LAUNCH_CHECK(ctx);
  if ((st = scan_counts(ctx, p.chunk_count, nunits, d_out_rows, stream))) return st;
  GHB_CUDA_TRY(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, write_kernel, threads, 0));
  grid = (int)std::min<int64_t>(p.nchunks, (int64_t)ctx->num_sms * std::max(1, per_sm));
  write_kernel<<<grid, threads, 0, stream>>>(p);
  GHB_LAUNCH_CHECK(ctx);
  if (p.lean && !p.out_brow) {   // the lean write pass, when the build's keys turn out unique
    GHB_CUDA_TRY(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, write_lean, threads, 0));
    grid = (int)std::min<int64_t>(p.nchunks, (int64_t)ctx->num_sms * std::max(1, per_sm));
    write_lean<<<grid, threads, 0, stream>>>(p);
  }
  GHB_LAUNCH_CHECK(ctx);
  return GHB_OK;
}

}  // namespace ghb

using namespace ghb;

extern "C" {

int32_t ghb_join_build(ghb_ctx* ctx, const ghb_column* build_key, const ghb_column* build_payload,
                       int32_t n_build_payload, const ghb_join_cfg* cfg, ghb_join_table** out,
                       void* stream) {
  if (!ctx) return GHB_ERR_INVALID;
  CallScope cs(ctx, "join_build", (cudaStream_t)stream);
  cs.rows(build_key ? build_key->n : 0);
  cs.bytes(cols_bytes(build_key, build_key ? 1 : 0) + cols_bytes(build_payload, n_build_payload));
  return cs.done(join_build_impl(ctx, build_key, build_payload, n_build_payload, cfg, out,
                                 (cudaStream_t)stream));
}

int32_t ghb_join_table_free(ghb_ctx* ctx, ghb_join_table* table) {
  if (!ctx || !table) return GHB_ERR_INVALID;
  if (table->l2_window) {
    cudaStreamSynchronize(table->stream);
    // the build stream's window, if it still points at this table, goes
    cudaStreamAttrValue attr;
    std::memset(&attr, 0, sizeof(attr));
    if (cudaStreamGetAttribute(table->stream, cudaStreamAttributeAccessPolicyWindow, &attr) == cudaSuccess &&
        attr.accessPolicyWindow.base_ptr == table->alloc) {
      std::memset(&attr, 0, sizeof(attr));
      cudaStreamSetAttribute(table->stream, cudaStreamAttributeAccessPolicyWindow, &attr);
    }
    cudaGetLastError();
    // the persisting carve-out is shared by every resident table of the
    // device: it is released with the last table that holds a window
    if (l2_window_count(table->device, -1) == 0) {
      cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, 0);
      cudaCtxResetPersistingL2Cache();
    }
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
  unsigned long long st[5] = {0, 0, 0, 0, 0};
  GHB_CUDA_TRY(ctx, cudaMemcpy(st, table->d_stats, sizeof(st), cudaMemcpyDeviceToHost));
  if (rows) *rows = (int64_t)st[0];
  if (max_dup) *max_dup = (int64_t)st[1];
  // a direct table reports its key range as its slots
  const JoinLayout L = join_layout(st, table->build_rows, table->slots);
  if (slots) *slots = L.direct ? L.drange : table->slots;
  return GHB_OK;
}

int32_t ghb_join_probe(ghb_ctx* ctx, const ghb_join_table* table, const ghb_column* probe_key,
                       int32_t join_type, ghb_out_column* out_build, const ghb_column* probe_payload,
                       int32_t n_probe_payload, ghb_out_column* out_probe, int32_t* out_probe_rowid,
                       int32_t* out_build_rowid, int64_t out_capacity, int64_t* d_out_rows,
                       void* stream) {
  if (!ctx) return GHB_ERR_INVALID;
  CallScope cs(ctx, "join_probe", (cudaStream_t)stream);
  int64_t n = probe_key ? probe_key->n : 0;
  cs.rows(n);
  cs.bytes(cols_bytes(probe_key, probe_key ? 1 : 0) + cols_bytes(probe_payload, n_probe_payload));
  scratch_reset(ctx);
  int32_t st = scratch_reserve(ctx, join_probe_scratch_bytes(n), (cudaStream_t)stream);
  if (st) return cs.done(st);
  return cs.done(join_probe_impl(ctx, table, probe_key, join_type, out_build, probe_payload, n_probe_payload,
                                 out_probe, out_probe_rowid, out_build_rowid, out_capacity, d_out_rows,
                                 (cudaStream_t)stream, 0));
}

}  // extern "C"
