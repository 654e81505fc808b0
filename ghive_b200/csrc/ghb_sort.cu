// ghb_sort.cu — stable ORDER BY sort (S1): LSD radix sort on packed keys.
//
// Replaces the Sink sort of the reference (gpu_impl/src/Operator/
// SinkOperator.cu:153-286: H2D of the key columns, thrust::sort of row
// indices with an indirect multi-column comparator, D2H of the index, host
// gather of every column).  The order is Hive's BinarySortable order
// (BinarySortableSerDe.java:921-960 and the null markers at :195-220):
// integers by signed value, doubles by IEEE total order, per key ASC/DESC and
// NULLS FIRST/LAST; ties keep input order (LSD radix sort is stable).
//
// Pipeline (one call):
//   1. analyse   one read of the key columns: per key the min/max of its
//                order image and whether it holds NULLs;
//   2. plan      (host) each key becomes sub-fields [null flag][value - min]
//                of just the width its range needs, packed least-significant
//                key first into 64-bit segments;
//   3. histogram one read per segment: 8-bit digit histograms of all of the
//                segment's passes at once; passes whose digit is constant are
//                skipped;
//   4. passes    onesweep-style: each CTA claims a tile, ranks its keys by
//                digit within each warp (stable: a lane's peers of an item
//                from one shared atomicOr per lane), gets each digit's global
//                offset by decoupled look-back over earlier tiles, reorders
//                the tile in shared memory and writes one run per digit.
// A one-segment key (the common case, e.g. (int32 d, int64 k) with the ranges
// of the sort workload) is packed by the first pass straight from the user's
// columns and unpacked by the last pass straight into the output columns; the
// value carried with it is the single payload column, or the row index.  A
// key wider than 64 bits is sorted segment by segment (least significant
// first), each later segment packed from the row order the previous one left,
// and the output is gathered by the final row order.
#include <algorithm>
#include <vector>

#include "ghb_ctx.hpp"
#include "ghb_log.hpp"

namespace ghb {

constexpr int kSortThreads = 256;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortThreads * kSortItems;   // 4096
constexpr int kDigitBits = 8;
constexpr int kBins = 1 << kDigitBits;
constexpr int kMaxPasses = 8;                          // per 64-bit segment
constexpr int kMaxSortKeys = 8;
constexpr int kMaxSortPay = 8;
constexpr int kMaxSub = 2 * kMaxSortKeys;
constexpr int kMaxSeg = kMaxSub;

struct KeyField {
  ghb_column col;
  int32_t desc;
  int32_t nulls_first;
  int32_t has_null;      // the column holds NULLs: the key has a flag sub-field
  int32_t vbits;         // value bits
  uint64_t umin;         // min of the (possibly inverted) order image
};

struct SubField {
  int8_t key;
  int8_t is_flag;        // 1: the NULL flag, 0: the value bits
  int8_t bits;
  int8_t shift;          // within the segment word
};

struct Segment {
  int32_t n;
  int32_t bits;
  SubField f[kMaxSub];
};

struct KeySet {
  int32_t nkeys;
  KeyField k[kMaxSortKeys];
};

__device__ __forceinline__ uint64_t key_image(const ghb_column& c, int64_t raw) {
  return c.type == GHB_DOUBLE ? flip_f64_bits((uint64_t)raw) : flip_i64(raw);
}

// Contribution of one sub-field for row r (value already shifted into place).
__device__ __forceinline__ uint64_t sub_bits(const KeySet& K, const SubField& sf, int64_t r) {
  const KeyField& kf = K.k[sf.key];
  int64_t raw = ld_raw(kf.col, r);
  bool null = kf.has_null && raw_is_null(kf.col, raw, r);
  uint64_t v;
  if (sf.is_flag) {
    v = (null == (bool)kf.nulls_first) ? 0 : 1;   // NULLS FIRST: null 0 / value 1
  } else {
    uint64_t u = key_image(kf.col, raw);
    if (kf.desc) u = ~u;
    v = null ? 0 : u - kf.umin;
  }
  return v << sf.shift;
}

// ---------------------------------------------------------------- analyse
struct MinMaxParams {
  KeySet K;
  int64_t n;
  unsigned long long* out;  // per key: [0] min image, [1] max image, [2] any NULL
};

__global__ void __launch_bounds__(256) sort_minmax_kernel(MinMaxParams p) {
  constexpr int U = 4;
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int j = 0; j < p.K.nkeys; j++) {
    const KeyField& f = p.K.k[j];
    unsigned long long mn = ~0ull, mx = 0, anynull = 0;
    auto fold = [&](int64_t raw, int64_t r) {
      if (f.col.null_mode != GHB_NULLS_NONE && raw_is_null(f.col, raw, r)) {
        anynull = 1;
        return;
      }
      uint64_t img = key_image(f.col, raw);
      if (f.desc) img = ~img;
      mn = min(mn, (unsigned long long)img);
      mx = max(mx, (unsigned long long)img);
    };
    // 16-byte loads, U of them in flight per thread (a column read once,
    // evict-first); rows past the last whole vector, and columns with a NULL
    // map or an unaligned base, one value at a time
    int64_t done = 0;
    if (f.col.null_mode != GHB_NULLS_BYTEMAP && ((uintptr_t)f.col.data & 15) == 0) {
      if (f.col.type == GHB_INT) {
        const int4* v = (const int4*)f.col.data;
        const int64_t nv = p.n / 4;
        for (int64_t b = tid; b < nv; b += U * stride) {
          int4 x[U];
#pragma unroll
          for (int u = 0; u < U; u++) x[u] = b + u * stride < nv ? __ldcs(v + b + u * stride) : make_int4(0, 0, 0, 0);
#pragma unroll
          for (int u = 0; u < U; u++) {
            if (b + u * stride >= nv) continue;
            fold(x[u].x, 0);
            fold(x[u].y, 0);
            fold(x[u].z, 0);
            fold(x[u].w, 0);
          }
        }
        done = nv * 4;
      } else {
        const longlong2* v = (const longlong2*)f.col.data;
        const int64_t nv = p.n / 2;
        for (int64_t b = tid; b < nv; b += U * stride) {
          longlong2 x[U];
#pragma unroll
          for (int u = 0; u < U; u++) x[u] = b + u * stride < nv ? __ldcs(v + b + u * stride) : make_longlong2(0, 0);
#pragma unroll
          for (int u = 0; u < U; u++) {
            if (b + u * stride >= nv) continue;
            fold(x[u].x, 0);
            fold(x[u].y, 0);
          }
        }
        done = nv * 2;
      }
    }
    for (int64_t r = done + tid; r < p.n; r += stride) fold(ld_raw(f.col, r), r);
    for (int o = 16; o > 0; o >>= 1) {
      mn = min(mn, __shfl_down_sync(0xffffffffu, mn, o));
      mx = max(mx, __shfl_down_sync(0xffffffffu, mx, o));
      anynull |= __shfl_down_sync(0xffffffffu, anynull, o);
    }
    // one set of atomics per CTA: every CTA's warps hitting the same three
    // words would serialise at L2
    __shared__ unsigned long long s_red[3][8];
    const int warp = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
      s_red[0][warp] = mn;
      s_red[1][warp] = mx;
      s_red[2][warp] = anynull;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      for (int w = 1; w < (int)(blockDim.x >> 5); w++) {
        mn = min(mn, s_red[0][w]);
        mx = max(mx, s_red[1][w]);
        anynull |= s_red[2][w];
      }
      atomicMin(&p.out[3 * j], mn);
      atomicMax(&p.out[3 * j + 1], mx);
      if (anynull) atomicOr(&p.out[3 * j + 2], 1ull);
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------- histogram
// One sub-field of a packed key with everything its bits need, so a kernel
// packing keys reads it with constant indices.
struct SubPlan {
  ghb_column col;
  uint64_t umin;
  int8_t shift;
  int8_t is_flag;
  int8_t desc;
  int8_t nulls_first;
  int8_t has_null;
};

__device__ __forceinline__ uint64_t sub_bits_plan(const SubPlan& sp, int64_t raw, int64_t r) {
  const bool null = sp.has_null && raw_is_null(sp.col, raw, r);
  uint64_t v;
  if (sp.is_flag) {
    v = (null == (bool)sp.nulls_first) ? 0 : 1;   // NULLS FIRST: null 0 / value 1
  } else {
    uint64_t u = key_image(sp.col, raw);
    if (sp.desc) u = ~u;
    v = null ? 0 : u - sp.umin;
  }
  return v << sp.shift;
}

struct HistParams {
  KeySet K;
  Segment seg;
  SubPlan sub[kMaxSub];     // the segment's sub-fields, self-contained
  int64_t n;
  int32_t npasses;
  uint32_t* hist;  // [npasses][kBins]
  // a one-segment key: the packed keys and carried values are written here
  // too, so every radix pass reads packed keys
  uint64_t* keys_out;        // nullptr: not written
  void* vals_out;
  int32_t vals_wide;         // values are 64-bit (else 32-bit)
  int32_t carry_rowid;       // value = row index (else the single payload's raw bits)
  ghb_column pay_src;
  int32_t vec;               // every column read has 16-byte aligned data and no NULL map
};

// Rows r..r+3 (r a multiple of 4) of a column with 16-byte aligned data, as
// raw 64-bit values, by 16-byte loads read once.
__device__ __forceinline__ void load4(const ghb_column& c, int64_t r, int64_t raw[4]) {
  if (c.type == GHB_INT) {
    const int4 x = __ldcs((const int4*)c.data + r / 4);
    raw[0] = x.x;
    raw[1] = x.y;
    raw[2] = x.z;
    raw[3] = x.w;
  } else {
    const longlong2* q = (const longlong2*)c.data + r / 2;
    const longlong2 a = __ldcs(q), b = __ldcs(q + 1);
    raw[0] = a.x;
    raw[1] = a.y;
    raw[2] = b.x;
    raw[3] = b.y;
  }
}

__global__ void __launch_bounds__(256) sort_hist_kernel(HistParams p) {
  constexpr int U = 4;
  __shared__ uint32_t sh[kMaxPasses][kBins];
  for (int i = threadIdx.x; i < kMaxPasses * kBins; i += blockDim.x) (&sh[0][0])[i] = 0;
  __syncthreads();
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  // four consecutive rows per thread by 16-byte loads and stores, then the
  // rows past the last group of four (or all rows) one at a time
  int64_t done = 0;
  if (p.vec) {
    const int64_t ng = p.n / 4;
    for (int64_t g = tid; g < ng; g += stride) {
      const int64_t r = g * 4;
      uint64_t k[4] = {0, 0, 0, 0};
#pragma unroll
      for (int i = 0; i < kMaxSub; i++) {
        if (i >= p.seg.n) break;
        const SubPlan& sp = p.sub[i];
        int64_t raw[4];
        load4(sp.col, r, raw);
#pragma unroll
        for (int u = 0; u < 4; u++) k[u] |= sub_bits_plan(sp, raw[u], r + u);
      }
#pragma unroll
      for (int u = 0; u < 4; u++)
        for (int q = 0; q < p.npasses; q++) atomicAdd(&sh[q][(k[u] >> (q * kDigitBits)) & (kBins - 1)], 1u);
      if (p.keys_out) {
        ulonglong2* ko = (ulonglong2*)(p.keys_out + r);
        __stcs(ko, make_ulonglong2(k[0], k[1]));
        __stcs(ko + 1, make_ulonglong2(k[2], k[3]));
        int64_t v[4] = {r, r + 1, r + 2, r + 3};
        if (!p.carry_rowid) load4(p.pay_src, r, v);
        if (p.vals_wide) {
          ulonglong2* vo = (ulonglong2*)p.vals_out + r / 2;
          __stcs(vo, make_ulonglong2((unsigned long long)v[0], (unsigned long long)v[1]));
          __stcs(vo + 1, make_ulonglong2((unsigned long long)v[2], (unsigned long long)v[3]));
        } else {
          __stcs((uint4*)p.vals_out + r / 4,
                 make_uint4((unsigned)v[0], (unsigned)v[1], (unsigned)v[2], (unsigned)v[3]));
        }
      }
    }
    done = ng * 4;
  }
  for (int64_t base = done + tid; base < p.n; base += U * stride) {
    uint64_t k[U];
#pragma unroll
    for (int u = 0; u < U; u++) k[u] = 0;
#pragma unroll
    for (int i = 0; i < kMaxSub; i++) {
      if (i >= p.seg.n) break;
      const SubPlan& sp = p.sub[i];
      int64_t raw[U];
#pragma unroll
      for (int u = 0; u < U; u++) {
        const int64_t r = base + u * stride;
        raw[u] = r < p.n ? ld_raw(sp.col, r) : 0;
      }
#pragma unroll
      for (int u = 0; u < U; u++) {
        const int64_t r = base + u * stride;
        if (r < p.n) k[u] |= sub_bits_plan(sp, raw[u], r);
      }
    }
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int64_t r = base + u * stride;
      if (r >= p.n) continue;
      for (int q = 0; q < p.npasses; q++) atomicAdd(&sh[q][(k[u] >> (q * kDigitBits)) & (kBins - 1)], 1u);
      if (p.keys_out) {
        __stcs((unsigned long long*)p.keys_out + r, (unsigned long long)k[u]);
        const uint64_t v = p.carry_rowid ? (uint64_t)r : (uint64_t)ld_raw(p.pay_src, r);
        if (p.vals_wide) __stcs((unsigned long long*)p.vals_out + r, (unsigned long long)v);
        else __stcs((unsigned int*)p.vals_out + r, (unsigned int)v);
      }
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < p.npasses * kBins; i += blockDim.x) {
    uint32_t v = (&sh[0][0])[i];
    if (v) atomicAdd(&p.hist[i], v);
  }
}

// ---------------------------------------------------------------- passes
enum SrcMode { kSrcPacked = 0, kSrcCols = 1, kSrcPerm = 2 };
enum DstMode { kDstPacked = 0, kDstDecode = 1, kDstGather = 2 };

struct PassParams {
  KeySet K;
  Segment seg;
  int64_t n;
  int64_t ntiles;
  int32_t shift;
  int32_t carry_rowid;       // value = row index (else the single payload's raw bits)
  const uint64_t* keys_in;
  const void* vals_in;
  uint64_t* keys_out;
  void* vals_out;
  ghb_column pay_src;        // single carried payload (when !carry_rowid)
  ghb_out_column out_keys[kMaxSortKeys];
  int32_t npay;
  ghb_column pay[kMaxSortPay];
  ghb_out_column out_pay[kMaxSortPay];
  int32_t* out_rowid;
  // decoding a one-segment key, per key: value bits and shift, NULL flag
  // shift (-1 none)
  int8_t dec_vbits[kMaxSortKeys];
  int8_t dec_vshift[kMaxSortKeys];
  int8_t dec_fshift[kMaxSortKeys];
  uint32_t digit_base[kBins];  // exclusive global offset of each digit
  uint64_t* status;            // [ntiles][kBins] epoch-tagged look-back words
  uint32_t epoch;
  unsigned long long* counters;
  int32_t* dev_status;
  int32_t spin_limit;          // look-back polls before GHB_ERR_TIMEOUT
};

__device__ __forceinline__ void write_raw(const ghb_out_column& o, int64_t pos, int type, int64_t raw,
                                          bool null) {
  if (null) {
    if (o.is_null) o.is_null[pos] = 1;
    if (type == GHB_INT) ((int32_t*)o.data)[pos] = INT32_MAX;
    else if (type == GHB_LONG) ((int64_t*)o.data)[pos] = INT64_MAX;
    else ((long long*)o.data)[pos] = 0x7ff8000000000000ll;
    return;
  }
  if (type == GHB_INT) ((int32_t*)o.data)[pos] = (int32_t)raw;
  else ((long long*)o.data)[pos] = raw;
  if (o.is_null) o.is_null[pos] = 0;
}

// Copies keys and payloads of input row `row` to output position `pos`.
__device__ __forceinline__ void gather_write(const PassParams& p, int64_t row, int64_t pos) {
  for (int j = 0; j < p.K.nkeys; j++) {
    const ghb_column& c = p.K.k[j].col;
    int64_t raw = ld_raw(c, row);
    write_raw(p.out_keys[j], pos, c.type, raw, c.null_mode != GHB_NULLS_NONE && raw_is_null(c, raw, row));
  }
  if (p.out_rowid) p.out_rowid[pos] = (int32_t)row;
  for (int j = 0; j < p.npay; j++) {
    const ghb_column& c = p.pay[j];
    int64_t raw = ld_raw(c, row);
    write_raw(p.out_pay[j], pos, c.type, raw, c.null_mode != GHB_NULLS_NONE && raw_is_null(c, raw, row));
  }
}

// The carried value of a decoded row: its row index (row id output and
// payloads gathered by it), or the single payload itself.
__device__ __forceinline__ void decode_value(const PassParams& p, uint64_t v, int64_t pos) {
  if (p.carry_rowid) {
    int64_t row = (int64_t)v;
    if (p.out_rowid) p.out_rowid[pos] = (int32_t)row;
    for (int j = 0; j < p.npay; j++) {
      const ghb_column& c = p.pay[j];
      int64_t raw = ld_raw(c, row);
      write_raw(p.out_pay[j], pos, c.type, raw, c.null_mode != GHB_NULLS_NONE && raw_is_null(c, raw, row));
    }
  } else if (p.npay == 1) {
    const ghb_column& c = p.pay[0];
    bool null = c.null_mode == GHB_NULLS_SENTINEL && raw_is_null(c, (int64_t)v, 0);
    write_raw(p.out_pay[0], pos, c.type, (int64_t)v, null);
  }
}

// Three CTAs per SM: the registers are held to 80 (a few bytes spill), and
// three CTAs' shared memory fits an SM.
template <typename V, int SRC, int DST>
__global__ void __launch_bounds__(kSortThreads, 3) sort_pass_kernel(PassParams p) {
  __shared__ uint32_t s_whist[kSortThreads / 32][kBins];  // per-warp counts, then exclusive over warps
  __shared__ uint32_t s_bexcl[kBins];                      // block-local exclusive offset per digit
  __shared__ uint64_t s_gbase[kBins];                      // global destination of each digit's run
  __shared__ uint32_t s_wsum[kSortThreads / 32];
  __shared__ uint32_t s_match[kSortThreads / 32][kBins];   // lanes of each digit, per warp
  __shared__ int64_t s_tile;
  extern __shared__ uint64_t s_dyn[];                      // reordered tile: keys, then values
  uint64_t* s_keys = s_dyn;
  V* s_vals = (V*)(s_dyn + kSortTile);
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const unsigned lt = (1u << lane) - 1u;
  const V* vals_in = (const V*)p.vals_in;
  V* vals_out = (V*)p.vals_out;

  while (true) {
    if (threadIdx.x == 0) {
      int64_t t = (int64_t)atomicAdd(&p.counters[0], 1ull);
      // a look-back of this sort that gave up left this pass's input invalid
      // (rows at wrong places, some never written): claim no more tiles, so no
      // key or row index read from that input addresses anything
      if (*(volatile int32_t*)p.dev_status == kDevTimeout) t = p.ntiles;
      s_tile = t;
      // the tile about one round of claims ahead starts toward L2, so the
      // CTA that claims it finds its keys and values there
      const int64_t ahead = t + gridDim.x;
      if (SRC == kSrcPacked && (ahead + 1) * kSortTile <= p.n) {
        bulk_prefetch_l2((const unsigned long long*)p.keys_in + ahead * kSortTile, kSortTile * 8);
        bulk_prefetch_l2(vals_in + ahead * kSortTile, kSortTile * (uint32_t)sizeof(V));
      }
    }
    for (int i = threadIdx.x; i < (kSortThreads / 32) * kBins; i += kSortThreads) {
      (&s_whist[0][0])[i] = 0;
      (&s_match[0][0])[i] = 0;
    }
    __syncthreads();
    const int64_t tile = s_tile;
    if (tile >= p.ntiles) break;
    const int64_t wbase = tile * kSortTile + (int64_t)warp * (32 * kSortItems);

    uint64_t key[kSortItems];
    V val[kSortItems];
    if (SRC == kSrcPacked) {
#pragma unroll
      for (int k = 0; k < kSortItems; k++) {
        int64_t row = wbase + k * 32 + lane;
        key[k] = row < p.n ? __ldcs((const unsigned long long*)p.keys_in + row) : ~0ull;
      }
#pragma unroll
      for (int k = 0; k < kSortItems; k++) {
        int64_t row = wbase + k * 32 + lane;
        val[k] = row < p.n ? vals_in[row] : (V)0;
      }
    } else {
      int64_t src[kSortItems];
#pragma unroll
      for (int k = 0; k < kSortItems; k++) {
        int64_t row = wbase + k * 32 + lane;
        key[k] = 0;
        if (SRC == kSrcPerm) src[k] = row < p.n ? (int64_t)vals_in[row] : 0;
        else src[k] = row;
      }
      // one sub-field at a time over all items: the loads are independent
      for (int i = 0; i < p.seg.n; i++) {
        const SubField sf = p.seg.f[i];
#pragma unroll
        for (int k = 0; k < kSortItems; k++) {
          int64_t row = wbase + k * 32 + lane;
          if (row < p.n) key[k] |= sub_bits(p.K, sf, src[k]);
        }
      }
#pragma unroll
      for (int k = 0; k < kSortItems; k++) {
        int64_t row = wbase + k * 32 + lane;
        if (row >= p.n) key[k] = ~0ull;
        if (p.carry_rowid) val[k] = (V)src[k];
        else val[k] = row < p.n ? (V)ld_raw(p.pay_src, row) : (V)0;
      }
    }
    // stable rank of each key among the warp's keys with the same digit
    uint32_t rank[kSortItems];
#pragma unroll
    for (int k = 0; k < kSortItems; k++) {
      int64_t row = wbase + k * 32 + lane;
      bool live = row < p.n;
      uint32_t d = (uint32_t)(key[k] >> p.shift) & (kBins - 1);
      // the warp's lanes holding digit d: each lane sets its bit in the
      // digit's word (one shared atomic, no per-bit ballots), reads the word
      // back, and the lowest of them clears it for the next item
      unsigned peers = 0;
      if (live) atomicOr(&s_match[warp][d], 1u << lane);
      __syncwarp();
      if (live) peers = s_match[warp][d];
      __syncwarp();
      if (live && (peers & lt) == 0) s_match[warp][d] = 0;
      uint32_t before = live ? s_whist[warp][d] : 0;
      __syncwarp();
      if (live && (peers & lt) == 0) s_whist[warp][d] = before + __popc(peers);
      __syncwarp();
      rank[k] = before + __popc(peers & lt);
    }
    __syncthreads();
    // per digit (one thread each): exclusive over warps, block total
    const int d = threadIdx.x;  // kSortThreads == kBins
    uint32_t total = 0;
#pragma unroll
    for (int w = 0; w < kSortThreads / 32; w++) {
      uint32_t c = s_whist[w][d];
      s_whist[w][d] = total;
      total += c;
    }
    // publish this tile's count of digit d, then look back for its prefix
    {
      uint64_t* st = p.status + tile * kBins;
      uint64_t excl = 0;
      if (tile == 0) {
        lb_store(&st[d], lb_pack(p.epoch, kFlagPrefix, total));
      } else {
        lb_store(&st[d], lb_pack(p.epoch, kFlagAgg, total));
        int64_t t = tile - 1;
        int spins = 0;
        while (t >= 0) {
          uint64_t v = lb_load(&p.status[t * kBins + d]);
          bool ok = ((v >> kEpochShift) & kEpochMask) == (p.epoch & kEpochMask);
          if (ok && (v & kFlagPrefix)) { excl += v & kCountMask; break; }
          if (ok && (v & kFlagAgg)) { excl += v & kCountMask; t--; continue; }
          if (++spins >= p.spin_limit) { raise_status(p.dev_status, kDevTimeout); break; }
        }
        lb_store(&st[d], lb_pack(p.epoch, kFlagPrefix, excl + total));
      }
      s_gbase[d] = (uint64_t)p.digit_base[d] + excl;
    }
    // block-wide exclusive scan of the per-digit totals
    {
      uint32_t incl = total;
      for (int o = 1; o < 32; o <<= 1) {
        uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
      }
      if (lane == 31) s_wsum[warp] = incl;
      __syncthreads();
      if (warp == 0) {
        uint32_t v = lane < kSortThreads / 32 ? s_wsum[lane] : 0;
        uint32_t x = v;
        for (int o = 1; o < 32; o <<= 1) {
          uint32_t t = __shfl_up_sync(0xffffffffu, x, o);
          if (lane >= o) x += t;
        }
        if (lane < kSortThreads / 32) s_wsum[lane] = x - v;
      }
      __syncthreads();
      s_bexcl[d] = s_wsum[warp] + incl - total;
    }
    __syncthreads();
    // scatter into shared memory in digit order (stable)
#pragma unroll
    for (int k = 0; k < kSortItems; k++) {
      int64_t row = wbase + k * 32 + lane;
      if (row >= p.n) continue;
      uint32_t dk = (uint32_t)(key[k] >> p.shift) & (kBins - 1);
      uint32_t at = s_bexcl[dk] + s_whist[warp][dk] + rank[k];
      s_keys[at] = key[k];
      s_vals[at] = val[k];
    }
    __syncthreads();
    // write runs: element i of the reordered tile goes to gbase[d] + (i - bexcl[d])
    const int64_t tile_n = min((int64_t)kSortTile, p.n - tile * kSortTile);
    if (DST == kDstDecode) {
      // one key column at a time, its decoding parameters held in registers,
      // then the carried values
      for (int j = 0; j < p.K.nkeys; j++) {
        const KeyField& kf = p.K.k[j];
        const int vb = p.dec_vbits[j], vs = p.dec_vshift[j], fs = p.dec_fshift[j];
        const uint64_t vmask = vb == 0 ? 0 : (vb >= 64 ? ~0ull : ((1ull << vb) - 1));
        const uint64_t umin = kf.umin;
        const bool desc = kf.desc, nf = kf.nulls_first;
        const int type = kf.col.type;
        const ghb_out_column o = p.out_keys[j];
        for (int i = threadIdx.x; i < tile_n; i += kSortThreads) {
          const uint64_t k = s_keys[i];
          const uint32_t dk = (uint32_t)(k >> p.shift) & (kBins - 1);
          const int64_t pos = (int64_t)(s_gbase[dk] + (i - s_bexcl[dk]));
          const bool null = fs >= 0 && (((k >> fs) & 1ull) == 0) == nf;
          uint64_t u = (vb == 0 ? 0 : (k >> vs) & vmask) + umin;
          if (desc) u = ~u;
          const int64_t raw = type == GHB_DOUBLE ? (int64_t)unflip_f64_bits(u) : (int64_t)(u ^ 0x8000000000000000ull);
          write_raw(o, pos, type, raw, null);
        }
      }
      for (int i = threadIdx.x; i < tile_n; i += kSortThreads) {
        const uint64_t k = s_keys[i];
        const uint32_t dk = (uint32_t)(k >> p.shift) & (kBins - 1);
        const int64_t pos = (int64_t)(s_gbase[dk] + (i - s_bexcl[dk]));
        decode_value(p, (uint64_t)s_vals[i], pos);
      }
    } else
    for (int i = threadIdx.x; i < tile_n; i += kSortThreads) {
      uint64_t k = s_keys[i];
      uint32_t dk = (uint32_t)(k >> p.shift) & (kBins - 1);
      int64_t pos = (int64_t)(s_gbase[dk] + (i - s_bexcl[dk]));
      if (DST == kDstGather) {
        gather_write(p, (int64_t)s_vals[i], pos);
      } else {
        __stcs((unsigned long long*)p.keys_out + pos, (unsigned long long)k);
        vals_out[pos] = s_vals[i];
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

// Output in input order (keys all equal, or n tiny): gathers row r to r, or
// row perm[r] to r when a permutation is given.
template <typename V>
__global__ void sort_identity_kernel(PassParams p, const V* perm) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < p.n;
       r += (int64_t)gridDim.x * blockDim.x)
    gather_write(p, perm ? (int64_t)perm[r] : r, r);
}

static inline size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

// Scratch needed by sort_impl for n rows.
size_t sort_scratch_bytes(int64_t n) {
  int64_t ntiles = (n + kSortTile - 1) / kSortTile;
  size_t b = 0;
  b += 2 * align256((size_t)n * 8);                        // keys ping-pong
  b += 2 * align256((size_t)n * 8);                        // values ping-pong
  b += align256((size_t)ntiles * kBins * 8);               // look-back status
  b += align256((size_t)kMaxSeg * kMaxPasses * kBins * 4); // histograms
  b += align256(3 * 8 * kMaxSortKeys);                     // min/max
  return b + 4096;
}

template <typename V>
static void launch_pass(int src, int dst, int grid, size_t dyn, cudaStream_t s, const PassParams& pp) {
#define GHB_PASS(S, D) sort_pass_kernel<V, S, D><<<grid, kSortThreads, dyn, s>>>(pp)
  if (src == kSrcPacked && dst == kDstPacked) GHB_PASS(kSrcPacked, kDstPacked);
  else if (src == kSrcPacked && dst == kDstDecode) GHB_PASS(kSrcPacked, kDstDecode);
  else if (src == kSrcPacked && dst == kDstGather) GHB_PASS(kSrcPacked, kDstGather);
  else if (src == kSrcCols && dst == kDstPacked) GHB_PASS(kSrcCols, kDstPacked);
  else if (src == kSrcCols && dst == kDstDecode) GHB_PASS(kSrcCols, kDstDecode);
  else if (src == kSrcCols && dst == kDstGather) GHB_PASS(kSrcCols, kDstGather);
  else if (src == kSrcPerm && dst == kDstPacked) GHB_PASS(kSrcPerm, kDstPacked);
  else if (src == kSrcPerm && dst == kDstGather) GHB_PASS(kSrcPerm, kDstGather);
#undef GHB_PASS
}

template <typename V>
static int32_t set_smem(ghb_ctx* ctx, size_t dyn) {
#define GHB_ATTR(S, D) \
  do {                                                                      \
    int32_t _st = ensure_dyn_smem(ctx, (const void*)sort_pass_kernel<V, S, D>, dyn); \
    if (_st) return _st;                                                    \
  } while (0)
  GHB_ATTR(kSrcPacked, kDstPacked);
  GHB_ATTR(kSrcPacked, kDstDecode);
  GHB_ATTR(kSrcPacked, kDstGather);
  GHB_ATTR(kSrcCols, kDstPacked);
  GHB_ATTR(kSrcCols, kDstDecode);
  GHB_ATTR(kSrcCols, kDstGather);
  GHB_ATTR(kSrcPerm, kDstPacked);
  GHB_ATTR(kSrcPerm, kDstGather);
#undef GHB_ATTR
  return GHB_OK;
}

// kb / vb: key and value ping-pong buffers; packed: kb[0] / vb[0] already
// hold the packed keys and values of a one-segment key.
template <typename V>
static int32_t run_passes(ghb_ctx* ctx, PassParams& pp, const std::vector<Segment>& segs,
                          const std::vector<std::vector<int>>& run, const std::vector<uint32_t>& hist,
                          uint64_t* const kb[2], void* const vbv[2], bool packed, cudaStream_t stream) {
  int32_t st;
  int total = 0;
  for (auto& r : run) total += (int)r.size();
  const int64_t n = pp.n;
  V* vb[2] = {(V*)vbv[0], (V*)vbv[1]};
  const bool multi = segs.size() > 1;
  if (total == 0) {
    int grid = (int)std::min<int64_t>((n + 255) / 256, (int64_t)ctx->num_sms * 8);
    sort_identity_kernel<V><<<grid, 256, 0, stream>>>(pp, (const V*)nullptr);
    GHB_LAUNCH_CHECK(ctx);
    return GHB_OK;
  }
  uint64_t* status = nullptr;
  size_t status_bytes = (size_t)pp.ntiles * kBins * 8;
  if ((st = scratch_alloc(ctx, status_bytes, (void**)&status, stream))) return st;
  GHB_CUDA_TRY(ctx, cudaMemsetAsync(status, 0, status_bytes, stream));
  pp.status = status;
  const size_t dyn = (size_t)kSortTile * (8 + sizeof(V));
  if ((st = set_smem<V>(ctx, dyn))) return st;
  int per_sm = 0;
  GHB_CUDA_TRY(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                        &per_sm, sort_pass_kernel<V, kSrcPacked, kDstPacked>, kSortThreads, dyn));
  int pgrid = (int)std::min<int64_t>(pp.ntiles, (int64_t)ctx->num_sms * std::max(1, per_sm));
  int done = 0;
  bool have_perm = false;  // a previous pass left the row order in vb[cur]
  int cur = 0;
  for (size_t s = 0; s < segs.size(); s++) {
    pp.seg = segs[s];
    for (size_t i = 0; i < run[s].size(); i++) {
      int q = run[s][i];
      bool last = ++done == total;
      int src = i == 0 ? (have_perm ? kSrcPerm : packed ? kSrcPacked : kSrcCols) : kSrcPacked;
      int dst = last ? (multi ? kDstGather : kDstDecode) : kDstPacked;
      pp.shift = q * kDigitBits;
      uint32_t acc = 0;
      const uint32_t* h = &hist[((size_t)s * kMaxPasses + q) * kBins];
      for (int b = 0; b < kBins; b++) {
        pp.digit_base[b] = acc;
        acc += h[b];
      }
      pp.keys_in = kb[cur];
      pp.vals_in = vb[cur];
      pp.keys_out = kb[cur ^ 1];
      pp.vals_out = vb[cur ^ 1];
      // the status region was cleared at the start of this call: tag pass k with k
      pp.epoch = (uint32_t)done;
      launch_pass<V>(src, dst, pgrid, dyn, stream, pp);
      GHB_LAUNCH_CHECK(ctx);
      cur ^= 1;
      have_perm = true;
    }
  }
  return GHB_OK;
}

int32_t sort_impl(ghb_ctx* ctx, const ghb_column* keys, const int32_t* orders,
                  const int32_t* null_orders, int32_t nkeys, const ghb_column* payload,
                  int32_t npayload, ghb_out_column* out_keys, ghb_out_column* out_payload,
                  int32_t* out_rowid, const ghb_sort_cfg* cfg, cudaStream_t stream) {
  (void)cfg;
  if (nkeys < 1 || nkeys > kMaxSortKeys)
    return set_error(ctx, GHB_ERR_INVALID, "nkeys=%d outside [1,%d]", nkeys, kMaxSortKeys);
  if (npayload < 0 || npayload > kMaxSortPay)
    return set_error(ctx, GHB_ERR_INVALID, "npayload=%d outside [0,%d]", npayload, kMaxSortPay);
  int64_t n = 0;
  int32_t st = validate_columns(ctx, keys, nkeys, &n);
  if (st) return st;
  if (npayload) {
    int64_t pn = 0;
    if ((st = validate_columns(ctx, payload, npayload, &pn))) return st;
    if (pn != n) return set_error(ctx, GHB_ERR_INVALID, "payload rows %lld != key rows %lld",
                                  (long long)pn, (long long)n);
  }
  if (n >= (int64_t)INT32_MAX) return set_error(ctx, GHB_ERR_UNSUPPORTED, "sort of 2^31 rows or more");
  if (!out_keys) return set_error(ctx, GHB_ERR_INVALID, "out_keys is NULL");
  for (int j = 0; j < nkeys; j++)
    if (out_keys[j].type != keys[j].type || (!out_keys[j].data && n > 0))
      return set_error(ctx, GHB_ERR_INVALID, "out_keys[%d]: bad type or data", j);
  for (int j = 0; j < npayload; j++)
    if (out_payload[j].type != payload[j].type || (!out_payload[j].data && n > 0))
      return set_error(ctx, GHB_ERR_INVALID, "out_payload[%d]: bad type or data", j);
  if (n == 0) return GHB_OK;

  PassParams pp;
  std::memset(&pp, 0, sizeof(pp));
  KeySet& K = pp.K;
  K.nkeys = nkeys;
  for (int j = 0; j < nkeys; j++) {
    K.k[j].col = keys[j];
    K.k[j].desc = orders && orders[j] == GHB_DESC;
    int no = null_orders ? null_orders[j] : GHB_NULLS_DEFAULT;
    K.k[j].nulls_first = no == GHB_NULLS_FIRST || (no == GHB_NULLS_DEFAULT && !K.k[j].desc);
  }
  unsigned long long* d_mm = nullptr;
  uint32_t* d_hist = nullptr;
  if ((st = scratch_alloc(ctx, 3 * 8 * kMaxSortKeys, (void**)&d_mm, stream))) return st;
  if ((st = scratch_alloc(ctx, (size_t)kMaxSeg * kMaxPasses * kBins * 4, (void**)&d_hist, stream))) return st;
  std::vector<unsigned long long> mm_init(3 * kMaxSortKeys, 0);
  for (int j = 0; j < kMaxSortKeys; j++) mm_init[3 * j] = ~0ull;
  GHB_CUDA_TRY(ctx, cudaMemcpyAsync(d_mm, mm_init.data(), mm_init.size() * 8, cudaMemcpyHostToDevice, stream));
  int grid = (int)std::min<int64_t>((n + 255) / 256, (int64_t)ctx->num_sms * 8);
  MinMaxParams mp;
  mp.K = K;
  mp.n = n;
  mp.out = d_mm;
  sort_minmax_kernel<<<grid, 256, 0, stream>>>(mp);
  GHB_LAUNCH_CHECK(ctx);
  unsigned long long mm[3 * kMaxSortKeys];
  GHB_CUDA_TRY(ctx, cudaMemcpyAsync(mm, d_mm, sizeof(mm), cudaMemcpyDeviceToHost, stream));
  GHB_CUDA_TRY(ctx, cudaStreamSynchronize(stream));

  // plan: least significant key first, value bits then its NULL flag above
  std::vector<Segment> segs(1);
  std::memset(&segs[0], 0, sizeof(Segment));
  auto add_sub = [&](int key, int is_flag, int bits) {
    if (bits == 0) return;
    if (segs.back().bits + bits > 64) {
      segs.emplace_back();
      std::memset(&segs.back(), 0, sizeof(Segment));
    }
    Segment& sg = segs.back();
    SubField& sf = sg.f[sg.n++];
    sf.key = (int8_t)key;
    sf.is_flag = (int8_t)is_flag;
    sf.bits = (int8_t)bits;
    sf.shift = (int8_t)sg.bits;
    sg.bits += bits;
  };
  for (int j = nkeys - 1; j >= 0; j--) {
    KeyField& f = K.k[j];
    bool anyval = mm[3 * j] <= mm[3 * j + 1];
    f.umin = anyval ? mm[3 * j] : 0;
    uint64_t range = anyval ? mm[3 * j + 1] - mm[3 * j] : 0;
    f.vbits = range == 0 ? 0 : 64 - __builtin_clzll(range);
    f.has_null = mm[3 * j + 2] ? 1 : 0;
    add_sub(j, 0, f.vbits);
    add_sub(j, 1, f.has_null);
  }
  if (segs.size() > (size_t)kMaxSeg) return set_error(ctx, GHB_ERR_UNSUPPORTED, "too many key segments");
  const bool multi = segs.size() > 1;

  // the value: the single payload itself, else the row index
  const bool carry_rowid = multi || out_rowid != nullptr || npayload != 1 ||
                           payload[0].null_mode == GHB_NULLS_BYTEMAP;
  const bool wide = !carry_rowid && type_width(payload[0].type) == 8;
  const size_t vw = wide ? 8 : 4;
  uint64_t* kb[2] = {nullptr, nullptr};
  void* vb[2] = {nullptr, nullptr};
  for (int i = 0; i < 2; i++) {
    if ((st = scratch_alloc(ctx, (size_t)n * 8, (void**)&kb[i], stream))) return st;
    if ((st = scratch_alloc(ctx, (size_t)n * vw, &vb[i], stream))) return st;
  }

  // histograms of every segment, one read each, then one sync; a
  // one-segment key is packed on the way
  GHB_CUDA_TRY(ctx, cudaMemsetAsync(d_hist, 0, segs.size() * kMaxPasses * kBins * 4, stream));
  for (size_t s = 0; s < segs.size(); s++) {
    int np = (segs[s].bits + kDigitBits - 1) / kDigitBits;
    if (np == 0) continue;
    HistParams hp;
    hp.K = K;
    hp.seg = segs[s];
    hp.n = n;
    hp.npasses = np;
    hp.hist = d_hist + s * kMaxPasses * kBins;
    for (int i = 0; i < segs[s].n; i++) {
      const SubField& sf = segs[s].f[i];
      const KeyField& kf = K.k[sf.key];
      SubPlan& sp = hp.sub[i];
      sp.col = kf.col;
      sp.umin = kf.umin;
      sp.shift = sf.shift;
      sp.is_flag = sf.is_flag;
      sp.desc = (int8_t)kf.desc;
      sp.nulls_first = (int8_t)kf.nulls_first;
      sp.has_null = (int8_t)kf.has_null;
    }
    hp.keys_out = multi ? nullptr : kb[0];
    hp.vals_out = vb[0];
    hp.vals_wide = wide ? 1 : 0;
    hp.carry_rowid = carry_rowid ? 1 : 0;
    hp.pay_src = carry_rowid ? ghb_column{} : payload[0];
    // 16-byte loads and stores when every column read allows them
    auto vec_ok = [](const ghb_column& c) {
      return c.null_mode != GHB_NULLS_BYTEMAP && ((uintptr_t)c.data & 15) == 0;
    };
    hp.vec = 1;
    for (int i = 0; i < segs[s].n; i++) hp.vec &= vec_ok(hp.sub[i].col) ? 1 : 0;
    if (!carry_rowid) hp.vec &= vec_ok(hp.pay_src) ? 1 : 0;
    if (hp.keys_out && (((uintptr_t)hp.keys_out | (uintptr_t)hp.vals_out) & 15)) hp.vec = 0;
    sort_hist_kernel<<<std::min(grid, ctx->num_sms * 8), 256, 0, stream>>>(hp);
    GHB_LAUNCH_CHECK(ctx);
  }
  std::vector<uint32_t> hist((size_t)segs.size() * kMaxPasses * kBins, 0);
  GHB_CUDA_TRY(ctx, cudaMemcpyAsync(hist.data(), d_hist, hist.size() * 4, cudaMemcpyDeviceToHost, stream));
  GHB_CUDA_TRY(ctx, cudaStreamSynchronize(stream));
  std::vector<std::vector<int>> run(segs.size());
  for (size_t s = 0; s < segs.size(); s++) {
    int np = (segs[s].bits + kDigitBits - 1) / kDigitBits;
    for (int q = 0; q < np; q++) {
      bool trivial = false;
      for (int b = 0; b < kBins; b++)
        if (hist[((size_t)s * kMaxPasses + q) * kBins + b] == (uint32_t)n) trivial = true;
      if (!trivial) run[s].push_back(q);
    }
  }

  pp.carry_rowid = carry_rowid ? 1 : 0;
  for (int j = 0; j < kMaxSortKeys; j++) {
    pp.dec_vbits[j] = 0;
    pp.dec_vshift[j] = 0;
    pp.dec_fshift[j] = -1;
  }
  if (!multi)
    for (int i = 0; i < segs[0].n; i++) {
      const SubField& sf = segs[0].f[i];
      if (sf.is_flag) {
        pp.dec_fshift[sf.key] = sf.shift;
      } else {
        pp.dec_vbits[sf.key] = sf.bits;
        pp.dec_vshift[sf.key] = sf.shift;
      }
    }
  if (!carry_rowid) pp.pay_src = payload[0];
  for (int j = 0; j < nkeys; j++) pp.out_keys[j] = out_keys[j];
  pp.npay = npayload;
  for (int j = 0; j < npayload; j++) {
    pp.pay[j] = payload[j];
    pp.out_pay[j] = out_payload[j];
  }
  pp.out_rowid = out_rowid;
  pp.n = n;
  pp.ntiles = (n + kSortTile - 1) / kSortTile;
  pp.counters = ctx->d_counters + 2;
  pp.dev_status = ctx->d_status;
  pp.spin_limit = ctx->spin_limit;
  const bool packed = !multi;
  if (wide) return run_passes<uint64_t>(ctx, pp, segs, run, hist, kb, vb, packed, stream);
  return run_passes<uint32_t>(ctx, pp, segs, run, hist, kb, vb, packed, stream);
}

// ---------------------------------------------------------------- STRING keys
// A STRING sort key compares as Hive's StringExpr.compare (storage-api/src/
// java/org/apache/hadoop/hive/ql/exec/vector/expressions/StringExpr.java:
// 37-47): unsigned bytes, then length.  It is sorted as the tuple
// (chunk 0, ..., chunk m-1, length) of fixed-width keys, chunk i being bytes
// [8i, 8i + 8) big-endian with 0x00 past the end (top bit flipped, so the
// signed order of the int64 is the unsigned order of the bytes): equal
// chunks with a shorter length sort first, as the byte compare does.  A NULL
// string is NULL in every part.
__global__ void __launch_bounds__(256) string_maxlen_kernel(ghb_column c, unsigned long long* out) {
  const int2* aux = (const int2*)c.aux;
  unsigned long long mx = 0;
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < c.n; r += (int64_t)gridDim.x * blockDim.x) {
    const int2 ix = aux[r];
    if (ix.x >= 0) mx = max(mx, (unsigned long long)(ix.y - ix.x));
  }
  for (int o = 16; o > 0; o >>= 1) mx = max(mx, __shfl_down_sync(0xffffffffu, mx, o));
  if ((threadIdx.x & 31) == 0 && mx) atomicMax(out, mx);
}

__global__ void __launch_bounds__(256) string_parts_kernel(ghb_column c, int32_t nchunks, int64_t* chunks,
                                                            int32_t* lens, uint8_t* nulls) {
  const int2* aux = (const int2*)c.aux;
  const uint8_t* bytes = (const uint8_t*)c.data;
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < c.n; r += (int64_t)gridDim.x * blockDim.x) {
    const int2 ix = aux[r];
    const bool null = ix.x < 0;
    const int len = null ? 0 : ix.y - ix.x;
    nulls[r] = null ? 1 : 0;
    lens[r] = len;
    for (int k = 0; k < nchunks; k++) {
      uint64_t w = 0;
      for (int b = 0; b < 8; b++) {
        const int at = 8 * k + b;
        w = (w << 8) | (at < len ? (uint64_t)bytes[ix.x + at] : 0ull);
      }
      chunks[(int64_t)k * c.n + r] = (int64_t)(w ^ 0x8000000000000000ull);
    }
  }
}

// out[i] = the [start,end) of row rowid[i] of a STRING column (NULL: -1, -1).
__global__ void __launch_bounds__(256) string_gather_kernel(ghb_column c, const int32_t* rowid, int64_t n,
                                                             ghb_out_column out) {
  const int2* aux = (const int2*)c.aux;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int2 ix = aux[rowid[i]];
    ((int2*)out.data)[i] = ix;
    if (out.is_null) out.is_null[i] = ix.x < 0 ? 1 : 0;
  }
}

// ORDER BY with STRING keys: each STRING key becomes its parts; the sort
// runs on the parts with the row ids carried; the STRING outputs are
// gathered from the row ids.
static int32_t sort_with_strings(ghb_ctx* ctx, const ghb_column* keys, const int32_t* orders,
                                 const int32_t* null_orders, int32_t nkeys, const ghb_column* payload,
                                 int32_t npayload, ghb_out_column* out_keys, ghb_out_column* out_payload,
                                 int32_t* out_rowid, const ghb_sort_cfg* cfg, cudaStream_t stream) {
  int64_t n = 0;
  int32_t st = validate_columns(ctx, keys, nkeys, &n, true);
  if (st) return st;
  if (n >= (int64_t)INT32_MAX) return set_error(ctx, GHB_ERR_UNSUPPORTED, "sort of 2^31 rows or more");
  if (!out_keys) return set_error(ctx, GHB_ERR_INVALID, "out_keys is NULL");
  // the longest string of each STRING key (one read, one synchronisation)
  unsigned long long* d_len = nullptr;
  if ((st = scratch_alloc(ctx, 8 * kMaxSortKeys, (void**)&d_len, stream))) return st;
  GHB_CUDA_TRY(ctx, cudaMemsetAsync(d_len, 0, 8 * kMaxSortKeys, stream));
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)ctx->num_sms * 8));
  for (int j = 0; j < nkeys; j++)
    if (keys[j].type == GHB_STRING) {
      string_maxlen_kernel<<<grid, 256, 0, stream>>>(keys[j], d_len + j);
      GHB_LAUNCH_CHECK(ctx);
    }
  unsigned long long len[kMaxSortKeys];
  GHB_CUDA_TRY(ctx, cudaMemcpyAsync(len, d_len, sizeof(len), cudaMemcpyDeviceToHost, stream));
  GHB_CUDA_TRY(ctx, cudaStreamSynchronize(stream));
  std::vector<ghb_column> ek;
  std::vector<int32_t> eo, en;
  std::vector<ghb_out_column> eout;
  for (int j = 0; j < nkeys; j++) {
    const int32_t o = orders ? orders[j] : GHB_ASC, no = null_orders ? null_orders[j] : GHB_NULLS_DEFAULT;
    if (keys[j].type != GHB_STRING) {
      ek.push_back(keys[j]);
      eo.push_back(o);
      en.push_back(no);
      eout.push_back(out_keys[j]);
      continue;
    }
    const int m = (int)((len[j] + 7) / 8);
    if ((int)ek.size() + m + 1 > kMaxSortKeys)
      return set_error(ctx, GHB_ERR_UNSUPPORTED, "STRING sort key %d of up to %llu bytes needs more than %d key "
                       "parts in all", j, len[j], kMaxSortKeys);
    int64_t* chunks = nullptr;
    int32_t* lens = nullptr;
    uint8_t* nulls = nullptr;
    if ((st = scratch_alloc(ctx, (size_t)std::max<int64_t>(n, 1) * 8 * std::max(m, 1), (void**)&chunks, stream)) ||
        (st = scratch_alloc(ctx, (size_t)std::max<int64_t>(n, 1) * 4, (void**)&lens, stream)) ||
        (st = scratch_alloc(ctx, (size_t)std::max<int64_t>(n, 1), (void**)&nulls, stream)))
      return st;
    string_parts_kernel<<<grid, 256, 0, stream>>>(keys[j], m, chunks, lens, nulls);
    GHB_LAUNCH_CHECK(ctx);
    for (int k = 0; k <= m; k++) {
      ghb_column pc{k < m ? GHB_LONG : GHB_INT, GHB_NULLS_BYTEMAP, k < m ? (const void*)(chunks + (int64_t)k * n)
                                                                         : (const void*)lens,
                    nulls, nullptr, n};
      ek.push_back(pc);
      eo.push_back(o);
      en.push_back(no);
      // the parts' sorted values are not kept
      void* od = nullptr;
      if ((st = scratch_alloc(ctx, (size_t)std::max<int64_t>(n, 1) * type_width(pc.type), &od, stream))) return st;
      eout.push_back(ghb_out_column{pc.type, 0, od, nullptr});
    }
  }
  int32_t* rowid = out_rowid;
  if (!rowid && (st = scratch_alloc(ctx, (size_t)std::max<int64_t>(n, 1) * 4, (void**)&rowid, stream))) return st;
  st = sort_impl(ctx, ek.data(), eo.data(), en.data(), (int32_t)ek.size(), payload, npayload, eout.data(),
                 out_payload, rowid, cfg, stream);
  if (st) return st;
  for (int j = 0; j < nkeys; j++)
    if (keys[j].type == GHB_STRING) {
      if (out_keys[j].type != GHB_STRING || (!out_keys[j].data && n > 0))
        return set_error(ctx, GHB_ERR_INVALID, "out_keys[%d]: bad type or data", j);
      string_gather_kernel<<<grid, 256, 0, stream>>>(keys[j], rowid, n, out_keys[j]);
      GHB_LAUNCH_CHECK(ctx);
    }
  return GHB_OK;
}

// Scratch a sort with STRING keys needs beside the sort's own.
static size_t string_sort_scratch_bytes(const ghb_column* keys, int32_t nkeys, int64_t n) {
  size_t b = 4096 + (size_t)n * 4 + 256;
  for (int j = 0; j < nkeys; j++)
    if (keys[j].type == GHB_STRING) b += (size_t)n * (2 * 8 * kMaxSortKeys + 4 + 4 + 1) + 8 * 1024;
  return b;
}

}  // namespace ghb

using namespace ghb;

extern "C" int32_t ghb_sort(ghb_ctx* ctx, const ghb_column* keys, const int32_t* orders,
                            const int32_t* null_orders, int32_t nkeys, const ghb_column* payload,
                            int32_t npayload, ghb_out_column* out_keys, ghb_out_column* out_payload,
                            int32_t* out_rowid, const ghb_sort_cfg* cfg, void* stream) {
  if (!ctx) return GHB_ERR_INVALID;
  CallScope cs(ctx, "sort", (cudaStream_t)stream);
  int64_t n = keys && nkeys > 0 ? keys[0].n : 0;
  cs.rows(n);
  cs.bytes(cols_bytes(keys, nkeys) + cols_bytes(payload, npayload));
  scratch_reset(ctx);
  bool strings = false;
  for (int j = 0; keys && j < nkeys && j < kMaxSortKeys; j++) strings |= keys[j].type == GHB_STRING;
  const size_t extra = strings ? string_sort_scratch_bytes(keys, nkeys, n) : 0;
  int32_t st = scratch_reserve(ctx, sort_scratch_bytes(n) + extra, (cudaStream_t)stream);
  if (st) return cs.done(st);
  if (strings)
    return cs.done(sort_with_strings(ctx, keys, orders, null_orders, nkeys, payload, npayload, out_keys,
                                     out_payload, out_rowid, cfg, (cudaStream_t)stream));
  return cs.done(sort_impl(ctx, keys, orders, null_orders, nkeys, payload, npayload, out_keys, out_payload,
                           out_rowid, cfg, (cudaStream_t)stream));
}
