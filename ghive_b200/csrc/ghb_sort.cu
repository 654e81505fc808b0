// ghb_sort.cu — stable ORDER BY sort (S1): LSD radix sort on a packed key.
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
//   1. analyse  one read of the key columns: per key the min/max of its
//               order image and whether it holds NULLs;
//   2. plan     (host) each key becomes a bit field [null bit][value - min]
//               of just the width its range needs; the fields are packed
//               most-significant-key-first into one 64-bit word;
//   3. histogram one read: 8-bit digit histograms of every pass at once;
//               passes whose digit is constant are skipped;
//   4. passes   onesweep-style: each CTA claims a tile, ranks its keys by
//               digit with warp ballots (stable), gets each digit's global
//               offset by decoupled look-back over earlier tiles, reorders
//               the tile in shared memory and writes runs per digit.  The
//               first pass reads the user's columns and packs on the fly; the
//               last pass unpacks straight into the user's output columns.
// The carried value is the payload itself when there is one payload column
// and no permutation is asked for, else the row index (payloads are then
// gathered in the last pass).
#include <algorithm>
#include <vector>

#include "ghb_ctx.hpp"

namespace ghb {

constexpr int kSortThreads = 256;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortThreads * kSortItems;   // 4096
constexpr int kDigitBits = 8;
constexpr int kBins = 1 << kDigitBits;
constexpr int kMaxPasses = 8;
constexpr int kMaxSortKeys = 8;
constexpr int kMaxSortPay = 8;
constexpr uint32_t kSFlagA = 1u << 30, kSFlagP = 2u << 30, kSCount = (1u << 30) - 1;

struct KeyField {
  ghb_column col;
  int32_t desc;
  int32_t nulls_first;
  int32_t has_null_bit;  // field carries a null flag above its value bits
  int32_t vbits;         // value bits
  int32_t shift;         // position of the field's lowest bit in the packed key
  uint64_t umin;         // min of the (possibly inverted) order image
};

struct SortLayout {
  int32_t nkeys;
  KeyField f[kMaxSortKeys];
};

__device__ __forceinline__ uint64_t key_image(const ghb_column& c, int64_t raw) {
  return c.type == GHB_DOUBLE ? flip_f64_bits((uint64_t)raw) : flip_i64(raw);
}

// ---------------------------------------------------------------- analyse
struct MinMaxParams {
  SortLayout L;
  int64_t n;
  unsigned long long* out;  // per key: [0] min image, [1] max image, [2] any NULL
};

__global__ void __launch_bounds__(256) sort_minmax_kernel(MinMaxParams p) {
  for (int j = 0; j < p.L.nkeys; j++) {
    const KeyField& f = p.L.f[j];
    unsigned long long mn = ~0ull, mx = 0, anynull = 0;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < p.n;
         r += (int64_t)gridDim.x * blockDim.x) {
      int64_t raw = ld_raw(f.col, r);
      if (raw_is_null(f.col, raw, r)) { anynull = 1; continue; }
      uint64_t u = key_image(f.col, raw);
      if (f.desc) u = ~u;
      mn = min(mn, (unsigned long long)u);
      mx = max(mx, (unsigned long long)u);
    }
    for (int o = 16; o > 0; o >>= 1) {
      mn = min(mn, __shfl_down_sync(0xffffffffu, mn, o));
      mx = max(mx, __shfl_down_sync(0xffffffffu, mx, o));
      anynull |= __shfl_down_sync(0xffffffffu, anynull, o);
    }
    if ((threadIdx.x & 31) == 0) {
      atomicMin(&p.out[3 * j], mn);
      atomicMax(&p.out[3 * j + 1], mx);
      if (anynull) atomicOr(&p.out[3 * j + 2], 1ull);
    }
  }
}

// Packed key of row r.
__device__ __forceinline__ uint64_t pack_row(const SortLayout& L, int64_t r) {
  uint64_t k = 0;
  for (int j = 0; j < L.nkeys; j++) {
    const KeyField& f = L.f[j];
    int64_t raw = ld_raw(f.col, r);
    uint64_t field;
    if (f.col.null_mode != GHB_NULLS_NONE && raw_is_null(f.col, raw, r)) {
      field = f.nulls_first ? 0 : (1ull << f.vbits);   // value bits 0
    } else {
      uint64_t u = key_image(f.col, raw);
      if (f.desc) u = ~u;
      field = u - f.umin;
      if (f.has_null_bit && f.nulls_first) field |= 1ull << f.vbits;
    }
    k |= field << f.shift;
  }
  return k;
}

// ---------------------------------------------------------------- histogram
struct HistParams {
  SortLayout L;
  int64_t n;
  int32_t npasses;
  uint32_t* hist;  // [npasses][kBins]
};

__global__ void __launch_bounds__(256) sort_hist_kernel(HistParams p) {
  __shared__ uint32_t sh[kMaxPasses][kBins];
  for (int i = threadIdx.x; i < kMaxPasses * kBins; i += blockDim.x) (&sh[0][0])[i] = 0;
  __syncthreads();
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < p.n;
       r += (int64_t)gridDim.x * blockDim.x) {
    uint64_t k = pack_row(p.L, r);
    for (int q = 0; q < p.npasses; q++) atomicAdd(&sh[q][(k >> (q * kDigitBits)) & (kBins - 1)], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < p.npasses * kBins; i += blockDim.x) {
    uint32_t v = (&sh[0][0])[i];
    if (v) atomicAdd(&p.hist[i], v);
  }
}

// ---------------------------------------------------------------- passes
struct PassParams {
  SortLayout L;
  int64_t n;
  int64_t ntiles;
  int32_t shift;
  int32_t carry_rowid;       // value = row index (else the single payload's raw bits)
  // packed buffers
  const uint64_t* keys_in;
  const uint64_t* vals_in;
  uint64_t* keys_out;
  uint64_t* vals_out;
  // first pass source
  ghb_column pay_src;        // single carried payload (when !carry_rowid)
  // last pass destination
  ghb_out_column out_keys[kMaxSortKeys];
  int32_t npay;
  ghb_column pay[kMaxSortPay];
  ghb_out_column out_pay[kMaxSortPay];
  int32_t* out_rowid;
  uint32_t digit_base[kBins];  // exclusive global offset of each digit
  uint32_t* status;           // [ntiles][kBins]
  unsigned long long* counters;
  int32_t* dev_status;
};

__device__ __forceinline__ void unpack_write(const PassParams& p, uint64_t k, uint64_t v, int64_t pos) {
  for (int j = 0; j < p.L.nkeys; j++) {
    const KeyField& f = p.L.f[j];
    uint64_t field = (k >> f.shift);
    uint64_t vmask = f.vbits >= 64 ? ~0ull : ((1ull << f.vbits) - 1);
    bool null = false;
    if (f.has_null_bit) {
      bool flag = (field >> f.vbits) & 1ull;
      null = f.nulls_first ? !flag : flag;
    }
    const ghb_out_column& o = p.out_keys[j];
    if (null) {
      if (o.is_null) o.is_null[pos] = 1;
      if (o.type == GHB_INT) ((int32_t*)o.data)[pos] = INT32_MAX;
      else if (o.type == GHB_LONG) ((int64_t*)o.data)[pos] = INT64_MAX;
      else ((long long*)o.data)[pos] = 0x7ff8000000000000ll;
      continue;
    }
    uint64_t u = (field & vmask) + f.umin;
    if (f.desc) u = ~u;
    int64_t raw = f.col.type == GHB_DOUBLE ? (int64_t)unflip_f64_bits(u) : (int64_t)(u ^ 0x8000000000000000ull);
    if (o.type == GHB_INT) ((int32_t*)o.data)[pos] = (int32_t)raw;
    else ((long long*)o.data)[pos] = raw;
    if (o.is_null) o.is_null[pos] = 0;
  }
  if (p.carry_rowid) {
    int64_t row = (int64_t)v;
    if (p.out_rowid) p.out_rowid[pos] = (int32_t)row;
    for (int j = 0; j < p.npay; j++) {
      const ghb_column& c = p.pay[j];
      const ghb_out_column& o = p.out_pay[j];
      int64_t raw = ld_raw(c, row);
      if (c.type == GHB_INT) ((int32_t*)o.data)[pos] = (int32_t)raw;
      else ((long long*)o.data)[pos] = raw;
      if (o.is_null) o.is_null[pos] = (c.null_mode != GHB_NULLS_NONE && raw_is_null(c, raw, row)) ? 1 : 0;
    }
  } else if (p.npay == 1) {
    const ghb_out_column& o = p.out_pay[0];
    if (p.pay[0].type == GHB_INT) ((int32_t*)o.data)[pos] = (int32_t)v;
    else ((unsigned long long*)o.data)[pos] = v;
    if (o.is_null) {
      const ghb_column& c = p.pay[0];
      o.is_null[pos] = (c.null_mode == GHB_NULLS_SENTINEL && raw_is_null(c, (int64_t)v, 0)) ? 1 : 0;
    }
  }
}

template <bool FIRST, bool LAST>
__global__ void __launch_bounds__(kSortThreads) sort_pass_kernel(PassParams p) {
  __shared__ uint32_t s_whist[kSortThreads / 32][kBins];  // per-warp counts, then exclusive over warps
  __shared__ uint32_t s_bexcl[kBins];                      // block-local exclusive offset per digit
  __shared__ uint64_t s_gbase[kBins];                      // global destination of each digit's run
  extern __shared__ uint64_t s_dyn[];                      // reordered tile: keys, then values
  uint64_t* s_keys = s_dyn;
  uint64_t* s_vals = s_dyn + kSortTile;
  __shared__ int64_t s_tile;
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const unsigned lt = (1u << lane) - 1u;

  while (true) {
    if (threadIdx.x == 0) s_tile = (int64_t)atomicAdd(&p.counters[0], 1ull);
    for (int i = threadIdx.x; i < (kSortThreads / 32) * kBins; i += kSortThreads) (&s_whist[0][0])[i] = 0;
    __syncthreads();
    const int64_t tile = s_tile;
    if (tile >= p.ntiles) break;
    const int64_t wbase = tile * kSortTile + (int64_t)warp * (32 * kSortItems);

    uint64_t key[kSortItems], val[kSortItems];
    uint32_t rank[kSortItems];
#pragma unroll
    for (int k = 0; k < kSortItems; k++) {
      int64_t row = wbase + k * 32 + lane;
      bool live = row < p.n;
      if (FIRST) {
        key[k] = live ? pack_row(p.L, row) : ~0ull;
        val[k] = p.carry_rowid ? (uint64_t)row : (live ? (uint64_t)ld_raw(p.pay_src, row) : 0);
      } else {
        key[k] = live ? p.keys_in[row] : ~0ull;
        val[k] = live ? p.vals_in[row] : 0;
      }
    }
    // stable rank of each key among the warp's keys with the same digit
#pragma unroll
    for (int k = 0; k < kSortItems; k++) {
      int64_t row = wbase + k * 32 + lane;
      bool live = row < p.n;
      uint32_t d = (uint32_t)(key[k] >> p.shift) & (kBins - 1);
      unsigned peers = __ballot_sync(0xffffffffu, live);
#pragma unroll
      for (int b = 0; b < kDigitBits; b++) {
        unsigned bb = __ballot_sync(0xffffffffu, (d >> b) & 1u);
        peers &= ((d >> b) & 1u) ? bb : ~bb;
      }
      uint32_t before = live ? s_whist[warp][d] : 0;
      __syncwarp();
      if (live && (peers & lt) == 0) s_whist[warp][d] = before + __popc(peers);
      __syncwarp();
      rank[k] = before + __popc(peers & lt);
    }
    __syncthreads();
    // per digit (one thread each): exclusive over warps, block total
    uint32_t total = 0;
    {
      const int d = threadIdx.x;  // kSortThreads == kBins
#pragma unroll
      for (int w = 0; w < kSortThreads / 32; w++) {
        uint32_t c = s_whist[w][d];
        s_whist[w][d] = total;
        total += c;
      }
    }
    // publish this tile's count of digit d, then look back for its prefix
    {
      const int d = threadIdx.x;
      uint32_t* st = p.status + tile * kBins;
      uint64_t excl = 0;
      if (tile == 0) {
        atomicExch(&st[d], kSFlagP | total);
      } else {
        atomicExch(&st[d], kSFlagA | total);
        int64_t t = tile - 1;
        int spins = 0;
        while (t >= 0) {
          uint32_t v = *(volatile uint32_t*)&p.status[t * kBins + d];
          if (v & kSFlagP) { excl += v & kSCount; break; }
          if (v & kSFlagA) { excl += v & kSCount; t--; continue; }
          if (++spins > kSpinLimit) { raise_status(p.dev_status, kDevTimeout); break; }
        }
        atomicExch(&st[d], kSFlagP | (uint32_t)((excl + total) & kSCount));
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
      __shared__ uint32_t s_wsum[kSortThreads / 32];
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
      s_bexcl[threadIdx.x] = s_wsum[warp] + incl - total;
    }
    __syncthreads();
    // scatter into shared memory in digit order (stable)
#pragma unroll
    for (int k = 0; k < kSortItems; k++) {
      int64_t row = wbase + k * 32 + lane;
      if (row >= p.n) continue;
      uint32_t d = (uint32_t)(key[k] >> p.shift) & (kBins - 1);
      uint32_t at = s_bexcl[d] + s_whist[warp][d] + rank[k];
      s_keys[at] = key[k];
      s_vals[at] = val[k];
    }
    __syncthreads();
    // write runs: element i of the reordered tile goes to gbase[d] + (i - bexcl[d])
    const int64_t tile_n = min((int64_t)kSortTile, p.n - tile * kSortTile);
    for (int i = threadIdx.x; i < tile_n; i += kSortThreads) {
      uint64_t k = s_keys[i];
      uint32_t d = (uint32_t)(k >> p.shift) & (kBins - 1);
      int64_t pos = (int64_t)(s_gbase[d] + (i - s_bexcl[d]));
      if (LAST) {
        unpack_write(p, k, s_vals[i], pos);
      } else {
        p.keys_out[pos] = k;
        p.vals_out[pos] = s_vals[i];
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

// Identity pass for an input whose packed keys are all equal (or n <= 1):
// copies keys and payloads in input order.
__global__ void sort_copy_kernel(PassParams p) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < p.n;
       r += (int64_t)gridDim.x * blockDim.x) {
    uint64_t k = pack_row(p.L, r);
    uint64_t v = p.carry_rowid ? (uint64_t)r : (uint64_t)ld_raw(p.pay_src, r);
    unpack_write(p, k, v, r);
  }
}

// Scratch needed by sort_impl for n rows.
size_t sort_scratch_bytes(int64_t n) {
  int64_t ntiles = (n + kSortTile - 1) / kSortTile;
  size_t b = 0;
  b += 2 * (((size_t)n * 8 + 255) & ~(size_t)255);       // keys ping-pong
  b += 2 * (((size_t)n * 8 + 255) & ~(size_t)255);       // values ping-pong
  b += (size_t)kMaxPasses * ntiles * kBins * 4 + 256;    // look-back status
  b += (size_t)kMaxPasses * kBins * 4 + 256;             // histograms
  b += 3 * 8 * kMaxSortKeys + 256;                       // min/max
  return b + 4096;
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
  if (n >= (int64_t)kSCount) return set_error(ctx, GHB_ERR_UNSUPPORTED, "sort of more than 2^30-1 rows");
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
  SortLayout& L = pp.L;
  L.nkeys = nkeys;
  for (int j = 0; j < nkeys; j++) {
    L.f[j].col = keys[j];
    L.f[j].desc = orders && orders[j] == GHB_DESC;
    int no = null_orders ? null_orders[j] : GHB_NULLS_DEFAULT;
    L.f[j].nulls_first = no == GHB_NULLS_FIRST || (no == GHB_NULLS_DEFAULT && !L.f[j].desc);
  }
  unsigned long long* d_mm = nullptr;
  uint32_t* d_hist = nullptr;
  if ((st = scratch_alloc(ctx, 3 * 8 * kMaxSortKeys, (void**)&d_mm, stream))) return st;
  if ((st = scratch_alloc(ctx, kMaxPasses * kBins * 4, (void**)&d_hist, stream))) return st;
  std::vector<unsigned long long> mm_init(3 * kMaxSortKeys, 0);
  for (int j = 0; j < kMaxSortKeys; j++) mm_init[3 * j] = ~0ull;
  GHB_CUDA_TRY(ctx, cudaMemcpyAsync(d_mm, mm_init.data(), mm_init.size() * 8, cudaMemcpyHostToDevice, stream));
  GHB_CUDA_TRY(ctx, cudaMemsetAsync(d_hist, 0, kMaxPasses * kBins * 4, stream));
  int grid = (int)std::min<int64_t>((n + 255) / 256, (int64_t)ctx->num_sms * 8);
  MinMaxParams mp;
  mp.L = L;
  mp.n = n;
  mp.out = d_mm;
  sort_minmax_kernel<<<grid, 256, 0, stream>>>(mp);
  GHB_LAUNCH_CHECK(ctx);
  unsigned long long mm[3 * kMaxSortKeys];
  GHB_CUDA_TRY(ctx, cudaMemcpyAsync(mm, d_mm, sizeof(mm), cudaMemcpyDeviceToHost, stream));
  GHB_CUDA_TRY(ctx, cudaStreamSynchronize(stream));

  // plan the packed layout: key 0 most significant
  int bits = 0;
  for (int j = nkeys - 1; j >= 0; j--) {
    KeyField& f = L.f[j];
    bool anyval = mm[3 * j] <= mm[3 * j + 1];
    f.umin = anyval ? mm[3 * j] : 0;
    uint64_t range = anyval ? mm[3 * j + 1] - mm[3 * j] : 0;
    f.vbits = range == 0 ? 0 : 64 - __builtin_clzll(range);
    f.has_null_bit = mm[3 * j + 2] ? 1 : 0;
    f.shift = bits;
    bits += f.vbits + f.has_null_bit;
  }
  if (bits > 64)
    return set_error(ctx, GHB_ERR_UNSUPPORTED, "sort keys need %d bits after range packing (max 64)", bits);
  const int npasses = (bits + kDigitBits - 1) / kDigitBits;

  // a BYTEMAP payload's NULL flags do not travel with its value: carry the row
  bool carry_rowid = out_rowid != nullptr || npayload > 1 ||
                     (npayload == 1 && payload[0].null_mode == GHB_NULLS_BYTEMAP);
  pp.carry_rowid = carry_rowid ? 1 : 0;
  if (!carry_rowid && npayload == 1) pp.pay_src = payload[0];
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

  std::vector<int> run_passes;
  std::vector<uint32_t> hist((size_t)kMaxPasses * kBins, 0);
  if (npasses > 0) {
    HistParams hp;
    hp.L = L;
    hp.n = n;
    hp.npasses = npasses;
    hp.hist = d_hist;
    sort_hist_kernel<<<std::min(grid, ctx->num_sms * 4), 256, 0, stream>>>(hp);
    GHB_LAUNCH_CHECK(ctx);
    GHB_CUDA_TRY(ctx, cudaMemcpyAsync(hist.data(), d_hist, (size_t)npasses * kBins * 4,
                                      cudaMemcpyDeviceToHost, stream));
    GHB_CUDA_TRY(ctx, cudaStreamSynchronize(stream));
    for (int q = 0; q < npasses; q++) {
      bool trivial = false;
      for (int b = 0; b < kBins; b++)
        if (hist[(size_t)q * kBins + b] == (uint32_t)n) trivial = true;
      if (!trivial) run_passes.push_back(q);
    }
  }
  if (run_passes.empty()) {
    sort_copy_kernel<<<grid, 256, 0, stream>>>(pp);
    GHB_LAUNCH_CHECK(ctx);
    return GHB_OK;
  }
  uint64_t *kb[2] = {nullptr, nullptr}, *vb[2] = {nullptr, nullptr};
  uint32_t* status = nullptr;
  size_t nb = (size_t)n * 8;
  if (run_passes.size() > 1) {
    for (int i = 0; i < 2; i++) {
      if ((st = scratch_alloc(ctx, nb, (void**)&kb[i], stream))) return st;
      if ((st = scratch_alloc(ctx, nb, (void**)&vb[i], stream))) return st;
    }
  }
  size_t status_bytes = (size_t)run_passes.size() * pp.ntiles * kBins * 4;
  if ((st = scratch_alloc(ctx, status_bytes, (void**)&status, stream))) return st;
  GHB_CUDA_TRY(ctx, cudaMemsetAsync(status, 0, status_bytes, stream));
  const size_t dyn = 2 * (size_t)kSortTile * sizeof(uint64_t);
  GHB_CUDA_TRY(ctx, cudaFuncSetAttribute(sort_pass_kernel<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn));
  GHB_CUDA_TRY(ctx, cudaFuncSetAttribute(sort_pass_kernel<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn));
  GHB_CUDA_TRY(ctx, cudaFuncSetAttribute(sort_pass_kernel<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn));
  GHB_CUDA_TRY(ctx, cudaFuncSetAttribute(sort_pass_kernel<false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn));
  int per_sm = 0;
  GHB_CUDA_TRY(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sort_pass_kernel<false, false>,
                                                                 kSortThreads, dyn));
  int pgrid = (int)std::min<int64_t>(pp.ntiles, (int64_t)ctx->num_sms * std::max(1, per_sm));
  for (size_t i = 0; i < run_passes.size(); i++) {
    int q = run_passes[i];
    bool first = i == 0, last = i + 1 == run_passes.size();
    pp.shift = q * kDigitBits;
    uint32_t acc = 0;
    for (int b = 0; b < kBins; b++) {
      pp.digit_base[b] = acc;
      acc += hist[(size_t)q * kBins + b];
    }
    pp.keys_in = kb[(i + 1) & 1];
    pp.vals_in = vb[(i + 1) & 1];
    pp.keys_out = kb[i & 1];
    pp.vals_out = vb[i & 1];
    pp.status = status + i * (size_t)pp.ntiles * kBins;
    if (first && last) sort_pass_kernel<true, true><<<pgrid, kSortThreads, dyn, stream>>>(pp);
    else if (first) sort_pass_kernel<true, false><<<pgrid, kSortThreads, dyn, stream>>>(pp);
    else if (last) sort_pass_kernel<false, true><<<pgrid, kSortThreads, dyn, stream>>>(pp);
    else sort_pass_kernel<false, false><<<pgrid, kSortThreads, dyn, stream>>>(pp);
    GHB_LAUNCH_CHECK(ctx);
  }
  return GHB_OK;
}

}  // namespace ghb

using namespace ghb;

extern "C" int32_t ghb_sort(ghb_ctx* ctx, const ghb_column* keys, const int32_t* orders,
                            const int32_t* null_orders, int32_t nkeys, const ghb_column* payload,
                            int32_t npayload, ghb_out_column* out_keys, ghb_out_column* out_payload,
                            int32_t* out_rowid, const ghb_sort_cfg* cfg, void* stream) {
  if (!ctx) return GHB_ERR_INVALID;
  scratch_reset(ctx);
  int64_t n = keys && nkeys > 0 ? keys[0].n : 0;
  int32_t st = scratch_reserve(ctx, sort_scratch_bytes(n), (cudaStream_t)stream);
  if (st) return st;
  return sort_impl(ctx, keys, orders, null_orders, nkeys, payload, npayload, out_keys, out_payload,
                   out_rowid, cfg, (cudaStream_t)stream);
}
