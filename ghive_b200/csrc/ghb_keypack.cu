// ghb_keypack.cu — GROUP BY over several key columns, by packing the keys of
// a row into one 64-bit key.
//
// GHive groups by any number of key columns of mixed types: it sorts row
// indices with a comparator over all `key_num` key columns
// (gpu_impl/src/Operator/GroupByPredicate.cu:24-105, comparator
// gpu_impl/inc/Operator/GroupByPredicate.hpp:22-101) and reduces runs of
// equal keys.  Here the keys of a row become one int64 value, and the
// single-key hash group-by (ghb_groupby.cu) runs on that value:
//
//   1. one read of the key columns: per key the min/max of its order image
//      (BinarySortable order: sign-flipped integers, IEEE total order for
//      doubles) and whether it holds NULLs;
//   2. plan (host): key j becomes a field [null flag][image - min] of just the
//      width its range needs; the fields are concatenated into at most 63
//      bits (the packed value is a non-negative int64).  Equal key tuples
//      pack to equal values and different ones to different values, so the
//      groups are exactly Hive's (a NULL key component is its own value);
//   3. one pass writes the packed keys as an int64 column;
//   4. after the group-by, the packed key of each output group is unpacked
//      into the caller's key output columns (NULL components as NULL).
//
// Key tuples that need more than 63 bits (a DOUBLE key of both signs, two
// full-range LONG keys) are grouped instead by the row of each tuple's first
// occurrence, found through a lock-free device hash table of the tuples.
#include <algorithm>

#include "ghb_ctx.hpp"

namespace ghb {

__device__ __forceinline__ uint64_t kp_image(const ghb_column& c, int64_t raw) {
  return c.type == GHB_DOUBLE ? flip_f64_bits((uint64_t)raw) : flip_i64(raw);
}

struct KpMinMaxParams {
  int32_t nkeys;
  ghb_column col[kMaxPackKeys];
  int64_t n;
  unsigned long long* out;   // per key: [0] min image, [1] max image, [2] any NULL
};

__global__ void __launch_bounds__(256) keypack_minmax_kernel(KpMinMaxParams p) {
  __shared__ unsigned long long s_red[3][8];
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int warp = threadIdx.x >> 5;
  for (int j = 0; j < p.nkeys; j++) {
    const ghb_column c = p.col[j];
    unsigned long long mn = ~0ull, mx = 0, anynull = 0;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < p.n; r += stride) {
      const int64_t raw = ld_raw_cs(c, r);
      if (c.null_mode != GHB_NULLS_NONE && raw_is_null(c, raw, r)) {
        anynull = 1;
        continue;
      }
      const unsigned long long img = kp_image(c, raw);
      mn = min(mn, img);
      mx = max(mx, img);
    }
    for (int o = 16; o > 0; o >>= 1) {
      mn = min(mn, __shfl_down_sync(0xffffffffu, mn, o));
      mx = max(mx, __shfl_down_sync(0xffffffffu, mx, o));
      anynull |= __shfl_down_sync(0xffffffffu, anynull, o);
    }
    if ((threadIdx.x & 31) == 0) {
      s_red[0][warp] = mn;
      s_red[1][warp] = mx;
      s_red[2][warp] = anynull;
    }
    __syncthreads();
    if (threadIdx.x == 0) {   // one set of atomics per CTA
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

__global__ void __launch_bounds__(256) keypack_pack_kernel(KeyPackPlan p, int64_t n, int64_t* out) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n;
       r += (int64_t)gridDim.x * blockDim.x) {
    uint64_t v = 0;
#pragma unroll
    for (int j = 0; j < kMaxPackKeys; j++) {
      if (j >= p.nkeys) break;
      const ghb_column& c = p.col[j];
      const int64_t raw = ld_raw_cs(c, r);
      const bool null = c.null_mode != GHB_NULLS_NONE && raw_is_null(c, raw, r);
      if (p.fshift[j] >= 0 && !null) v |= 1ull << p.fshift[j];
      if (!null && p.vbits[j] > 0) v |= (kp_image(c, raw) - p.umin[j]) << p.vshift[j];
    }
    __stcs((unsigned long long*)out + r, (unsigned long long)v);
  }
}

// Unpacks the packed key of each of the first min(*d_groups, cap) output
// rows into the key output columns.
__global__ void __launch_bounds__(256) keypack_unpack_kernel(KeyPackPlan p, const int64_t* packed,
                                                              const int64_t* d_groups, int64_t cap,
                                                              KeyOuts outs) {
  const int64_t g = min(*d_groups, cap);
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < g;
       r += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t v = (uint64_t)packed[r];
#pragma unroll
    for (int j = 0; j < kMaxPackKeys; j++) {
      if (j >= p.nkeys) break;
      const ghb_out_column& o = outs.o[j];
      const bool null = p.fshift[j] >= 0 && ((v >> p.fshift[j]) & 1ull) == 0;
      const int vb = p.vbits[j];
      const uint64_t field = vb == 0 ? 0 : (v >> p.vshift[j]) & ((1ull << vb) - 1);
      const uint64_t img = field + p.umin[j];
      if (p.str_aux[j]) {   // the row of the value's first occurrence -> its bytes
        const int2 ix = null ? make_int2(-1, -1) : p.str_aux[j][(int64_t)(img ^ 0x8000000000000000ull)];
        ((int2*)o.data)[r] = ix;
        if (o.is_null) o.is_null[r] = null ? 1 : 0;
        continue;
      }
      const int64_t raw = o.type == GHB_DOUBLE ? (int64_t)unflip_f64_bits(img)
                                               : (int64_t)(img ^ 0x8000000000000000ull);
      if (o.is_null) o.is_null[r] = null ? 1 : 0;
      switch (o.type) {
        case GHB_LONG: ((int64_t*)o.data)[r] = null ? INT64_MAX : raw; break;
        case GHB_INT: ((int32_t*)o.data)[r] = null ? INT32_MAX : (int32_t)raw; break;
        case GHB_DOUBLE: ((int64_t*)o.data)[r] = null ? 0x7ff8000000000000ll : raw; break;
      }
    }
  }
}

// FNV-1a, 64-bit (Fowler, Noll and Vo's published hash), then a 64-bit mixer.
__device__ __forceinline__ uint64_t string_hash(const uint8_t* b, int len) {
  uint64_t h = 1469598103934665603ull;
  for (int k = 0; k < len; k++) {
    h ^= b[k];
    h *= 1099511628211ull;
  }
  return mix64(h);
}

// Row of each row's value's first occurrence, through a lock-free table of
// (hash tag << 32 | row + 1) words: the first row of a value claims a slot by
// CAS; the bytes a slot stands for are that row's own, so a later row with
// the same tag compares bytes with it directly.
__global__ void __launch_bounds__(256) string_rep_kernel(ghb_column c, const int32_t* pass, int64_t* rep,
                                                          unsigned long long* table, int64_t mask,
                                                          int32_t* status) {
  const int2* aux = (const int2*)c.aux;
  const uint8_t* bytes = (const uint8_t*)c.data;
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < c.n;
       r += (int64_t)gridDim.x * blockDim.x) {
    const int2 ix = aux[r];
    if (ix.x < 0 || (pass && pass[r] == 0)) {
      rep[r] = INT64_MAX;
      continue;
    }
    const uint8_t* b = bytes + ix.x;
    const int len = ix.y - ix.x;
    const uint64_t h = string_hash(b, len);
    const uint32_t tag = (uint32_t)(h >> 32) | 1u;
    const unsigned long long mine = ((unsigned long long)tag << 32) | (unsigned long long)(r + 1);
    int64_t s = (int64_t)(h & (uint64_t)mask), found = -1;
    for (int64_t probe = 0; probe <= mask; probe++) {
      unsigned long long w = *(volatile unsigned long long*)&table[s];
      if (w == 0) {
        const unsigned long long old = atomicCAS(&table[s], 0ull, mine);
        if (old == 0) {
          found = r;
          break;
        }
        w = old;
      }
      if ((uint32_t)(w >> 32) == tag) {
        const int64_t o = (int64_t)(w & 0xffffffffull) - 1;
        const int2 io = aux[o];
        if (io.y - io.x == len && str_compare(bytes + io.x, len, b, len) == 0) {
          found = o;
          break;
        }
      }
      s = (s + 1) & mask;
    }
    if (found < 0) raise_status(status, kDevCapacity);   // more distinct values than slots
    rep[r] = found < 0 ? INT64_MAX : found;
  }
}

__global__ void __launch_bounds__(256) predicate_pass_kernel(const __grid_constant__ PredProg prog,
                                                              const __grid_constant__ ColSet cs, int64_t n,
                                                              int32_t* pass) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x)
    pass[r] = eval_pred(prog, cs, r) ? 1 : 0;
}

int32_t string_rep_rows(ghb_ctx* ctx, const ghb_column& c, const int32_t* pass, int64_t* rep,
                        unsigned long long* table, int64_t slots, cudaStream_t stream) {
  if (c.n >= (int64_t)UINT32_MAX - 1) return set_error(ctx, GHB_ERR_UNSUPPORTED, "STRING key of 2^32 rows");
  GHB_CUDA_TRY(ctx, cudaMemsetAsync(table, 0, (size_t)slots * 8, stream));
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((c.n + 255) / 256, (int64_t)ctx->num_sms * 8));
  string_rep_kernel<<<grid, 256, 0, stream>>>(c, pass, rep, table, slots - 1, ctx->d_status);
  GHB_LAUNCH_CHECK(ctx);
  return GHB_OK;
}

int32_t predicate_pass(ghb_ctx* ctx, const PredProg& prog, const ghb_column* cols, int32_t ncols, int64_t n,
                       int32_t* pass, cudaStream_t stream) {
  ColSet cs;
  std::memset(&cs, 0, sizeof(cs));
  for (int i = 0; i < ncols; i++) cs.c[i] = cols[i];
  cs.n = ncols;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)ctx->num_sms * 8));
  predicate_pass_kernel<<<grid, 256, 0, stream>>>(prog, cs, n, pass);
  GHB_LAUNCH_CHECK(ctx);
  return GHB_OK;
}

// Plans the packing of the key columns and writes the packed keys (n int64
// values) to `packed`.  Reads the keys' ranges back to the host (one
// stream synchronisation).
int32_t keypack_prepare(ghb_ctx* ctx, const ghb_column* cols, const int32_t* key_cols, int32_t nkeys,
                        int64_t n, int64_t* packed, KeyPackPlan* plan, cudaStream_t stream, bool* too_wide) {
  if (nkeys < 1 || nkeys > kMaxPackKeys)
    return set_error(ctx, GHB_ERR_UNSUPPORTED, "%d key columns: at most %d", nkeys, kMaxPackKeys);
  KeyPackPlan& P = *plan;
  std::memset(&P, 0, sizeof(P));
  P.nkeys = nkeys;
  KpMinMaxParams mp;
  std::memset(&mp, 0, sizeof(mp));
  mp.nkeys = nkeys;
  mp.n = n;
  for (int j = 0; j < nkeys; j++) {
    const ghb_column& c = cols[key_cols[j]];
    if (c.type == GHB_STRING)
      return set_error(ctx, GHB_ERR_UNSUPPORTED, "key %d: STRING keys are not on the device path", j);
    P.col[j] = c;
    mp.col[j] = c;
  }
  unsigned long long* d_mm = nullptr;
  int32_t st = scratch_alloc(ctx, 3 * 8 * kMaxPackKeys, (void**)&d_mm, stream);
  if (st) return st;
  unsigned long long init[3 * kMaxPackKeys];
  for (int j = 0; j < kMaxPackKeys; j++) {
    init[3 * j] = ~0ull;
    init[3 * j + 1] = 0;
    init[3 * j + 2] = 0;
  }
  GHB_CUDA_TRY(ctx, cudaMemcpyAsync(d_mm, init, sizeof(init), cudaMemcpyHostToDevice, stream));
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)ctx->num_sms * 8));
  mp.out = d_mm;
  keypack_minmax_kernel<<<grid, 256, 0, stream>>>(mp);
  GHB_LAUNCH_CHECK(ctx);
  unsigned long long mm[3 * kMaxPackKeys];
  GHB_CUDA_TRY(ctx, cudaMemcpyAsync(mm, d_mm, sizeof(mm), cudaMemcpyDeviceToHost, stream));
  GHB_CUDA_TRY(ctx, cudaStreamSynchronize(stream));
  int bits = 0;
  for (int j = 0; j < nkeys; j++) {
    const bool anyval = mm[3 * j] <= mm[3 * j + 1];
    P.umin[j] = anyval ? mm[3 * j] : 0;
    const uint64_t range = anyval ? mm[3 * j + 1] - mm[3 * j] : 0;
    P.vbits[j] = (int8_t)(range == 0 ? 0 : 64 - __builtin_clzll(range));
    P.vshift[j] = (int8_t)bits;
    bits += P.vbits[j];
    P.fshift[j] = -1;
    if (mm[3 * j + 2]) {
      P.fshift[j] = (int8_t)bits;
      bits++;
    }
    if (bits > 63) {   // the caller groups by first occurrences instead
      *too_wide = true;
      return GHB_OK;
    }
  }
  *too_wide = false;
  keypack_pack_kernel<<<grid, 256, 0, stream>>>(P, n, packed);
  GHB_LAUNCH_CHECK(ctx);
  return GHB_OK;
}

// ---- key tuples too wide to pack: the row of each tuple's first occurrence
struct TupleCols {
  int32_t nkeys;
  ghb_column col[kMaxPackKeys];
};

__device__ __forceinline__ uint64_t tuple_hash(const TupleCols& t, int64_t r) {
  uint64_t h = 0x9e3779b97f4a7c15ull;
#pragma unroll
  for (int j = 0; j < kMaxPackKeys; j++) {
    if (j >= t.nkeys) break;
    const int64_t raw = ld_raw(t.col[j], r);
    const bool null = t.col[j].null_mode != GHB_NULLS_NONE && raw_is_null(t.col[j], raw, r);
    h = mix64(h ^ (null ? 0x5bd1e9955bd1e995ull : (uint64_t)raw) ^ ((uint64_t)j << 56));
  }
  return h;
}

// Equal tuples: per key both NULL, or both non-NULL with the same raw value
// (the single-key group-by's rule: a double key by its bits).
__device__ __forceinline__ bool tuple_equal(const TupleCols& t, int64_t a, int64_t b) {
#pragma unroll
  for (int j = 0; j < kMaxPackKeys; j++) {
    if (j >= t.nkeys) break;
    const ghb_column& c = t.col[j];
    const int64_t x = ld_raw(c, a), y = ld_raw(c, b);
    const bool nx = c.null_mode != GHB_NULLS_NONE && raw_is_null(c, x, a);
    const bool ny = c.null_mode != GHB_NULLS_NONE && raw_is_null(c, y, b);
    if (nx != ny || (!nx && x != y)) return false;
  }
  return true;
}

// The same lock-free table of (hash tag << 32 | row + 1) words as the STRING
// keys': the first row of a tuple claims a slot, later rows compare tuples
// with the claiming row's own.
__global__ void __launch_bounds__(256) tuple_rep_kernel(TupleCols t, const int32_t* pass, int64_t n, int64_t* rep,
                                                         unsigned long long* table, int64_t mask, int32_t* status) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
    if (pass && pass[r] == 0) {
      rep[r] = INT64_MAX;
      continue;
    }
    const uint64_t h = tuple_hash(t, r);
    const uint32_t tag = (uint32_t)(h >> 32) | 1u;
    const unsigned long long mine = ((unsigned long long)tag << 32) | (unsigned long long)(r + 1);
    int64_t s = (int64_t)(h & (uint64_t)mask), found = -1;
    for (int64_t probe = 0; probe <= mask; probe++) {
      unsigned long long w = *(volatile unsigned long long*)&table[s];
      if (w == 0) {
        const unsigned long long old = atomicCAS(&table[s], 0ull, mine);
        if (old == 0) {
          found = r;
          break;
        }
        w = old;
      }
      if ((uint32_t)(w >> 32) == tag) {
        const int64_t o = (int64_t)(w & 0xffffffffull) - 1;
        if (tuple_equal(t, o, r)) {
          found = o;
          break;
        }
      }
      s = (s + 1) & mask;
    }
    if (found < 0) raise_status(status, kDevCapacity);   // more distinct tuples than slots
    rep[r] = found < 0 ? INT64_MAX : found;
  }
}

// Each output group's key tuple from its first row: the key columns' values
// (NULL as GHive's sentinel and in the NULL map), a STRING key's [start,end).
__global__ void __launch_bounds__(256) tuple_unpack_kernel(TupleCols t, KeyPackPlan p, const int64_t* rows,
                                                            const int64_t* d_groups, int64_t cap, KeyOuts outs) {
  const int64_t g = min(*d_groups, cap);
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < g; r += (int64_t)gridDim.x * blockDim.x) {
    const int64_t row = rows[r];
#pragma unroll
    for (int j = 0; j < kMaxPackKeys; j++) {
      if (j >= t.nkeys) break;
      const ghb_column& c = t.col[j];
      const ghb_out_column& o = outs.o[j];
      const int64_t raw = ld_raw(c, row);
      const bool null = c.null_mode != GHB_NULLS_NONE && raw_is_null(c, raw, row);
      if (o.is_null) o.is_null[r] = null ? 1 : 0;
      if (p.str_aux[j]) {
        ((int2*)o.data)[r] = null ? make_int2(-1, -1) : p.str_aux[j][raw];
        continue;
      }
      switch (o.type) {
        case GHB_LONG: ((int64_t*)o.data)[r] = null ? INT64_MAX : raw; break;
        case GHB_INT: ((int32_t*)o.data)[r] = null ? INT32_MAX : (int32_t)raw; break;
        case GHB_DOUBLE: ((int64_t*)o.data)[r] = null ? 0x7ff8000000000000ll : raw; break;
      }
    }
  }
}

int32_t tuple_rep_rows(ghb_ctx* ctx, const ghb_column* cols, const int32_t* key_cols, int32_t nkeys, int64_t n,
                       const int32_t* pass, int64_t* rep, unsigned long long* table, int64_t slots,
                       cudaStream_t stream) {
  if (n >= (int64_t)UINT32_MAX - 1) return set_error(ctx, GHB_ERR_UNSUPPORTED, "key tuples of 2^32 rows");
  TupleCols t;
  std::memset(&t, 0, sizeof(t));
  t.nkeys = nkeys;
  for (int j = 0; j < nkeys; j++) t.col[j] = cols[key_cols[j]];
  GHB_CUDA_TRY(ctx, cudaMemsetAsync(table, 0, (size_t)slots * 8, stream));
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)ctx->num_sms * 8));
  tuple_rep_kernel<<<grid, 256, 0, stream>>>(t, pass, n, rep, table, slots - 1, ctx->d_status);
  GHB_LAUNCH_CHECK(ctx);
  return GHB_OK;
}

int32_t tuple_unpack(ghb_ctx* ctx, const ghb_column* cols, const int32_t* key_cols, const KeyPackPlan& plan,
                     const int64_t* rows, const int64_t* d_groups, int64_t cap, const ghb_out_column* key_out,
                     cudaStream_t stream) {
  TupleCols t;
  std::memset(&t, 0, sizeof(t));
  t.nkeys = plan.nkeys;
  for (int j = 0; j < plan.nkeys; j++) t.col[j] = cols[key_cols[j]];
  KeyOuts outs;
  std::memset(&outs, 0, sizeof(outs));
  for (int j = 0; j < plan.nkeys; j++) outs.o[j] = key_out[j];
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((cap + 255) / 256, (int64_t)ctx->num_sms * 4));
  tuple_unpack_kernel<<<grid, 256, 0, stream>>>(t, plan, rows, d_groups, cap, outs);
  GHB_LAUNCH_CHECK(ctx);
  return GHB_OK;
}

// Packs the key tuples of a join's two sides with one plan (the ranges of
// both sides), so that equal tuples pack to equal values across the sides.
// A tuple with a NULL component never matches (SQL equality): its packed
// value is NULL (null_out = 1).
__global__ void __launch_bounds__(256) keypack_join_kernel(KeyPackPlan p, int64_t n, int64_t* out,
                                                           uint8_t* null_out) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n;
       r += (int64_t)gridDim.x * blockDim.x) {
    uint64_t v = 0;
    bool anynull = false;
#pragma unroll
    for (int j = 0; j < kMaxPackKeys; j++) {
      if (j >= p.nkeys) break;
      const ghb_column& c = p.col[j];
      const int64_t raw = ld_raw_cs(c, r);
      const bool null = c.null_mode != GHB_NULLS_NONE && raw_is_null(c, raw, r);
      anynull |= null;
      if (!null && p.vbits[j] > 0) v |= (kp_image(c, raw) - p.umin[j]) << p.vshift[j];
    }
    out[r] = anynull ? 0 : (int64_t)v;
    null_out[r] = anynull ? 1 : 0;
  }
}

int32_t keypack_join(ghb_ctx* ctx, const ghb_column* a, const ghb_column* b, int32_t nkeys, int64_t* a_packed,
                     uint8_t* a_null, int64_t* b_packed, uint8_t* b_null, cudaStream_t stream) {
  if (nkeys < 1 || nkeys > kMaxPackKeys)
    return set_error(ctx, GHB_ERR_UNSUPPORTED, "%d join key columns: at most %d", nkeys, kMaxPackKeys);
  for (int j = 0; j < nkeys; j++) {
    if (a[j].type == GHB_STRING || b[j].type == GHB_STRING)
      return set_error(ctx, GHB_ERR_UNSUPPORTED, "join key %d: STRING join keys are not on the device path", j);
    if (a[j].type != b[j].type)
      return set_error(ctx, GHB_ERR_INVALID, "join key %d: types %d and %d differ", j, a[j].type, b[j].type);
  }
  unsigned long long* d_mm = nullptr;
  int32_t st = scratch_alloc(ctx, 3 * 8 * kMaxPackKeys, (void**)&d_mm, stream);
  if (st) return st;
  unsigned long long init[3 * kMaxPackKeys];
  for (int j = 0; j < kMaxPackKeys; j++) {
    init[3 * j] = ~0ull;
    init[3 * j + 1] = 0;
    init[3 * j + 2] = 0;
  }
  GHB_CUDA_TRY(ctx, cudaMemcpyAsync(d_mm, init, sizeof(init), cudaMemcpyHostToDevice, stream));
  for (int side = 0; side < 2; side++) {
    const ghb_column* c = side ? b : a;
    KpMinMaxParams mp;
    std::memset(&mp, 0, sizeof(mp));
    mp.nkeys = nkeys;
    mp.n = c[0].n;
    for (int j = 0; j < nkeys; j++) mp.col[j] = c[j];
    mp.out = d_mm;
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((mp.n + 255) / 256, (int64_t)ctx->num_sms * 8));
    keypack_minmax_kernel<<<grid, 256, 0, stream>>>(mp);
    GHB_LAUNCH_CHECK(ctx);
  }
  unsigned long long mm[3 * kMaxPackKeys];
  GHB_CUDA_TRY(ctx, cudaMemcpyAsync(mm, d_mm, sizeof(mm), cudaMemcpyDeviceToHost, stream));
  GHB_CUDA_TRY(ctx, cudaStreamSynchronize(stream));
  KeyPackPlan P;
  std::memset(&P, 0, sizeof(P));
  P.nkeys = nkeys;
  int bits = 0;
  for (int j = 0; j < nkeys; j++) {
    const bool anyval = mm[3 * j] <= mm[3 * j + 1];
    P.umin[j] = anyval ? mm[3 * j] : 0;
    const uint64_t range = anyval ? mm[3 * j + 1] - mm[3 * j] : 0;
    P.vbits[j] = (int8_t)(range == 0 ? 0 : 64 - __builtin_clzll(range));
    P.vshift[j] = (int8_t)bits;
    P.fshift[j] = -1;
    bits += P.vbits[j];
    if (bits > 63)
      return set_error(ctx, GHB_ERR_UNSUPPORTED, "the %d join key columns' ranges need more than 63 bits", nkeys);
  }
  for (int side = 0; side < 2; side++) {
    const ghb_column* c = side ? b : a;
    for (int j = 0; j < nkeys; j++) P.col[j] = c[j];
    const int64_t n = c[0].n;
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)ctx->num_sms * 8));
    keypack_join_kernel<<<grid, 256, 0, stream>>>(P, n, side ? b_packed : a_packed, side ? b_null : a_null);
    GHB_LAUNCH_CHECK(ctx);
  }
  return GHB_OK;
}

int32_t keypack_unpack(ghb_ctx* ctx, const KeyPackPlan& plan, const int64_t* packed,
                       const int64_t* d_groups, int64_t cap, const ghb_out_column* key_out,
                       cudaStream_t stream) {
  KeyOuts outs;
  std::memset(&outs, 0, sizeof(outs));
  for (int j = 0; j < plan.nkeys; j++) outs.o[j] = key_out[j];
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((cap + 255) / 256, (int64_t)ctx->num_sms * 4));
  keypack_unpack_kernel<<<grid, 256, 0, stream>>>(plan, packed, d_groups, cap, outs);
  GHB_LAUNCH_CHECK(ctx);
  return GHB_OK;
}

}  // namespace ghb
