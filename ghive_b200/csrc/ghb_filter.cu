// ghb_filter.cu — filter with order-preserving stream compaction (F1).
//
// Replaces FilterPredicate::process (gpu_impl/src/Operator/FilterPredicate.cu:
// 434-571: one int32 bitmap per predicate leaf, one thrust::transform per
// AND/OR node) and FilterOperator::clean_data (gpu_impl/src/Operator/
// FilterOperator.cu:36-93: thrust::reduce + thrust::copy_if of row indices,
// D2H of the indices, then a host gather over every column, in place).
//
// One kernel: each CTA claims ranges of rows (whole tiles, about one range
// per resident CTA) in launch order, evaluates the whole predicate tree in
// registers, keeps the per-row results as warp ballots in shared memory,
// scans their popcounts across the range, gets the range's global output
// offset by decoupled look-back over earlier ranges, and copies the projected
// columns of the selected rows to their final positions.  No bitmap or index
// list goes to global memory; the output keeps input order (Hive's
// selected[]).
#include <algorithm>

#include "ghb_ctx.hpp"
#include "ghb_log.hpp"

namespace ghb {

constexpr int kFiltThreads = 256;
constexpr int kFiltItems = 8;   // rows per thread per tile
constexpr int kFiltTile = kFiltThreads * kFiltItems;
constexpr int kFiltWarps = kFiltThreads / 32;
constexpr int kFiltWords = kFiltItems * kFiltWarps;   // ballot words of one tile
constexpr int kFiltMaxTiles = 16;                     // tiles of one claimed range
constexpr int kMaxProj = kMaxCols;

struct FilterParams {
  ColSet cols;
  PredProg pred;
  int32_t nproj;
  int32_t proj[kMaxProj];
  ghb_out_column out[kMaxProj];
  int64_t n;
  int64_t range_rows;            // rows of a claimed range: whole tiles, at most kFiltMaxTiles
  int64_t nranges;
  int64_t cap;
  int64_t* d_out_rows;
  uint64_t* lb;
  uint32_t epoch;
  unsigned long long* counters;  // [0] next range, [1] finished CTAs
  int32_t* status;
  int32_t spin_limit;            // look-back polls before GHB_ERR_TIMEOUT
};

// Copies column c's value of the selected rows row0 + k * kFiltThreads (bit
// `lane` of word b[k]) to output row pos[k]: every load of the tile is issued
// before its stores.
__device__ __forceinline__ void copy_rows(const ghb_column& c, const ghb_out_column& o, int64_t row0,
                                          const bool (&live)[kFiltItems], const int64_t (&pos)[kFiltItems]) {
  if (c.type == GHB_INT) {
    int32_t v[kFiltItems];
#pragma unroll
    for (int k = 0; k < kFiltItems; k++)
      if (live[k]) v[k] = __ldcs((const int*)c.data + row0 + k * kFiltThreads);
#pragma unroll
    for (int k = 0; k < kFiltItems; k++)
      if (live[k]) ((int32_t*)o.data)[pos[k]] = v[k];
    if (o.is_null) {
#pragma unroll
      for (int k = 0; k < kFiltItems; k++)
        if (live[k]) o.is_null[pos[k]] = raw_is_null(c, (int64_t)v[k], row0 + k * kFiltThreads) ? 1 : 0;
    }
    return;
  }
  // LONG, DOUBLE bits, or a STRING row's [start,end) pair into the same bytes
  const long long* src = c.type == GHB_STRING ? (const long long*)c.aux : (const long long*)c.data;
  long long v[kFiltItems];
#pragma unroll
  for (int k = 0; k < kFiltItems; k++)
    if (live[k]) v[k] = __ldcs(src + row0 + k * kFiltThreads);
#pragma unroll
  for (int k = 0; k < kFiltItems; k++)
    if (live[k]) ((long long*)o.data)[pos[k]] = v[k];
  if (o.is_null) {
#pragma unroll
    for (int k = 0; k < kFiltItems; k++) {
      if (!live[k]) continue;
      const bool null = c.type == GHB_STRING ? (int32_t)(v[k] & 0xffffffff) < 0
                                             : raw_is_null(c, (int64_t)v[k], row0 + k * kFiltThreads);
      o.is_null[pos[k]] = null ? 1 : 0;
    }
  }
}

// Each CTA claims ranges of rows in launch order.  Per range: the predicate
// tree of every row, kept as warp ballots in shared memory; one scan of the
// ballots' counts; the range's global output offset by decoupled look-back
// over earlier ranges (one per range, so a range's writes do not wait per
// tile); then the projected columns of the selected rows, every load of a
// tile's column issued before its stores.  The parameters stay in the
// constant bank (__grid_constant__): the string leaves' out-of-line compare
// takes references into them, which would otherwise copy the whole parameter
// block to every thread's stack.
__global__ void __launch_bounds__(kFiltThreads) filter_kernel(const __grid_constant__ FilterParams p) {
  constexpr int kWords = kFiltMaxTiles * kFiltWords;
  constexpr int kPer = kWords / kFiltThreads;
  static_assert(kWords % kFiltThreads == 0, "whole ballot words per thread");
  __shared__ int64_t s_range;
  __shared__ uint32_t s_mask[kWords];   // ballot words in row order: (tile, item, warp)
  __shared__ uint32_t s_off[kWords];    // each word's first output row within the range
  __shared__ uint32_t s_wsum[kFiltWarps];
  __shared__ uint64_t s_excl;
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const unsigned lt_mask = (1u << lane) - 1u;
  const bool leaf1 = p.pred.n_nodes == 1 && p.pred.nodes[0].col2 < 0 &&
                     p.cols.c[p.pred.nodes[0].col].type != GHB_STRING;

  while (true) {
    claim_tile(&p.counters[0], &s_range);
    const int64_t r = s_range;
    if (r >= p.nranges) break;
    const int64_t base = r * p.range_rows;
    const int64_t end = min(p.n, base + p.range_rows);
    const int tiles = (int)((end - base + kFiltTile - 1) / kFiltTile);
    for (int t = 0; t < tiles; t++) {
      const int64_t row0 = base + (int64_t)t * kFiltTile + threadIdx.x;
      unsigned ballots[kFiltItems];
      if (leaf1) {
        // one leaf on a fixed-width column: the tile's values are loaded
        // before any is compared
        const ghb_pred_node& nd = p.pred.nodes[0];
        const ghb_column& c = p.cols.c[nd.col];
        int64_t x[kFiltItems];
#pragma unroll
        for (int k = 0; k < kFiltItems; k++) {
          const int64_t row = row0 + k * kFiltThreads;
          x[k] = row < end ? ld_raw(c, row) : 0;
        }
#pragma unroll
        for (int k = 0; k < kFiltItems; k++) {
          const int64_t row = row0 + k * kFiltThreads;
          ballots[k] = __ballot_sync(0xffffffffu, row < end && leaf_on_raw(nd, c, x[k], row));
        }
      } else {
#pragma unroll
        for (int k = 0; k < kFiltItems; k++) {
          const int64_t row = row0 + k * kFiltThreads;
          ballots[k] = __ballot_sync(0xffffffffu, row < end && eval_pred(p.pred, p.cols, row));
        }
      }
      if (lane == 0) {
#pragma unroll
        for (int k = 0; k < kFiltItems; k++) s_mask[(t * kFiltItems + k) * kFiltWarps + warp] = ballots[k];
      }
    }
    __syncthreads();
    // exclusive scan of the words' counts in row order: kPer consecutive
    // words per thread, then across the warps
    const int nwords = tiles * kFiltWords;
    uint32_t cnt[kPer];
    uint32_t mine = 0;
#pragma unroll
    for (int q = 0; q < kPer; q++) {
      const int w = threadIdx.x * kPer + q;
      cnt[q] = w < nwords ? __popc(s_mask[w]) : 0;
      mine += cnt[q];
    }
    uint32_t incl = mine;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += v;
    }
    if (lane == 31) s_wsum[warp] = incl;
    __syncthreads();
    if (warp == 0) {
      const uint32_t ws = lane < kFiltWarps ? s_wsum[lane] : 0;
      uint32_t wi = ws;
#pragma unroll
      for (int o = 1; o < kFiltWarps; o <<= 1) {
        const uint32_t v = __shfl_up_sync(0xffffffffu, wi, o);
        if (lane >= o) wi += v;
      }
      const uint32_t total = __shfl_sync(0xffffffffu, wi, kFiltWarps - 1);
      const uint64_t ex = lookback_exclusive(p.lb, p.epoch, r, total, p.status, p.spin_limit);
      if (lane < kFiltWarps) s_wsum[lane] = wi - ws;
      if (lane == 0) {
        s_excl = ex;
        if (r == p.nranges - 1) *p.d_out_rows = (int64_t)(ex + total);
        if ((int64_t)(ex + total) > p.cap) raise_status(p.status, kDevCapacity);
      }
    }
    __syncthreads();
    uint32_t run = s_wsum[warp] + incl - mine;
#pragma unroll
    for (int q = 0; q < kPer; q++) {
      const int w = threadIdx.x * kPer + q;
      if (w < nwords) s_off[w] = run;
      run += cnt[q];
    }
    __syncthreads();
    const uint64_t rex = s_excl;
    if (p.nproj > 0) {
      for (int t = 0; t < tiles; t++) {
        bool live[kFiltItems];
        int64_t pos[kFiltItems];
#pragma unroll
        for (int k = 0; k < kFiltItems; k++) {
          const int w = (t * kFiltItems + k) * kFiltWarps + warp;
          const unsigned b = s_mask[w];
          pos[k] = (int64_t)(rex + s_off[w] + __popc(b & lt_mask));
          live[k] = ((b >> lane) & 1u) && pos[k] < p.cap;
        }
        const int64_t row0 = base + (int64_t)t * kFiltTile + threadIdx.x;
        for (int j = 0; j < p.nproj; j++) copy_rows(p.cols.c[p.proj[j]], p.out[j], row0, live, pos);
      }
    }
    __syncthreads();   // the next range reuses the ballots and offsets
  }
  claim_finish(p.counters);
}

int32_t filter_impl(ghb_ctx* ctx, const ghb_predicate* pred, const ghb_column* cols, int32_t ncols,
                    const int32_t* proj, int32_t nproj, ghb_out_column* out, int64_t out_capacity,
                    int64_t* d_out_rows, cudaStream_t stream) {
  int64_t n = 0;
  int32_t st = validate_columns(ctx, cols, ncols, &n, true);
  if (st) return st;
  if (nproj < 0 || nproj > kMaxProj) return set_error(ctx, GHB_ERR_INVALID, "nproj=%d", nproj);
  if (nproj > 0 && (!proj || !out)) return set_error(ctx, GHB_ERR_INVALID, "proj/out is NULL");
  if (!d_out_rows) return set_error(ctx, GHB_ERR_INVALID, "d_out_rows is NULL");
  if (out_capacity < 0) return set_error(ctx, GHB_ERR_INVALID, "negative out_capacity");
  FilterParams p;
  std::memset(&p, 0, sizeof(p));
  st = build_pred_prog(ctx, pred, cols, ncols, &p.pred);
  if (st) return st;
  for (int j = 0; j < nproj; j++) {
    if (proj[j] < 0 || proj[j] >= ncols)
      return set_error(ctx, GHB_ERR_INVALID, "projection %d: column %d out of range", j, proj[j]);
    if (out[j].type != cols[proj[j]].type)
      return set_error(ctx, GHB_ERR_INVALID, "projection %d: output type %d differs from input %d", j,
                       out[j].type, cols[proj[j]].type);
    if (!out[j].data && out_capacity > 0)
      return set_error(ctx, GHB_ERR_INVALID, "projection %d: output data is NULL", j);
    p.proj[j] = proj[j];
    p.out[j] = out[j];
  }
  for (int i = 0; i < ncols; i++) p.cols.c[i] = cols[i];
  p.cols.n = ncols;
  p.nproj = nproj;
  p.n = n;
  p.cap = out_capacity;
  p.d_out_rows = d_out_rows;
  p.status = ctx->d_status;
  p.counters = ctx->d_counters;
  p.spin_limit = ctx->spin_limit;
  if (n == 0) {
    GHB_CUDA_TRY(ctx, cudaMemsetAsync(d_out_rows, 0, sizeof(int64_t), stream));
    return GHB_OK;
  }
  int per_sm = 0;
  GHB_CUDA_TRY(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, filter_kernel, kFiltThreads, 0));
  const int64_t slots = (int64_t)ctx->num_sms * std::max(1, per_sm);
  // one range per resident CTA where the rows allow, in whole tiles
  const int64_t ntiles = (n + kFiltTile - 1) / kFiltTile;
  const int64_t per = std::min<int64_t>(kFiltMaxTiles, std::max<int64_t>(1, (ntiles + slots - 1) / slots));
  p.range_rows = per * kFiltTile;
  p.nranges = (ntiles + per - 1) / per;
  st = lookback_prepare(ctx, p.nranges, &p.epoch, stream);
  if (st) return st;
  p.lb = ctx->lb_status;
  int grid = (int)std::min<int64_t>(p.nranges, slots);
  filter_kernel<<<grid, kFiltThreads, 0, stream>>>(p);
  GHB_LAUNCH_CHECK(ctx);
  return GHB_OK;
}

}  // namespace ghb

using namespace ghb;

extern "C" int32_t ghb_filter(ghb_ctx* ctx, const ghb_predicate* pred, const ghb_column* cols,
                              int32_t ncols, const int32_t* proj, int32_t nproj, ghb_out_column* out,
                              int64_t out_capacity, int64_t* d_out_rows, void* stream) {
  if (!ctx) return GHB_ERR_INVALID;
  CallScope cs(ctx, "filter", (cudaStream_t)stream);
  cs.rows(ncols > 0 && cols ? cols[0].n : 0);
  cs.bytes(cols_bytes(cols, ncols));
  scratch_reset(ctx);
  return cs.done(filter_impl(ctx, pred, cols, ncols, proj, nproj, out, out_capacity, d_out_rows,
                             (cudaStream_t)stream));
}
