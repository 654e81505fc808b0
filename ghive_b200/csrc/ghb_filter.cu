// ghb_filter.cu — filter with order-preserving stream compaction (F1).
//
// Replaces FilterPredicate::process (gpu_impl/src/Operator/FilterPredicate.cu:
// 434-571: one int32 bitmap per predicate leaf, one thrust::transform per
// AND/OR node) and FilterOperator::clean_data (gpu_impl/src/Operator/
// FilterOperator.cu:36-93: thrust::reduce + thrust::copy_if of row indices,
// D2H of the indices, then a host gather over every column, in place).
//
// One kernel: each CTA claims tiles of rows in launch order, evaluates the
// whole predicate tree in registers, turns the per-row results into warp
// ballots, scans the popcounts across the CTA, gets the tile's global output
// offset by decoupled look-back over earlier tiles, and copies the projected
// columns of the selected rows to their final positions.  No bitmap or index
// list is materialised; the output keeps input order (Hive's selected[]).
#include <algorithm>

#include "ghb_ctx.hpp"
#include "ghb_log.hpp"

namespace ghb {

constexpr int kFiltThreads = 256;
constexpr int kFiltItems = 8;   // rows per thread per tile
constexpr int kFiltTile = kFiltThreads * kFiltItems;
constexpr int kMaxProj = kMaxCols;

struct FilterParams {
  ColSet cols;
  PredProg pred;
  int32_t nproj;
  int32_t proj[kMaxProj];
  ghb_out_column out[kMaxProj];
  int64_t n;
  int64_t ntiles;
  int64_t cap;
  int64_t* d_out_rows;
  uint64_t* lb;
  uint32_t epoch;
  unsigned long long* counters;  // [0] next tile, [1] finished CTAs
  int32_t* status;
  int32_t spin_limit;            // look-back polls before GHB_ERR_TIMEOUT
};

__device__ __forceinline__ void copy_value(const ghb_column& c, const ghb_out_column& o, int64_t row,
                                           int64_t pos) {
  if (c.type == GHB_STRING) {
    // a STRING output row is the input row's [start,end) into the same bytes
    const int2 ix = __ldg((const int2*)c.aux + row);
    ((int2*)o.data)[pos] = ix;
    if (o.is_null) o.is_null[pos] = ix.x < 0 ? 1 : 0;
    return;
  }
  if (c.type == GHB_INT) ((int32_t*)o.data)[pos] = __ldg((const int32_t*)c.data + row);
  else ((long long*)o.data)[pos] = __ldg((const long long*)c.data + row);
  if (o.is_null) {
    bool null = false;
    if (c.null_mode != GHB_NULLS_NONE) null = raw_is_null(c, ld_raw(c, row), row);
    o.is_null[pos] = null ? 1 : 0;
  }
}

// The parameters stay in the constant bank (__grid_constant__): the string
// leaves' out-of-line compare takes references into them, which would
// otherwise copy the whole parameter block to every thread's stack.
__global__ void __launch_bounds__(kFiltThreads) filter_kernel(const __grid_constant__ FilterParams p) {
  __shared__ int64_t s_tile;
  __shared__ uint32_t s_warp_cnt[kFiltItems][kFiltThreads / 32];
  __shared__ uint32_t s_warp_off[kFiltItems][kFiltThreads / 32];
  __shared__ uint64_t s_tile_excl;
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const unsigned lt_mask = (1u << lane) - 1u;

  while (true) {
    claim_tile(&p.counters[0], &s_tile);
    const int64_t tile = s_tile;
    if (tile >= p.ntiles) break;
    const int64_t base = tile * kFiltTile;
    // the projected columns of a whole tile start toward L2 while the
    // predicate is evaluated and the tile's offset looked up, so the copies
    // after the look-back read L2
    if (threadIdx.x < p.nproj && base + kFiltTile <= p.n) {
      const ghb_column& c = p.cols.c[p.proj[threadIdx.x]];
      const int w = c.type == GHB_INT ? 4 : 8;
      const void* src = c.type == GHB_STRING ? (const void*)((const int2*)c.aux + base)
                                             : (const void*)((const char*)c.data + base * w);
      if (((uintptr_t)src & 15) == 0) bulk_prefetch_l2(src, (uint32_t)(kFiltTile * w));
    }

    unsigned ballots[kFiltItems];
#pragma unroll
    for (int k = 0; k < kFiltItems; k++) {
      int64_t row = base + (int64_t)k * kFiltThreads + threadIdx.x;
      bool pass = row < p.n && eval_pred(p.pred, p.cols, row);
      ballots[k] = __ballot_sync(0xffffffffu, pass);
    }
    if (lane == 0) {
#pragma unroll
      for (int k = 0; k < kFiltItems; k++) s_warp_cnt[k][warp] = __popc(ballots[k]);
    }
    __syncthreads();
    // exclusive scan over (item, warp) in row order, by warp 0
    if (warp == 0) {
      // each lane scans kPer consecutive (item, warp) slots
      constexpr int kSlots = kFiltItems * (kFiltThreads / 32);
      constexpr int kPer = kSlots / 32;
      static_assert(kSlots % 32 == 0, "whole slots per lane");
      uint32_t v[kPer];
      uint32_t mine = 0;
#pragma unroll
      for (int q = 0; q < kPer; q++) {
        v[q] = ((uint32_t*)s_warp_cnt)[kPer * lane + q];
        mine += v[q];
      }
      uint32_t incl = mine;
      for (int o = 1; o < 32; o <<= 1) {
        uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
      }
      uint32_t run = incl - mine;
#pragma unroll
      for (int q = 0; q < kPer; q++) {
        ((uint32_t*)s_warp_off)[kPer * lane + q] = run;
        run += v[q];
      }
      uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
      uint64_t ex = lookback_exclusive(p.lb, p.epoch, tile, total, p.status, p.spin_limit);
      if (lane == 0) {
        s_tile_excl = ex;
        if (tile == p.ntiles - 1) *p.d_out_rows = (int64_t)(ex + total);
      }
    }
    __syncthreads();
    const uint64_t tile_excl = s_tile_excl;
#pragma unroll
    for (int k = 0; k < kFiltItems; k++) {
      if (!((ballots[k] >> lane) & 1u)) continue;
      int64_t row = base + (int64_t)k * kFiltThreads + threadIdx.x;
      int64_t pos = (int64_t)(tile_excl + s_warp_off[k][warp] + __popc(ballots[k] & lt_mask));
      if (pos >= p.cap) {
        raise_status(p.status, kDevCapacity);
        continue;
      }
      for (int j = 0; j < p.nproj; j++) copy_value(p.cols.c[p.proj[j]], p.out[j], row, pos);
    }
    __syncthreads();
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
  p.ntiles = (n + kFiltTile - 1) / kFiltTile;
  p.cap = out_capacity;
  p.d_out_rows = d_out_rows;
  p.status = ctx->d_status;
  p.counters = ctx->d_counters;
  p.spin_limit = ctx->spin_limit;
  if (p.ntiles == 0) {
    GHB_CUDA_TRY(ctx, cudaMemsetAsync(d_out_rows, 0, sizeof(int64_t), stream));
    return GHB_OK;
  }
  st = lookback_prepare(ctx, p.ntiles, &p.epoch, stream);
  if (st) return st;
  p.lb = ctx->lb_status;
  int per_sm = 0;
  GHB_CUDA_TRY(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, filter_kernel, kFiltThreads, 0));
  int grid = (int)std::min<int64_t>(p.ntiles, (int64_t)ctx->num_sms * std::max(1, per_sm));
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
