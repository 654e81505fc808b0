// ghb_groupby.cu — fused filter + hash group-by aggregation (G1 + G2), one
// operator call.
//
// Replaces GroupByPredicate::gpu_execute (gpu_impl/src/Operator/
// GroupByPredicate.cu:19-359), which sorted row indices with a comparison
// sort and then ran one H2D + reduce_by_key + D2H pass per aggregate
// (:506-720).  Here one pass over the rows evaluates the filter predicate and
// folds every aggregate of the row into a hash table:
//
//   G1  persistent CTAs; each streams tiles of the columns it needs into
//       shared memory with bulk copies (cp.async.bulk, completing on an
//       mbarrier, two stages so the next tile loads while this one is
//       folded), evaluates the predicate from shared memory, and folds each
//       passing row into a shared-memory open-addressing table (keys + one
//       64-bit accumulator per aggregate state); rows whose key does not fit
//       go straight to the global table; at the end the CTA merges its shared
//       table into the global one.
//   G2  finalize: walks the claimed-slot bitmap of the global table, emits
//       one output row per group (COUNT, SUM, AVG = sum/count, MIN, MAX with
//       Hive's NULL rules) and zeroes what it read, so the next call needs no
//       memset.
//
// The fold and finalize bodies live in ghb_groupby.cuh; the batched form of
// the operator (ghb_batch.cu) runs the same bodies over many instances.
#include <algorithm>

#include "ghb_groupby.cuh"
#include "ghb_log.hpp"

namespace ghb {

const void* jit_groupby_kernel(const GbParams& p, bool keyed, bool batch, int threads);
bool jit_enabled();

template <bool KEYED, bool NULLABLE>
__global__ void __launch_bounds__(kGbThreads) gb_fold_kernel(GbParams p) {
  fold_kernel_body<GenericFolder<KEYED, NULLABLE>>(p);
}

__global__ void __launch_bounds__(kFinThreads) gb_finalize_kernel(FinParams f) {
  __shared__ uint64_t rb[kFinThreads * (kMaxAcc + 1)];
  const int64_t nu = fin_units(f.C);
  for (int64_t u = blockIdx.x; u < nu; u += gridDim.x) finalize_unit(f, u, rb);
  if (blockIdx.x == 0 && threadIdx.x == 0) finalize_sides(f, rb);
  // the last CTA to finish publishes the group count and resets the counters
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(f.done, 1ull) == gridDim.x - 1) {
      __threadfence();
      *f.d_out_groups = (int64_t)atomicExch(f.growc, 0ull);
      *f.done = 0;
    }
  }
}

// ---------------------------------------------------------------- host
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
                         int32_t nkeys, AccPlan* ap_out, FinParams* fin) {
  if (naggs < 0 || naggs > kMaxAggs)
    return set_error(ctx, GHB_ERR_INVALID, "naggs=%d outside [0,%d]", naggs, kMaxAggs);
  AccPlan& ap = *ap_out;
  ap.n_acc = 0;
  add_acc(ap, A_CNT_STAR, -1);
  for (int i = 0; i < naggs; i++) {
    const ghb_agg_desc& d = aggs[i];
    OutAgg& o = fin->agg[i];
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
    fin->out[i] = oc;
  }
  fin->naggs = naggs;
  return GHB_OK;
}

int64_t next_pow2_i64(int64_t v) {
  int64_t p = 1;
  while (p < v) p <<= 1;
  return p;
}

static int log2_exact(int64_t v) {
  int l = 0;
  while ((1ll << l) < v) l++;
  return l;
}

int32_t gb_setup(ghb_ctx* ctx, const ghb_predicate* pred, const ghb_column* cols, int32_t ncols,
                 const int32_t* key_cols, int32_t nkeys, const ghb_agg_desc* aggs, int32_t naggs,
                 const ghb_out_column* out, int64_t out_capacity, int64_t* d_out_groups,
                 const GbSetup& su, GbParams* pp, FinParams* ff, size_t* table_bytes, size_t* smem) {
  int64_t n = 0;
  int32_t st = validate_columns(ctx, cols, ncols, &n, true);   // STRING columns only if unused
  if (st) return st;
  if (nkeys < 0 || nkeys > 1)
    return set_error(ctx, GHB_ERR_INVALID, "nkeys=%d: this kernel takes 0 or 1 key column", nkeys);
  if (nkeys == 1 && (!key_cols || key_cols[0] < 0 || key_cols[0] >= ncols))
    return set_error(ctx, GHB_ERR_INVALID, "key column out of range");
  if (naggs > 0 && !aggs) return set_error(ctx, GHB_ERR_INVALID, "aggs is NULL");
  if ((nkeys + naggs) > 0 && !out) return set_error(ctx, GHB_ERR_INVALID, "out is NULL");
  if (!d_out_groups) return set_error(ctx, GHB_ERR_INVALID, "d_out_groups is NULL");
  if (out_capacity < 1) return set_error(ctx, GHB_ERR_INVALID, "out_capacity must be >= 1");

  GbParams& p = *pp;
  FinParams& f = *ff;
  std::memset(&p, 0, sizeof(p));
  std::memset(&f, 0, sizeof(f));
  st = plan_aggs(ctx, cols, ncols, aggs, naggs, out, nkeys, &p.acc, &f);
  if (st) return st;
  st = build_pred_prog(ctx, pred, cols, ncols, &p.pred);
  if (st) return st;
  for (int i = 0; i < ncols; i++) p.cols.c[i] = cols[i];
  p.cols.n = ncols;
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
  for (int c = 0; c < ncols; c++)
    if (used[c] && cols[c].type == GHB_STRING)
      return set_error(ctx, GHB_ERR_UNSUPPORTED, "column %d: a STRING column as a key, predicate or "
                       "aggregate input of this kernel", c);

  int64_t max_groups = su.max_groups > 0 ? su.max_groups : out_capacity;
  if (nkeys == 0) max_groups = 1;
  max_groups = std::min<int64_t>(max_groups, std::max<int64_t>(n, 1));
  const double lf = su.load_factor > 0.f ? std::min<double>(su.load_factor, 0.9) : 0.5;
  int64_t C = next_pow2_i64(std::max<int64_t>((int64_t)((double)max_groups / lf) + 1, 64));
  if (C > (1ll << 30))
    return set_error(ctx, GHB_ERR_CAPACITY, "group-by table of %lld slots exceeds 2^30", (long long)C);
  int S;
  if (su.smem_slots < 0) S = 0;
  else if (su.smem_slots > 0) S = (int)std::min<int64_t>(kGbMaxSlots, next_pow2_i64(su.smem_slots));
  else S = (int)std::min<int64_t>(4096, next_pow2_i64(std::max<int64_t>(2 * max_groups, 64)));
  if (nkeys == 0) S = 64;
  const int threads = su.threads == 512 ? 512 : kGbThreads;
  int reserve = std::max(S, su.smem_table_slots);

  // Shared memory: [stages][control][table][warp staging].  The table keeps
  // (S + 2) slots of slot_words 32-bit words: the specialised folds' narrow
  // layout (ghb_gb_sig.cuh: u32 keys of an INT key column, u32 counts and
  // INT extremes, u32 pairs for integer sums) or one 64-bit word per key and
  // accumulator.
  size_t row_bytes = 0;
  for (int c = 0; c < ncols; c++)
    if (used[c]) row_bytes += type_width(cols[c].type) + (cols[c].null_mode == GHB_NULLS_BYTEMAP ? 1 : 0);
  const size_t smem_cap = 225 * 1024 - (size_t)std::max(0, su.extra_smem);
  int slot_words = 2 * (1 + p.acc.n_acc);
  if (su.narrow) {
    slot_words = (nkeys && cols[key_cols[0]].type == GHB_INT) ? 1 : 2;
    for (int a = 0; a < p.acc.n_acc; a++) {
      const int k = p.acc.kind[a];
      const bool int_col = p.acc.col[a] >= 0 && cols[p.acc.col[a]].type == GHB_INT;
      slot_words += (k == A_CNT_STAR || k == A_CNT_NN || ((k == A_MAX_O || k == A_MIN_O) && int_col)) ? 1 : 2;
    }
  }
  auto table_bytes_smem = [&](int s) {
    return (size_t)(s + 2) * 4 * slot_words + (size_t)(threads / 32) * 32 * 8 + kGbCtrlBytes;
  };
  auto stage_bytes_of = [&](int t) { return (row_bytes * (size_t)t + 127) & ~(size_t)127; };
  int tile_rows = su.tile_rows > 0 ? su.tile_rows : kGbRows * threads;
  if (tile_rows != threads && tile_rows != 2 * threads && tile_rows != 4 * threads)
    return set_error(ctx, GHB_ERR_INVALID, "tile_rows %d: must be the block size times 1, 2 or 4", tile_rows);
  if (su.nstages != 0 && (su.nstages < 2 || su.nstages > kGbMaxStages))
    return set_error(ctx, GHB_ERR_INVALID, "nstages %d outside [2,%d]", su.nstages, kGbMaxStages);
  if (su.smem_slots == 0)
    while (S > 64 && table_bytes_smem(S) + 2 * stage_bytes_of(threads) > smem_cap) S /= 2;
  reserve = std::max(S, su.smem_table_slots);
  if (table_bytes_smem(reserve) + 2 * stage_bytes_of(threads) > smem_cap)
    return set_error(ctx, GHB_ERR_UNSUPPORTED,
                     "rows of %zu bytes and %d shared slots do not fit a shared-memory tile", row_bytes,
                     reserve);
  // Tile: the most rows per thread whose two stages fit next to the table
  // (rows per thread are independent work for a thread, which hides the
  // latency of its shared-memory atomics); then stages while they fit, up to
  // about kInflight bytes of copies in flight while one stage is folded.
  const size_t room = smem_cap - table_bytes_smem(reserve);
  if (su.tile_rows == 0)
    while (tile_rows > threads && 2 * stage_bytes_of(tile_rows) > room) tile_rows /= 2;
  const size_t sb = stage_bytes_of(tile_rows);
  const size_t kInflight = 64 << 10;
  int ns = su.nstages ? su.nstages : 2;
  if (sb > 0 && !su.nstages)
    while (ns < kGbMaxStages && (size_t)(ns + 1) * sb <= room && (size_t)(ns - 1) * sb < kInflight) ns++;
  if ((size_t)ns * sb > room)
    return set_error(ctx, GHB_ERR_UNSUPPORTED,
                     "rows of %zu bytes and %d shared slots do not fit %d stages of %d rows", row_bytes, reserve,
                     ns, tile_rows);
  p.nstages = ns;
  p.table_words = (int32_t)((size_t)(reserve + 2) * slot_words / 2);
  p.smem_slots = S;
  p.warp_agg = su.warp_agg >= 0 ? su.warp_agg : ((nkeys == 0 || max_groups <= 64) ? 1 : 0);
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
  // words per global record: the key and the accumulators; a table too big
  // for L2 pads them to 2, 4, 8, 16 or 24 words so that the atomics of one
  // row touch one aligned 16/32/64-byte block of a DRAM line
  p.R = 1 + p.acc.n_acc;
  if (C > (1ll << 17)) p.R = p.R <= 2 ? 2 : p.R <= 4 ? 4 : p.R <= 8 ? 8 : p.R <= 16 ? 16 : 24;
  p.C = C;
  p.gshift = 64 - log2_exact(C);
  p.gprobe = (int32_t)std::min<int64_t>(C, 1 << 20);
  p.status = ctx->d_status;

  f.key_type = nkeys ? cols[key_cols[0]].type : -1;
  if (nkeys) f.key_out = out[0];
  f.cap = out_capacity;
  f.d_out_groups = d_out_groups;
  f.status = ctx->d_status;
  f.C = C;
  f.R = p.R;

  *table_bytes = gb_table_bytes(C, p.R);
  *smem = (size_t)p.nstages * p.stage_bytes + table_bytes_smem(reserve);
  return GHB_OK;
}

// Shared implementation; `fixed_table` (nullable) replaces the context's table.
int32_t filter_groupby_impl(ghb_ctx* ctx, const ghb_predicate* pred, const ghb_column* cols,
                            int32_t ncols, const int32_t* key_cols, int32_t nkeys,
                            const ghb_agg_desc* aggs, int32_t naggs, ghb_out_column* out,
                            int64_t out_capacity, int64_t* d_out_groups,
                            const ghb_groupby_cfg* cfg, cudaStream_t stream,
                            void* fixed_table, size_t fixed_table_bytes) {
  if (!ctx) return GHB_ERR_INVALID;
  // STRING keys or predicate leaves, or several keys: the fold itself reads
  // one fixed-width key and fixed-width predicate columns, so first
  //  - a predicate with STRING leaves (or any predicate beside STRING keys)
  //    becomes a pass flag column the fold tests for 1;
  //  - each STRING key becomes the row of its value's first occurrence;
  //  - several keys are packed into one int64 per row (unpacked afterwards).
  bool str_key = false, str_pred = false;
  if (cols && ncols > 0 && ncols <= kMaxCols) {
    for (int j = 0; key_cols && j < nkeys; j++)
      str_key |= key_cols[j] >= 0 && key_cols[j] < ncols && cols[key_cols[j]].type == GHB_STRING;
    for (int k = 0; pred && pred->nodes && k < pred->n_nodes && k < GHB_MAX_PRED_NODES; k++) {
      const ghb_pred_node& nd = pred->nodes[k];
      if (nd.mode != GHB_FILTER_AND && nd.mode != GHB_FILTER_OR && nd.col >= 0 && nd.col < ncols)
        str_pred |= cols[nd.col].type == GHB_STRING;
    }
  }
  if (nkeys > 1 || str_key || str_pred) {
    if (fixed_table)
      return set_error(ctx, GHB_ERR_UNSUPPORTED, "the allocation-free entry point takes one fixed-width key "
                       "and no STRING predicate");
    int64_t n = 0;
    int32_t st = validate_columns(ctx, cols, ncols, &n, true);
    if (st) return st;
    if (nkeys > 0 && !key_cols) return set_error(ctx, GHB_ERR_INVALID, "key_cols is NULL");
    if (!out) return set_error(ctx, GHB_ERR_INVALID, "out is NULL");
    if (nkeys > kMaxPackKeys)
      return set_error(ctx, GHB_ERR_UNSUPPORTED, "%d key columns: at most %d", nkeys, kMaxPackKeys);
    int nstr = 0;
    for (int j = 0; j < nkeys; j++) {
      if (key_cols[j] < 0 || key_cols[j] >= ncols)
        return set_error(ctx, GHB_ERR_INVALID, "key %d: column %d out of range", j, key_cols[j]);
      if (out[j].type != cols[key_cols[j]].type || !out[j].data)
        return set_error(ctx, GHB_ERR_INVALID, "key output %d: type %d (expected %d) or no data", j,
                         out[j].type, cols[key_cols[j]].type);
      nstr += cols[key_cols[j]].type == GHB_STRING;
    }
    for (int a = 0; a < naggs; a++)
      if (aggs && aggs[a].col >= 0 && aggs[a].col < ncols && cols[aggs[a].col].type == GHB_STRING)
        return set_error(ctx, GHB_ERR_UNSUPPORTED, "aggregate %d: STRING input", a);
    if (out_capacity < 1) return set_error(ctx, GHB_ERR_INVALID, "out_capacity must be >= 1");
    const bool use_pass = pred && pred->n_nodes > 0 && (str_pred || str_key);
    const bool packed_key = nkeys > 1 || str_key;
    if (ncols + (use_pass ? 1 : 0) + nstr + (packed_key ? 1 : 0) > kMaxCols)
      return set_error(ctx, GHB_ERR_UNSUPPORTED, "%d columns and the derived ones exceed %d", ncols, kMaxCols);
    const int64_t hint = std::max<int64_t>(1, std::min<int64_t>(n, cfg && cfg->max_groups > 0 ? cfg->max_groups
                                                                                            : out_capacity));
    const int64_t slots = next_pow2_i64(std::max<int64_t>(64, 2 * hint));
    if (ctx->scratch_used == 0) {
      size_t need = keypack_scratch_bytes(n, out_capacity) + (size_t)n * 4 + 512 + (size_t)slots * 8 + 512 +
                    (size_t)nstr * (((size_t)n * 8 + 255) + (size_t)slots * 8 + 512);
      if ((st = scratch_reserve(ctx, need, stream))) return st;
    }
    ghb_column pc[kMaxCols];
    for (int c = 0; c < ncols; c++) pc[c] = cols[c];
    int32_t pn = ncols;
    // the predicate as a pass flag column
    ghb_pred_node pass_node;
    ghb_predicate pass_pred{1, 0, &pass_node};
    const ghb_predicate* fpred = pred;
    int32_t* pass = nullptr;
    if (use_pass) {
      PredProg prog;
      if ((st = build_pred_prog(ctx, pred, cols, ncols, &prog))) return st;
      if ((st = scratch_alloc(ctx, (size_t)std::max<int64_t>(n, 1) * 4, (void**)&pass, stream))) return st;
      if ((st = predicate_pass(ctx, prog, cols, ncols, n, pass, stream))) return st;
      pc[pn] = ghb_column{GHB_INT, GHB_NULLS_NONE, pass, nullptr, nullptr, n};
      std::memset(&pass_node, 0, sizeof(pass_node));
      pass_node.mode = GHB_FILTER_EQ;
      pass_node.col = pn;
      pass_node.col2 = -1;
      pass_node.lit_i[0] = 1;
      pass_node.child[0] = pass_node.child[1] = -1;
      fpred = &pass_pred;
      pn++;
    }
    // STRING keys as the rows of their values' first occurrences
    int32_t kc[kMaxPackKeys];
    const int2* str_aux[kMaxPackKeys] = {nullptr};
    for (int j = 0; j < nkeys; j++) {
      kc[j] = key_cols[j];
      const ghb_column& c = cols[key_cols[j]];
      if (c.type != GHB_STRING) continue;
      int64_t* rep = nullptr;
      unsigned long long* table = nullptr;
      if ((st = scratch_alloc(ctx, (size_t)std::max<int64_t>(n, 1) * 8, (void**)&rep, stream))) return st;
      if ((st = scratch_alloc(ctx, (size_t)slots * 8, (void**)&table, stream))) return st;
      if ((st = string_rep_rows(ctx, c, pass, rep, table, slots, stream))) return st;
      pc[pn] = ghb_column{GHB_LONG, GHB_NULLS_SENTINEL, rep, nullptr, nullptr, n};
      kc[j] = pn++;
      str_aux[j] = (const int2*)c.aux;
    }
    if (!packed_key)   // a STRING predicate over one fixed-width key, or none
      return filter_groupby_impl(ctx, fpred, pc, pn, kc, nkeys, aggs, naggs, out, out_capacity, d_out_groups,
                                 cfg, stream, nullptr, 0);
    int64_t *packed = nullptr, *kout = nullptr;
    if ((st = scratch_alloc(ctx, (size_t)std::max<int64_t>(n, 1) * 8, (void**)&packed, stream))) return st;
    if ((st = scratch_alloc(ctx, (size_t)out_capacity * 8, (void**)&kout, stream))) return st;
    KeyPackPlan plan;
    bool too_wide = false;
    if ((st = keypack_prepare(ctx, pc, kc, nkeys, n, packed, &plan, stream, &too_wide))) return st;
    for (int j = 0; j < nkeys; j++) plan.str_aux[j] = str_aux[j];
    if (too_wide) {
      // group by the row of each tuple's first occurrence, then read each
      // group's tuple back from that row
      unsigned long long* table = nullptr;
      if ((st = scratch_alloc(ctx, (size_t)slots * 8, (void**)&table, stream))) return st;
      if ((st = tuple_rep_rows(ctx, pc, kc, nkeys, n, pass, packed, table, slots, stream))) return st;
      pc[pn] = ghb_column{GHB_LONG, GHB_NULLS_SENTINEL, packed, nullptr, nullptr, n};
      ghb_out_column po[kMaxAggs + 1];
      po[0] = ghb_out_column{GHB_LONG, 0, kout, nullptr};
      for (int i = 0; i < naggs && i < kMaxAggs; i++) po[1 + i] = out[nkeys + i];
      const int32_t pk = pn++;
      st = filter_groupby_impl(ctx, fpred, pc, pn, &pk, 1, aggs, naggs, po, out_capacity, d_out_groups, cfg,
                               stream, nullptr, 0);
      if (st) return st;
      return tuple_unpack(ctx, pc, kc, plan, kout, d_out_groups, out_capacity, out, stream);
    }
    pc[pn] = ghb_column{GHB_LONG, GHB_NULLS_NONE, packed, nullptr, nullptr, n};
    ghb_out_column po[kMaxAggs + 1];
    po[0] = ghb_out_column{GHB_LONG, 0, kout, nullptr};
    for (int i = 0; i < naggs && i < kMaxAggs; i++) po[1 + i] = out[nkeys + i];
    const int32_t pk = pn++;
    st = filter_groupby_impl(ctx, fpred, pc, pn, &pk, 1, aggs, naggs, po, out_capacity, d_out_groups, cfg, stream,
                             nullptr, 0);
    if (st) return st;
    return keypack_unpack(ctx, plan, kout, d_out_groups, out_capacity, out, stream);
  }
  GbSetup su{};
  su.max_groups = (cfg && cfg->max_groups > 0) ? cfg->max_groups : 0;
  su.smem_slots = cfg ? cfg->smem_slots : 0;
  su.threads = (cfg && cfg->block_threads == 512) ? 512 : kGbThreads;
  su.warp_agg = -1;
  su.tile_rows = cfg ? cfg->tile_rows : 0;
  su.nstages = cfg ? cfg->nstages : 0;
  if (cfg && cfg->global_slots_log2 > 0) {
    // an explicit table size: the load factor that yields it
    if (cfg->global_slots_log2 > 30)
      return set_error(ctx, GHB_ERR_INVALID, "global_slots_log2 %d > 30", cfg->global_slots_log2);
    su.max_groups = std::max<int64_t>(su.max_groups, 1);
    su.load_factor = (float)((double)su.max_groups / (double)(1ll << cfg->global_slots_log2));
  }
  GbParams p;
  FinParams f;
  size_t table_bytes = 0, smem = 0;
  // the kernel specialised for this signature when it compiles (not for the
  // allocation-free entry point: loading a kernel allocates), with the narrow
  // shared table; its u32 counters need fewer than 2^32 rows per CTA
  int64_t n_rows = 0;
  for (int c = 0; c < ncols; c++) n_rows = std::max<int64_t>(n_rows, cols ? cols[c].n : 0);
  su.narrow = !fixed_table && jit_enabled() && n_rows / std::max(1, ctx->num_sms) < (1ll << 31);
  int32_t st = gb_setup(ctx, pred, cols, ncols, key_cols, nkeys, aggs, naggs, out, out_capacity,
                        d_out_groups, su, &p, &f, &table_bytes, &smem);
  if (st) return st;
  const void* kfn = su.narrow ? jit_groupby_kernel(p, nkeys == 1, false, su.threads) : nullptr;
  if (su.narrow && !kfn) {
    su.narrow = 0;
    st = gb_setup(ctx, pred, cols, ncols, key_cols, nkeys, aggs, naggs, out, out_capacity, d_out_groups, su,
                  &p, &f, &table_bytes, &smem);
    if (st) return st;
  }

  void* table;
  if (fixed_table) {
    if (table_bytes > fixed_table_bytes)
      return set_error(ctx, GHB_ERR_CAPACITY, "group-by table needs %zu bytes, %zu available",
                       table_bytes, fixed_table_bytes);
    // a caller-provided table may hold anything: clear the part this call uses
    GHB_CUDA_TRY(ctx, cudaMemsetAsync(fixed_table, 0, table_bytes, stream));
    table = fixed_table;
  } else {
    if (table_bytes > ctx->gb_bytes || ctx->gb_dirty || !ctx->gb_table) {
      if (table_bytes > ctx->gb_bytes) {
        int32_t gst = regrow(ctx, &ctx->gb_table, &ctx->gb_bytes, std::max(table_bytes, (size_t)1 << 20),
                             stream, false);
        if (gst) return gst;
      }
      GHB_CUDA_TRY(ctx, cudaMemsetAsync(ctx->gb_table, 0, ctx->gb_bytes, stream));
      ctx->gb_dirty = false;
    }
    table = ctx->gb_table;
  }
  gb_table_bind(table, p.C, p.R, &p, &f);

  bool nullable = false;
  for (int c = 0; c < ncols; c++) nullable |= p.col_off[c] >= 0 && cols[c].null_mode != GHB_NULLS_NONE;
  if (!kfn)
    kfn = nkeys ? (nullable ? (const void*)gb_fold_kernel<true, true> : (const void*)gb_fold_kernel<true, false>)
                : (nullable ? (const void*)gb_fold_kernel<false, true> : (const void*)gb_fold_kernel<false, false>);
  const int threads = su.threads;
  int blocks_per_sm = 0;
  if (int32_t ast = ensure_dyn_smem(ctx, kfn, smem)) return ast;
  GHB_CUDA_TRY(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, kfn, threads, smem));
  blocks_per_sm = std::max(1, blocks_per_sm);
  if (cfg && cfg->ctas_per_sm > 0) blocks_per_sm = std::min(blocks_per_sm, cfg->ctas_per_sm);
  int grid = (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)ctx->num_sms * blocks_per_sm, p.ntiles));
  void* args[] = {&p};
  GHB_CUDA_TRY(ctx, cudaLaunchKernel(kfn, dim3(grid), dim3(threads), args, smem, stream));
  GHB_LAUNCH_CHECK(ctx);

  const int fgrid = (int)std::max<int64_t>(1, std::min<int64_t>(fin_units(p.C), (int64_t)ctx->num_sms * 8));
  gb_finalize_kernel<<<fgrid, kFinThreads, 0, stream>>>(f);
  GHB_LAUNCH_CHECK(ctx);
  return GHB_OK;
}

// Loads every kernel the fixed-table path can launch (the generic folds and
// the finalize) and sets their shared-memory attributes, so that a later call
// of that path loads no code.  CUDA loads kernels lazily, on first launch or
// first attribute query, and loading one may allocate device memory.
int32_t preload_fixed_table_kernels(ghb_ctx* ctx) {
  const void* folds[] = {(const void*)gb_fold_kernel<true, true>, (const void*)gb_fold_kernel<true, false>,
                         (const void*)gb_fold_kernel<false, true>, (const void*)gb_fold_kernel<false, false>};
  for (const void* fn : folds)
    if (int32_t st = ensure_dyn_smem(ctx, fn, 0)) return st;
  cudaFuncAttributes fa;
  GHB_CUDA_TRY(ctx, cudaFuncGetAttributes(&fa, (const void*)gb_finalize_kernel));
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
  CallScope cs(ctx, "filter_groupby", (cudaStream_t)stream);
  cs.rows(ncols > 0 && cols ? cols[0].n : 0);
  cs.bytes(cols_bytes(cols, ncols));
  scratch_reset(ctx);
  return cs.done(filter_groupby_impl(ctx, pred, cols, ncols, key_cols, nkeys, aggs, naggs, out, out_capacity,
                                     d_out_groups, cfg, (cudaStream_t)stream, nullptr, 0));
}
