// ghb_batch.cu — batched fused filter + group-by: many operator instances of
// one signature in one persistent kernel and one finalize, captured once in
// a CUDA graph and replayed.
//
// GHive runs GroupByPredicate::gpu_execute once per Tez task
// (GroupByOperator::execute, gpu_impl/src/Operator/GroupByOperator.cu:
// 101-130), so a vertex with hundreds of small splits pays a launch sequence,
// a sort and per-aggregate copies for each.  Here the instances share:
//
//   fold      gb_batch_fold_kernel: persistent CTAs claim chunks (a run of
//             tiles of one instance) from a list ordered by estimated cost,
//             largest first; a CTA keeps its shared-memory table while its
//             next chunk belongs to the same instance and flushes it into
//             that instance's global table when the instance changes.  The
//             per-tile work is fold_tile, the same code as the single call.
//   finalize  gb_batch_finalize_kernel: warps walk the claimed-slot bitmaps
//             of all instances at once; the last CTA publishes every
//             instance's group count and resets the counters.
//   autotune  candidate settings of the whole batch (CTA size, cap on the
//             shared-table slots, whether instances with many more groups
//             than the cap skip the shared table) are each planned and timed
//             on the batch itself, and the fastest is kept: the shared
//             reservation fixes every instance's tile size, and a setting
//             timed on one instance alone (warm in L2) misjudges the batch.
//   graph     the fold and finalize launches are captured once; a launch is
//             one cudaGraphLaunch.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <string>
#include <vector>

#include "ghb_groupby.cuh"

namespace ghb {

static_assert(sizeof(GbParams) % 8 == 0, "GbParams is copied to shared memory in 8-byte words");

struct BatchFinParams {
  const FinParams* fins;
  const int64_t* choff;        // [ninst + 1]: first finalize unit of each instance
  int32_t ninst;
  unsigned long long* done;
  unsigned long long* claim;
};

template <bool KEYED, bool NULLABLE>
__global__ void __launch_bounds__(kGbThreads) gb_batch_fold_kernel(BatchParams bp) {
  batch_fold_body<GenericFolder<KEYED, NULLABLE>>(bp);
}

__global__ void __launch_bounds__(kFinThreads) gb_batch_finalize_kernel(BatchFinParams b) {
  __shared__ uint64_t rb[kFinThreads * (kMaxAcc + 1)];
  const int64_t total = b.choff[b.ninst];
  for (int64_t ch = blockIdx.x; ch < total; ch += gridDim.x) {
    // the instance of unit ch: the last i with choff[i] <= ch
    int lo = 0, hi = b.ninst - 1;
    while (lo < hi) {
      int mid = (lo + hi + 1) >> 1;
      if (b.choff[mid] <= ch) lo = mid;
      else hi = mid - 1;
    }
    const FinParams& f = b.fins[lo];
    const int64_t local = ch - b.choff[lo];
    finalize_unit(f, local, rb);
    if (local == 0 && threadIdx.x == 0) finalize_sides(f, rb);
  }
  __shared__ int last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    last = atomicAdd(b.done, 1ull) == gridDim.x - 1;
  }
  __syncthreads();
  if (last) {
    __threadfence();
    for (int i = threadIdx.x; i < b.ninst; i += blockDim.x)
      *b.fins[i].d_out_groups = (int64_t)atomicExch(b.fins[i].growc, 0ull);
    if (threadIdx.x == 0) {
      *b.done = 0;
      *b.claim = 0;
    }
  }
}

const void* jit_groupby_kernel(const GbParams& p, bool keyed, bool batch, int threads);
bool jit_enabled();
std::string jit_groupby_source(const GbParams& p, bool keyed, bool batch, int threads);

static const void* fold_fn(bool keyed, bool nullable) {
  return keyed ? (nullable ? (const void*)gb_batch_fold_kernel<true, true>
                           : (const void*)gb_batch_fold_kernel<true, false>)
               : (nullable ? (const void*)gb_batch_fold_kernel<false, true>
                           : (const void*)gb_batch_fold_kernel<false, false>);
}

// Device image of a batch: params, chunk list, finalize offsets, counters and
// the global tables, in one allocation.
struct BatchImage {
  void* dev = nullptr;
  size_t bytes = 0;
  BatchParams bp{};
  BatchFinParams bf{};
  const void* fold = nullptr;   // the fold kernel (specialised or generic)
  int threads = kGbThreads;
  int grid = 1;
  int fgrid = 1;
  size_t smem = 0;
  bool specialised = false;   // the fold specialised for the batch's signature (else the generic one)
};

static size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

// Lays out and uploads a batch.  `tables` (nullable) is where the global
// tables go; otherwise they are placed in the image itself.  `chunk_tiles[i]`
// is the chunk length of instance i; `order` the order of instances in the
// chunk list.
static int32_t image_build(ghb_ctx* ctx, std::vector<GbParams>& ps, std::vector<FinParams>& fs,
                           const std::vector<int64_t>& chunk_tiles, const std::vector<int32_t>& order,
                           const void* fold, int threads, size_t smem_fold, int table_words,
                           cudaStream_t stream, BatchImage* im) {
  const int ninst = (int)ps.size();
  std::vector<BatchChunk> chunks;
  for (int32_t i : order) {
    const int64_t nt = ps[i].ntiles;
    const int64_t step = std::max<int64_t>(1, chunk_tiles[i]);
    for (int64_t t = 0; t < nt; t += step)
      chunks.push_back(BatchChunk{i, (int32_t)std::min<int64_t>(step, nt - t), t});
  }
  std::vector<int64_t> choff(ninst + 1, 0);
  for (int i = 0; i < ninst; i++) choff[i + 1] = choff[i] + fin_units(ps[i].C);

  size_t off = 0;
  const size_t o_ps = off;
  off = align256(off + sizeof(GbParams) * ninst);
  const size_t o_fs = off;
  off = align256(off + sizeof(FinParams) * ninst);
  const size_t o_ch = off;
  off = align256(off + sizeof(BatchChunk) * std::max<size_t>(1, chunks.size()));
  const size_t o_co = off;
  off = align256(off + sizeof(int64_t) * (ninst + 1));
  const size_t o_ctr = off;
  off = align256(off + 16);
  std::vector<size_t> o_tab(ninst);
  for (int i = 0; i < ninst; i++) {
    o_tab[i] = off;
    off = align256(off + gb_table_bytes(ps[i].C, ps[i].R));
  }
  if (cudaMalloc(&im->dev, off) != cudaSuccess) {
    cudaGetLastError();
    im->dev = nullptr;
    return set_error(ctx, GHB_ERR_OOM, "cannot allocate %zu bytes for the batch", off);
  }
  im->bytes = off;
  char* base = (char*)im->dev;
  for (int i = 0; i < ninst; i++) {
    gb_table_bind(base + o_tab[i], ps[i].C, ps[i].R, &ps[i], &fs[i]);
    fs[i].done = nullptr;  // the batched finalize counts CTAs with one counter
  }
  // tables and counters start zeroed; the finalize leaves them zeroed
  GHB_CUDA_TRY(ctx, cudaMemsetAsync(base + o_ctr, 0, off - o_ctr, stream));
  GHB_CUDA_TRY(ctx, cudaMemcpyAsync(base + o_ps, ps.data(), sizeof(GbParams) * ninst, cudaMemcpyHostToDevice, stream));
  GHB_CUDA_TRY(ctx, cudaMemcpyAsync(base + o_fs, fs.data(), sizeof(FinParams) * ninst, cudaMemcpyHostToDevice, stream));
  if (!chunks.empty())
    GHB_CUDA_TRY(ctx, cudaMemcpyAsync(base + o_ch, chunks.data(), sizeof(BatchChunk) * chunks.size(),
                                      cudaMemcpyHostToDevice, stream));
  GHB_CUDA_TRY(ctx, cudaMemcpyAsync(base + o_co, choff.data(), sizeof(int64_t) * (ninst + 1), cudaMemcpyHostToDevice, stream));
  // the host vectors go out of scope: the copies must have read them
  GHB_CUDA_TRY(ctx, cudaStreamSynchronize(stream));

  unsigned long long* ctr = (unsigned long long*)(base + o_ctr);
  im->bp.insts = (const GbParams*)(base + o_ps);
  im->bp.chunks = (const BatchChunk*)(base + o_ch);
  im->bp.nchunks = (int64_t)chunks.size();
  im->bp.claim = ctr;
  im->bp.stage_bytes = ps.empty() ? 0 : ps[0].stage_bytes;
  im->bp.table_words = table_words;
  im->bf.fins = (const FinParams*)(base + o_fs);
  im->bf.choff = (const int64_t*)(base + o_co);
  im->bf.ninst = ninst;
  im->bf.done = ctr + 1;
  im->bf.claim = ctr;
  im->fold = fold;
  im->threads = threads;
  im->smem = smem_fold;
  if (int32_t ast = ensure_dyn_smem(ctx, (const void*)im->fold, smem_fold)) return ast;
  int per_sm = 0;
  GHB_CUDA_TRY(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, im->fold, threads, smem_fold));
  per_sm = std::max(1, per_sm);
  im->grid = (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)ctx->num_sms * per_sm,
                                                          std::max<int64_t>(1, (int64_t)chunks.size())));
  im->fgrid = (int)std::max<int64_t>(1, std::min<int64_t>(choff[ninst], (int64_t)ctx->num_sms * 8));
  return GHB_OK;
}

static int32_t image_launch(ghb_ctx* ctx, const BatchImage& im, cudaStream_t stream) {
  if (im.bp.nchunks > 0) {
    BatchParams bp = im.bp;
    void* args[] = {&bp};
    GHB_CUDA_TRY(ctx, cudaLaunchKernel(im.fold, dim3(im.grid), dim3(im.threads), args, im.smem, stream));
    GHB_LAUNCH_CHECK(ctx);
  }
  gb_batch_finalize_kernel<<<im.fgrid, kFinThreads, 0, stream>>>(im.bf);
  GHB_LAUNCH_CHECK(ctx);
  return GHB_OK;
}

static void image_free(BatchImage* im) {
  if (im->dev) cudaFree(im->dev);
  im->dev = nullptr;
}

// ------------------------------------------------------------ autotuner
// A setting of the whole batch.  Shared memory is reserved per CTA for the
// largest shared table any instance uses, and that reservation fixes the
// tile size of every instance, so the settings are chosen for the batch as a
// whole and timed on the batch itself (its real sizes, its real L2 traffic).
struct BatchSetting {
  int32_t threads;      // CTA size: 512 or 1024
  int32_t smem_cap;     // shared-table slots at most; 0 = none (a global aggregate keeps 64)
  int32_t skip_large;   // 1: instances with more than 16 * smem_cap groups skip the shared table
  float load_factor;    // global tables
  // per group-count class (group_class): the global tables' load factor,
  // 0 = load_factor.  The autotuner's second stage sets these class by class.
  float lf_class[4];
};

static const char* kRowClass[] = {"<1e4", "1e4-1e5", "1e5-1e6", ">=1e6"};
static const char* kGroupClass[] = {"<=64", "65-2048", "2049-32768", ">32768"};

static int row_class(int64_t n) { return n < 10000 ? 0 : n < 100000 ? 1 : n < 1000000 ? 2 : 3; }
static int group_class(int64_t g) { return g <= 64 ? 0 : g <= 2048 ? 1 : g <= 32768 ? 2 : 3; }

}  // namespace ghb

struct ghb_batch {
  ghb_ctx* ctx = nullptr;
  ghb::BatchImage im;
  cudaStream_t cap_stream = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  std::string report;
};

namespace ghb {

struct InstSpec {
  const ghb_groupby_instance* in;
  int64_t rows;
  int64_t groups;
  int cls;
};

// Shared-table slots of one instance under a setting (-1: none).
static int32_t inst_slots(const InstSpec& s, int32_t nkeys, const BatchSetting& bs) {
  if (nkeys == 0) return 64;
  if (bs.smem_cap <= 0) return -1;
  if (bs.skip_large && s.groups > 16 * (int64_t)bs.smem_cap) return -1;
  return (int32_t)std::min<int64_t>(bs.smem_cap, std::max<int64_t>(64, next_pow2_i64(2 * s.groups)));
}

static int32_t setup_inst(ghb_ctx* ctx, const InstSpec& s, int32_t ncols, const int32_t* key_cols,
                          int32_t nkeys, const ghb_agg_desc* aggs, int32_t naggs, int64_t* d_count,
                          const BatchSetting& bs, int tile_rows, int reserve, bool narrow, GbParams* p,
                          FinParams* f, size_t* tb, size_t* smem) {
  GbSetup su{};
  su.max_groups = s.groups;
  su.smem_slots = inst_slots(s, nkeys, bs);
  const float lfc = bs.lf_class[group_class(s.groups)];
  su.load_factor = lfc > 0.f ? lfc : bs.load_factor;
  su.threads = bs.threads;
  su.tile_rows = tile_rows;
  su.smem_table_slots = reserve;
  su.warp_agg = -1;
  su.extra_smem = (int32_t)batch_extra_smem();
  su.nstages = 2;   // the batched fold double-buffers its tiles
  su.narrow = narrow ? 1 : 0;
  return gb_setup(ctx, s.in->pred, s.in->cols, ncols, key_cols, nkeys, aggs, naggs, s.in->out,
                  s.in->out_capacity, d_count, su, p, f, tb, smem);
}

static size_t batch_smem(size_t fold_smem) { return fold_smem + batch_extra_smem(); }

struct BatchSig {
  int32_t ncols;
  const int32_t* key_cols;
  int32_t nkeys;
  const ghb_agg_desc* aggs;
  int32_t naggs;
  int64_t* d_out_groups;
  bool nullable;
};

// Sets every instance up under `bs` (one stage layout and shared reservation
// for all) with the narrow shared table of the specialised folds or the wide
// one of the generic fold.  Returns GHB_ERR_UNSUPPORTED (with no error set)
// when `narrow` cannot be used.
static int32_t setup_all(ghb_ctx* ctx, const std::vector<InstSpec>& spec, const BatchSig& sig,
                         const BatchSetting& bs, bool narrow, std::vector<GbParams>& ps,
                         std::vector<FinParams>& fs, size_t* smem_fold) {
  const int ninst = (int)spec.size();
  int reserve = 0;
  for (int i = 0; i < ninst; i++) {
    size_t tb = 0, smem = 0;
    int32_t st = setup_inst(ctx, spec[i], sig.ncols, sig.key_cols, sig.nkeys, sig.aggs, sig.naggs,
                            sig.d_out_groups + i, bs, 0, 0, narrow, &ps[i], &fs[i], &tb, &smem);
    if (st) return st;
    reserve = std::max(reserve, ps[i].smem_slots);
  }
  // the most rows per thread whose stages fit every instance
  for (int tile_rows = kGbRows * bs.threads;; tile_rows /= 2) {
    bool ok = true;
    *smem_fold = 0;
    for (int i = 0; i < ninst && ok; i++) {
      size_t tb = 0, smem = 0;
      int32_t st = setup_inst(ctx, spec[i], sig.ncols, sig.key_cols, sig.nkeys, sig.aggs, sig.naggs,
                              sig.d_out_groups + i, bs, tile_rows, reserve, narrow, &ps[i], &fs[i], &tb, &smem);
      if (st) {
        if (tile_rows <= bs.threads) return st;
        ok = false;
        ctx->last_error.clear();
      }
      *smem_fold = std::max(*smem_fold, smem);
    }
    if (ok) break;
  }
  for (int i = 1; i < ninst; i++) {
    bool same = ps[i].stage_bytes == ps[0].stage_bytes && ps[i].tile_rows == ps[0].tile_rows &&
                ps[i].acc.n_acc == ps[0].acc.n_acc && ps[i].key_col == ps[0].key_col &&
                ps[i].table_words == ps[0].table_words;
    for (int c = 0; c < kMaxCols; c++) same = same && ps[i].col_off[c] == ps[0].col_off[c];
    if (!same)
      return set_error(ctx, GHB_ERR_INVALID,
                       "instance %d: predicate or aggregates read other columns than instance 0", i);
  }
  return GHB_OK;
}

// Orders and chunks the work of the batch under `bs` and builds the device
// image: the fold specialised for the batch's signature (narrow shared
// table) when every instance has the same signature and fewer than 2^31 rows
// (its shared counters are 32-bit), else the generic fold.
static int32_t plan_image(ghb_ctx* ctx, const std::vector<InstSpec>& spec, const BatchSig& sig,
                          const BatchSetting& bs, cudaStream_t stream, BatchImage* im,
                          std::vector<GbParams>* ps_out) {
  const int ninst = (int)spec.size();
  std::vector<GbParams> ps(ninst);
  std::vector<FinParams> fs(ninst);
  size_t smem_fold = 0;
  const void* fn = nullptr;
  bool specialised = false;
  if (jit_enabled()) {
    int32_t st = setup_all(ctx, spec, sig, bs, true, ps, fs, &smem_fold);
    if (st) return st;
    bool ok = true;
    for (int i = 0; i < ninst && ok; i++) ok = ps[i].n < (1ll << 31);
    if (ok) {
      const std::string s0 = jit_groupby_source(ps[0], sig.nkeys == 1, true, bs.threads);
      for (int i = 1; i < ninst && ok; i++) ok = jit_groupby_source(ps[i], sig.nkeys == 1, true, bs.threads) == s0;
    }
    if (ok) fn = jit_groupby_kernel(ps[0], sig.nkeys == 1, true, bs.threads);
    specialised = fn != nullptr;
  }
  if (!specialised) {
    int32_t st = setup_all(ctx, spec, sig, bs, false, ps, fs, &smem_fold);
    if (st) return st;
    fn = fold_fn(sig.nkeys == 1, sig.nullable);
  }
  const size_t smem = batch_smem(smem_fold);
  const int table_words = ps[0].table_words;

  // chunk list: instances by size, largest first, each cut into chunks so
  // that every CTA claims several; a fixed cost per instance stands for its
  // table flush and finalize
  std::vector<double> cost(ninst);
  double total = 0;
  for (int i = 0; i < ninst; i++) {
    cost[i] = (double)spec[i].rows + 4096.0;
    total += cost[i];
  }
  std::vector<int32_t> order(ninst);
  for (int i = 0; i < ninst; i++) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int32_t x, int32_t y) { return cost[x] > cost[y]; });
  int per_sm = 1;
  if (int32_t ast = ensure_dyn_smem(ctx, fn, smem)) return ast;
  GHB_CUDA_TRY(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, bs.threads, smem));
  per_sm = std::max(1, per_sm);
  const double target = total / ((double)ctx->num_sms * per_sm * 6.0);
  std::vector<int64_t> chunk_tiles(ninst);
  for (int i = 0; i < ninst; i++) {
    const double per_tile = cost[i] / (double)std::max<int64_t>(1, ps[i].ntiles);
    chunk_tiles[i] = std::max<int64_t>(1, (int64_t)(target / std::max(per_tile, 1e-9)));
  }
  int32_t st = image_build(ctx, ps, fs, chunk_tiles, order, fn, bs.threads, smem, table_words, stream, im);
  if (st) return st;
  im->specialised = specialised;
  if (ps_out) *ps_out = ps;
  return GHB_OK;
}

// Median-free timing: the best of `reps` launches after one warm-up, in ms.
static double time_image(ghb_ctx* ctx, const BatchImage& im, cudaStream_t stream, int reps) {
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  double best = 1e300;
  int32_t st = GHB_OK;
  for (int rep = 0; rep <= reps && st == GHB_OK; rep++) {
    cudaEventRecord(a, stream);
    st = image_launch(ctx, im, stream);
    cudaEventRecord(b, stream);
    cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    if (rep > 0) best = std::min(best, (double)ms);
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return st == GHB_OK ? best : -1.0;
}

static int32_t batch_create(ghb_ctx* ctx, const ghb_groupby_instance* inst, int32_t ninst, int32_t ncols,
                            const int32_t* key_cols, int32_t nkeys, const ghb_agg_desc* aggs,
                            int32_t naggs, int64_t* d_out_groups, const ghb_batch_cfg* cfg,
                            cudaStream_t stream, ghb_batch* b) {
  if (ninst < 1) return set_error(ctx, GHB_ERR_INVALID, "ninst=%d: a batch needs an instance", ninst);
  if (!inst) return set_error(ctx, GHB_ERR_INVALID, "instances is NULL");
  if (!d_out_groups) return set_error(ctx, GHB_ERR_INVALID, "d_out_groups is NULL");
  if (ncols < 1 || ncols > kMaxCols)
    return set_error(ctx, GHB_ERR_INVALID, "ncols=%d outside [1,%d]", ncols, kMaxCols);
  std::vector<InstSpec> spec(ninst);
  for (int i = 0; i < ninst; i++) {
    if (!inst[i].cols) return set_error(ctx, GHB_ERR_INVALID, "instance %d: cols is NULL", i);
    int64_t n = 0;
    int32_t st = validate_columns(ctx, inst[i].cols, ncols, &n);
    if (st) return st;
    int64_t g = inst[i].max_groups > 0 ? inst[i].max_groups : inst[i].out_capacity;
    if (nkeys == 0) g = 1;
    g = std::max<int64_t>(1, std::min<int64_t>(g, std::max<int64_t>(n, 1)));
    spec[i] = InstSpec{&inst[i], n, g, row_class(n) * 4 + group_class(g)};
  }
  // one signature: column types and NULL modes as in instance 0
  bool nullable = false;
  for (int i = 0; i < ninst; i++)
    for (int c = 0; c < ncols; c++) {
      if (inst[i].cols[c].type != inst[0].cols[c].type)
        return set_error(ctx, GHB_ERR_INVALID, "instance %d: column %d has type %d, instance 0 has %d", i,
                         c, inst[i].cols[c].type, inst[0].cols[c].type);
      nullable |= inst[i].cols[c].null_mode != GHB_NULLS_NONE;
    }

  const BatchSig sig{ncols, key_cols, nkeys, aggs, naggs, d_out_groups, nullable};
  const bool tune = cfg && cfg->autotune;
  const int forced_threads =
      (cfg && (cfg->block_threads == 512 || cfg->block_threads == 1024)) ? cfg->block_threads : 0;
  const float lf = (cfg && cfg->load_factor > 0.f) ? cfg->load_factor : 0.5f;
  BatchSetting base{forced_threads ? forced_threads : kGbThreads, 2048, 0, lf, {0.f, 0.f, 0.f, 0.f}};
  if (cfg && cfg->smem_slots < 0) base.smem_cap = 0;
  if (cfg && cfg->smem_slots > 0) base.smem_cap = (int32_t)next_pow2_i64(cfg->smem_slots);
  std::vector<BatchSetting> cands{base};
  if (tune) {
    cands.clear();
    for (int th : {1024, 512}) {
      if (forced_threads && th != forced_threads) continue;
      std::vector<int> caps{0, 512, 1024, 2048, 4096};
      if (cfg && cfg->smem_slots) caps = {base.smem_cap};
      for (int cap : caps)
        for (int skip = 0; skip < (cap > 0 && nkeys == 1 ? 2 : 1); skip++)
          cands.push_back({th, cap, skip, lf, {0.f, 0.f, 0.f, 0.f}});
    }
  }
  std::string trials = "[";
  double best_ms = 1e300;
  BatchSetting best = cands[0];
  if (cands.size() > 1) {
    for (const BatchSetting& c : cands) {
      BatchImage im;
      int32_t st = plan_image(ctx, spec, sig, c, stream, &im, nullptr);
      double ms = st ? -1.0 : time_image(ctx, im, stream, 2);
      cudaStreamSynchronize(stream);
      image_free(&im);
      if (st) ctx->last_error.clear();
      char tb[160];
      snprintf(tb, sizeof(tb), "%s{\"threads\": %d, \"smem_cap\": %d, \"skip_large\": %d, \"ms\": %.4f}",
               trials.size() > 1 ? ", " : "", c.threads, c.smem_cap, c.skip_large, ms);
      trials += tb;
      if (ms > 0 && ms < best_ms) {
        best_ms = ms;
        best = c;
      }
    }
    // Second stage, per size class: the load factor of the global tables of
    // the instances of one group-count class (the others keep theirs), tried
    // class by class on the batch itself, kept when the batch gets faster.
    // A sparser table has fewer collisions; a denser one stays in L2.
    if (nkeys == 1 && !(cfg && cfg->load_factor > 0.f)) {
      for (int gc = 0; gc < 4; gc++) {
        bool present = false;
        for (const InstSpec& sp : spec) present |= group_class(sp.groups) == gc;
        if (!present) continue;
        for (float cand : {0.25f, 0.75f}) {
          BatchSetting c = best;
          c.lf_class[gc] = cand;
          BatchImage im;
          int32_t st = plan_image(ctx, spec, sig, c, stream, &im, nullptr);
          double ms = st ? -1.0 : time_image(ctx, im, stream, 2);
          cudaStreamSynchronize(stream);
          image_free(&im);
          if (st) ctx->last_error.clear();
          char tb[200];
          snprintf(tb, sizeof(tb), ", {\"groups\": \"%s\", \"load_factor\": %.2f, \"ms\": %.4f}",
                   kGroupClass[gc], cand, ms);
          trials += tb;
          if (ms > 0 && ms < best_ms) {
            best_ms = ms;
            best = c;
          }
        }
      }
    }
    // a tuning launch may have raised a device status (a short output): clear it
    cudaMemsetAsync(ctx->d_status, 0, sizeof(int32_t), stream);
  }
  trials += "]";
  std::vector<GbParams> ps;
  int32_t st = plan_image(ctx, spec, sig, best, stream, &b->im, &ps);
  if (st) return st;

  // report: the setting, the trials and the shared slots per size class
  char buf[512];
  std::string rep_s = "{\"block_threads\": " + std::to_string(best.threads) +
                      ", \"smem_cap\": " + std::to_string(best.smem_cap) +
                      ", \"skip_large\": " + std::to_string(best.skip_large) +
                      ", \"load_factor\": " + std::to_string(best.load_factor) +
                      ", \"tile_rows\": " + std::to_string(ps[0].tile_rows) +
                      ", \"grid\": " + std::to_string(b->im.grid) +
                      ", \"chunks\": " + std::to_string(b->im.bp.nchunks) +
                      ", \"smem_bytes\": " + std::to_string(b->im.smem) +
                      ", \"kernel\": \"" + (b->im.specialised ? "specialised" : "generic") + "\"" +
                      ", \"autotuned\": " + (tune ? "true" : "false") + ", \"trials\": " + trials +
                      ", \"classes\": [";
  bool first = true;
  for (int k = 0; k < 16; k++) {
    int cnt = 0, slots = 0;
    double rows = 0;
    for (int i = 0; i < ninst; i++)
      if (spec[i].cls == k) {
        cnt++;
        rows += (double)spec[i].rows;
        slots = std::max(slots, ps[i].smem_slots);
      }
    if (!cnt) continue;
    snprintf(buf, sizeof(buf),
             "%s{\"rows\": \"%s\", \"groups\": \"%s\", \"instances\": %d, \"total_rows\": %.0f, "
             "\"smem_slots\": %d, \"load_factor\": %.2f}",
             first ? "" : ", ", kRowClass[k / 4], kGroupClass[k % 4], cnt, rows, slots,
             best.lf_class[k % 4] > 0.f ? best.lf_class[k % 4] : best.load_factor);
    rep_s += buf;
    first = false;
  }
  rep_s += "]}";
  b->report = rep_s;

  // capture the launches once
  const bool graph = !cfg || cfg->use_graph != 0;
  if (graph) {
    GHB_CUDA_TRY(ctx, cudaStreamCreateWithFlags(&b->cap_stream, cudaStreamNonBlocking));
    GHB_CUDA_TRY(ctx, cudaStreamBeginCapture(b->cap_stream, cudaStreamCaptureModeThreadLocal));
    const int64_t before = ctx->launches;
    int32_t lst = image_launch(ctx, b->im, b->cap_stream);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(b->cap_stream, &g);
    ctx->launches = before;  // captured, not launched
    if (lst) {
      if (g) cudaGraphDestroy(g);
      return lst;
    }
    if (e != cudaSuccess) return set_error(ctx, GHB_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(e));
    b->graph = g;
    e = cudaGraphInstantiate(&b->exec, g, 0);
    if (e != cudaSuccess) return set_error(ctx, GHB_ERR_CUDA, "graph instantiate failed: %s", cudaGetErrorString(e));
  }
  return GHB_OK;
}

static void batch_release(ghb_batch* b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  if (b->cap_stream) cudaStreamDestroy(b->cap_stream);
  image_free(&b->im);
}

}  // namespace ghb

using namespace ghb;

extern "C" int32_t ghb_batch_groupby_create(ghb_ctx* ctx, const ghb_groupby_instance* inst, int32_t ninst,
                                            int32_t ncols, const int32_t* key_cols, int32_t nkeys,
                                            const ghb_agg_desc* aggs, int32_t naggs, int64_t* d_out_groups,
                                            const ghb_batch_cfg* cfg, void* stream, ghb_batch** out) {
  if (!ctx || !out) return GHB_ERR_INVALID;
  *out = nullptr;
  cudaSetDevice(ctx->device);
  ghb_batch* b = new ghb_batch();
  b->ctx = ctx;
  int32_t st = batch_create(ctx, inst, ninst, ncols, key_cols, nkeys, aggs, naggs, d_out_groups, cfg,
                            (cudaStream_t)stream, b);
  if (st) {
    cudaStreamSynchronize((cudaStream_t)stream);
    batch_release(b);
    delete b;
    return st;
  }
  *out = b;
  return GHB_OK;
}

extern "C" int32_t ghb_batch_launch(ghb_batch* b, void* stream) {
  if (!b) return GHB_ERR_INVALID;
  ghb_ctx* ctx = b->ctx;
  if (b->exec) {
    cudaError_t e = cudaGraphLaunch(b->exec, (cudaStream_t)stream);
    if (e != cudaSuccess) return set_error(ctx, GHB_ERR_CUDA, "graph launch failed: %s", cudaGetErrorString(e));
    ctx->launches += b->im.bp.nchunks > 0 ? 2 : 1;
    return GHB_OK;
  }
  return image_launch(ctx, b->im, (cudaStream_t)stream);
}

extern "C" int32_t ghb_batch_describe(const ghb_batch* b, char* buf, int64_t len) {
  if (!b || !buf || len < 1) return GHB_ERR_INVALID;
  const size_t n = std::min<size_t>((size_t)len - 1, b->report.size());
  std::memcpy(buf, b->report.data(), n);
  buf[n] = 0;
  return b->report.size() < (size_t)len ? GHB_OK : GHB_ERR_CAPACITY;
}

extern "C" int32_t ghb_batch_destroy(ghb_batch* b) {
  if (!b) return GHB_OK;
  cudaSetDevice(b->ctx->device);
  batch_release(b);
  delete b;
  return GHB_OK;
}
