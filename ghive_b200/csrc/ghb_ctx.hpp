// ghb_ctx.hpp — the context object behind ghb_ctx* and host-side helpers.
//
// A context owns: a device status word that kernels raise errors into, a
// growable device scratch arena, the look-back tile-status array (tagged
// with a launch epoch so it is never cleared per launch), the group-by table
// (left zeroed by the finalize kernel, so each call starts clean without a
// memset), and the kernel-launch counter.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/ghive_b200.h"
#include "ghb_internal.cuh"

namespace ghb {
constexpr int kStageLanes = 4;                // host threads of a staged copy at most
constexpr size_t kStagePiece = 8u << 20;      // bytes of one staging buffer
}  // namespace ghb

struct ghb_ctx {
  int device = 0;
  int num_sms = 148;
  int32_t* d_status = nullptr;            // device error word
  std::string last_error;
  int64_t launches = 0;

  // scratch arena (bump allocated per operator call)
  char* scratch = nullptr;
  size_t scratch_bytes = 0;
  size_t scratch_used = 0;

  // decoupled look-back tile status
  uint64_t* lb_status = nullptr;
  int64_t lb_tiles = 0;
  uint32_t epoch = 0;

  // polls of a not-ready earlier tile before a look-back gives up
  // (ghb_ctx_set_spin_limit)
  int32_t spin_limit = ghb::kSpinLimit;

  // self-resetting counters: [0] tile claim, [1] finished CTAs, ...
  unsigned long long* d_counters = nullptr;

  // group-by global table, zeroed after each finalize
  void* gb_table = nullptr;
  size_t gb_bytes = 0;
  bool gb_dirty = false;

  // pinned staging for the host-buffer entry points
  void* pinned = nullptr;
  size_t pinned_bytes = 0;

  // the host-buffer join's copy-in, compute and copy-out streams and its
  // per-chunk events (created on first use)
  cudaStream_t hstream[3] = {nullptr, nullptr, nullptr};
  cudaEvent_t hev[4][2] = {{nullptr, nullptr}, {nullptr, nullptr}, {nullptr, nullptr}, {nullptr, nullptr}};

  // Every call of this context runs on one stream (a server slot): its
  // device buffers grow with stream-ordered frees and allocations instead of
  // a device-wide synchronisation, so other streams keep running.
  bool stream_ordered = false;
  // Pool for those stream-ordered allocations (nullptr = the device's
  // default pool).
  cudaMemPool_t pool = nullptr;

  // pinned staging of pageable host memory (ghb_copy.cu): two buffers per
  // lane and the events that say their last copy is done
  void* stage[ghb::kStageLanes][2] = {};
  cudaEvent_t stage_ev[ghb::kStageLanes][2] = {};

  // per-call JSON log (ghb_ctx_set_log): the file, its level, the peak the
  // roofline fraction divides by (0: none), and level 2's events
  FILE* log = nullptr;
  int32_t log_level = 0;
  double log_peak_gbs = 0;
  cudaEvent_t log_ev[2] = {nullptr, nullptr};
};

namespace ghb {
// Replaces *buf (of *bytes) with a zeroed or uninitialised buffer of `want`
// bytes: stream-ordered on `stream` for a stream_ordered context, else after a
// device synchronisation.
int32_t regrow(ghb_ctx* ctx, void** buf, size_t* bytes, size_t want, cudaStream_t stream, bool zero);
// Lets kernel `fn` use up to `bytes` of dynamic shared memory on the current
// device.  The attribute is set once per kernel and device (to the device's
// opt-in maximum): changing a kernel's attributes on every call would put a
// runtime call that may wait on running work into every launch path.
int32_t ensure_dyn_smem(ghb_ctx* ctx, const void* fn, size_t bytes);
}  // namespace ghb

struct ghb_join_table {
  unsigned long long* kimg = nullptr;  // per slot: key image (0 = empty)
  int2* meta = nullptr;                // per slot: {first row + 1, rows with the key}
  ulonglong2* payw = nullptr;          // per slot: first row's inline payload words
  int32_t* chain = nullptr;   // per slot: chain head (row + 1) of the key's 2nd.. rows
  int32_t* next = nullptr;    // per build row: next row + 1 in its key's chain
  int64_t slots = 0;          // hashed slots (power of two); slot `slots` is the side slot
                              // (a direct table uses the first key-range slots of them)
  int64_t build_rows = 0;
  int32_t key_type = GHB_LONG;
  int32_t nbp = 0;            // build payload columns the table serves
  int32_t n_inline = 0;       // of which copied into the slots
  ghb_column pay[8];          // the build payload columns (caller-owned)
  unsigned long long* d_stats = nullptr;  // [0] rows stored, [1] max duplicates, [2..4] key range
  void* alloc = nullptr;      // slots, then chain, next and stats
  size_t alloc_bytes = 0;
  cudaStream_t stream = 0;    // build stream; the table is released in its order
  bool l2_window = false;
  int device = 0;             // device of the L2 window
  int32_t probe_threads = 256; // probe CTA size (ghb_join_cfg.block_threads)
};

namespace ghb {

int32_t set_error(ghb_ctx* ctx, int32_t code, const char* fmt, ...);

#define GHB_CUDA_TRY(ctx, expr)                                                        \
  do {                                                                                 \
    cudaError_t _e = (expr);                                                           \
    if (_e != cudaSuccess)                                                             \
      return ::ghb::set_error((ctx), GHB_ERR_CUDA, "%s failed: %s", #expr,            \
                              cudaGetErrorString(_e));                                 \
  } while (0)

#define GHB_LAUNCH_CHECK(ctx)                                                          \
  do {                                                                                 \
    (ctx)->launches++;                                                                 \
    cudaError_t _e = cudaGetLastError();                                               \
    if (_e != cudaSuccess)                                                             \
      return ::ghb::set_error((ctx), GHB_ERR_CUDA, "kernel launch failed: %s",         \
                              cudaGetErrorString(_e));                                 \
  } while (0)

// Reserves `bytes` (256-aligned) from the scratch arena; grows it when too
// small (a cudaFree + cudaMalloc after syncing the device).  Resets with
// scratch_reset at the start of an operator call.
int32_t scratch_reset(ghb_ctx* ctx);
int32_t scratch_alloc(ghb_ctx* ctx, size_t bytes, void** out, cudaStream_t stream);
int32_t scratch_reserve(ghb_ctx* ctx, size_t total, cudaStream_t stream);

// Look-back status array with room for `tiles` tiles, and a fresh epoch.
int32_t lookback_prepare(ghb_ctx* ctx, int64_t tiles, uint32_t* epoch, cudaStream_t stream);

// Checks column descriptors and their common row count; STRING columns (bytes
// + int32 [start,end) index) only where the operator takes them.
int32_t validate_columns(ghb_ctx* ctx, const ghb_column* cols, int32_t ncols, int64_t* n,
                         bool allow_string = false);
// The predicate tree as a post-order program (literals of STRING leaves
// copied into it); `cols` (nullable) gives the column types to check.
int32_t build_pred_prog(ghb_ctx* ctx, const ghb_predicate* pred, const ghb_column* cols, int32_t ncols,
                        PredProg* prog);

inline size_t type_width(int32_t t) { return t == GHB_INT ? 4 : 8; }

// ---- several GROUP BY keys packed into one int64 key (ghb_keypack.cu)
constexpr int kMaxPackKeys = 8;
struct KeyOuts {
  ghb_out_column o[kMaxPackKeys];
};
struct KeyPackPlan {
  int32_t nkeys;
  const int2* str_aux[kMaxPackKeys];   // a STRING key: its [start,end) index (the packed
                                       // column holds the row of its value's first occurrence)
  ghb_column col[kMaxPackKeys];
  uint64_t umin[kMaxPackKeys];     // min order image of the key's non-NULL values
  int8_t vbits[kMaxPackKeys];      // value field width
  int8_t vshift[kMaxPackKeys];     // value field position
  int8_t fshift[kMaxPackKeys];     // NULL flag position, -1 when the key has no NULLs
};
// Scratch bytes the packing needs beside the group-by itself.
inline size_t keypack_scratch_bytes(int64_t n, int64_t cap) {
  int64_t slots = 64;   // a tuple table of twice the groups (keys too wide to pack)
  while (slots < 2 * std::min<int64_t>(std::max<int64_t>(n, 1), std::max<int64_t>(cap, 1))) slots <<= 1;
  return 3 * 8 * kMaxPackKeys + 256 + (((size_t)n * 8 + 255) & ~(size_t)255) +
         (((size_t)cap * 8 + 255) & ~(size_t)255) + (size_t)slots * 8 + 1024;
}
// Plans the packing and writes the packed keys; *too_wide (and nothing
// written) when the tuples need more than 63 bits.
int32_t keypack_prepare(ghb_ctx* ctx, const ghb_column* cols, const int32_t* key_cols, int32_t nkeys,
                        int64_t n, int64_t* packed, KeyPackPlan* plan, cudaStream_t stream, bool* too_wide);
// Tuples too wide to pack: rep[r] = the row of row r's tuple's first
// occurrence (INT64_MAX where pass is 0); `slots` (power of two, >= twice the
// distinct tuples) of table, cleared here.  A full table raises
// GHB_ERR_CAPACITY on the device.
int32_t tuple_rep_rows(ghb_ctx* ctx, const ghb_column* cols, const int32_t* key_cols, int32_t nkeys, int64_t n,
                       const int32_t* pass, int64_t* rep, unsigned long long* table, int64_t slots,
                       cudaStream_t stream);
// The key tuple of each output group, from the group's first row.
int32_t tuple_unpack(ghb_ctx* ctx, const ghb_column* cols, const int32_t* key_cols, const KeyPackPlan& plan,
                     const int64_t* rows, const int64_t* d_groups, int64_t cap, const ghb_out_column* key_out,
                     cudaStream_t stream);
int32_t keypack_unpack(ghb_ctx* ctx, const KeyPackPlan& plan, const int64_t* packed,
                       const int64_t* d_groups, int64_t cap, const ghb_out_column* key_out,
                       cudaStream_t stream);
// A STRING column as an int64 column: each row holds the row of its value's
// first occurrence (INT64_MAX for NULL, and for rows whose pass flag is 0);
// `slots` (a power of two, >= twice the distinct values) of hash table in
// `table` (cleared here).  A full table raises GHB_ERR_CAPACITY on the device.
int32_t string_rep_rows(ghb_ctx* ctx, const ghb_column& c, const int32_t* pass, int64_t* rep,
                        unsigned long long* table, int64_t slots, cudaStream_t stream);
// The key tuples of a join's two sides (nkeys columns each, same types)
// packed with one plan into int64 columns with NULL maps (a tuple with a NULL
// component is NULL and matches nothing).  GHB_ERR_UNSUPPORTED past 63 bits.
int32_t keypack_join(ghb_ctx* ctx, const ghb_column* a, const ghb_column* b, int32_t nkeys, int64_t* a_packed,
                     uint8_t* a_null, int64_t* b_packed, uint8_t* b_null, cudaStream_t stream);
// Copies between host memory and the device (ghb_copy.cu).  Pinned or
// registered host memory goes by one asynchronous copy; pageable memory (a
// JVM direct buffer) through pinned staging buffers in up to kStageLanes
// host threads, each overlapping the host copy of one piece with the DMA of
// the previous one.  copy_h2d_many returns once the sources may be reused
// (the copies are queued on `stream`); copy_d2h_many returns with the data
// in host memory.
struct CopyTask {
  void* dst;
  const void* src;
  size_t bytes;
};
int32_t copy_h2d_many(ghb_ctx* ctx, const std::vector<CopyTask>& tasks, cudaStream_t stream);
int32_t copy_h2d(ghb_ctx* ctx, void* dst, const void* src, size_t bytes, cudaStream_t stream);
int32_t copy_d2h_many(ghb_ctx* ctx, const std::vector<CopyTask>& tasks, cudaStream_t stream);
// True when p is pinned (or registered) host memory.
bool host_pinned(const void* p);
// Exclusive prefix sums of n int64 counts, in place; their total to the
// device word *d_total.  One CTA for a few thousand counts, else tiles of
// 1024 claimed in order with decoupled look-back (bounded by the context's
// spin limit).
int32_t scan_counts(ghb_ctx* ctx, int64_t* counts, int64_t n, int64_t* d_total, cudaStream_t stream);
// pass[r] = 1 when row r passes the predicate program, else 0.
int32_t predicate_pass(ghb_ctx* ctx, const PredProg& prog, const ghb_column* cols, int32_t ncols, int64_t n,
                       int32_t* pass, cudaStream_t stream);

}  // namespace ghb
