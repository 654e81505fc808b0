// ghb_internal.cuh — device-side building blocks shared by the kernels.
//
// Column access with Hive / GHive NULL conventions, the predicate-tree
// evaluator, order-preserving integer transforms, hashing, and the bounded
// decoupled look-back used by every order-preserving compaction.
#pragma once

// Also compiled at run time by NVRTC (specialised group-by kernels), which
// has no host headers: those are included only for the offline build.
#ifndef __CUDACC_RTC__
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#endif

#include "../../include/ghive_b200.h"

namespace ghb {

constexpr int kMaxCols = 12;          // input columns one operator call may touch
constexpr int kWarp = 32;
constexpr int kSpinLimit = 1 << 21;   // look-back polls (~1 s) before GHB_ERR_TIMEOUT

// Device status word values (first error wins).
enum DevStatus : int32_t {
  kDevOk = 0,
  kDevTimeout = GHB_ERR_TIMEOUT,
  kDevCapacity = GHB_ERR_CAPACITY,
};

// Column descriptors passed by value in kernel parameters.
struct ColSet {
  ghb_column c[kMaxCols];
  int32_t n;
};

// Predicate program: nodes in post-order (children before parents), so one
// forward sweep evaluates the tree with a bit per node.
struct PredProg {
  ghb_pred_node nodes[GHB_MAX_PRED_NODES];   // a STRING leaf's literal k is
                                             // sbytes[lit_i[k]], lit_s_len[k] bytes
  int32_t n_nodes;   // 0 = no predicate (all rows pass)
  int32_t has_str;   // some leaf reads a STRING column
  uint8_t sbytes[GHB_MAX_PRED_STR_BYTES];
};

// ----------------------------------------------------------- status
__device__ __forceinline__ void raise_status(int32_t* status, int32_t code) {
  atomicCAS(status, 0, code);
}

// ----------------------------------------------------------- column loads
__device__ __forceinline__ int64_t ld_i64(const ghb_column& c, int64_t i) {
  if (c.type == GHB_INT) return (int64_t)__ldg((const int32_t*)c.data + i);
  return __ldg((const long long*)c.data + i);   // LONG, or DOUBLE bits
}

// Raw 64-bit payload of row i: int32 sign-extended, int64 as is, double bits.
__device__ __forceinline__ int64_t ld_raw(const ghb_column& c, int64_t i) {
  return ld_i64(c, i);
}

// Same, for data read exactly once: an evict-first load (ld.global.cs) keeps
// a streamed column from pushing reused data (hash tables) out of L2.
__device__ __forceinline__ int64_t ld_raw_cs(const ghb_column& c, int64_t i) {
  if (c.type == GHB_INT) return (int64_t)__ldcs((const int*)c.data + i);
  return (int64_t)__ldcs((const long long*)c.data + i);
}

__device__ __forceinline__ double raw_to_f64(int type, int64_t raw) {
  return type == GHB_DOUBLE ? __longlong_as_double(raw) : (double)raw;
}

__device__ __forceinline__ bool raw_is_null(const ghb_column& c, int64_t raw, int64_t i) {
  if (c.null_mode == GHB_NULLS_NONE) return false;
  if (c.null_mode == GHB_NULLS_BYTEMAP) return c.is_null[i] != 0;
  if (c.type == GHB_INT) return raw == (int64_t)INT32_MAX;
  if (c.type == GHB_LONG) return raw == INT64_MAX;
  double d = __longlong_as_double(raw);
  return d != d;
}

// ----------------------------------------------------------- predicates
template <typename T>
__device__ __forceinline__ bool cmp_mode(int mode, T x, T a, T b) {
  switch (mode) {
    case GHB_FILTER_EQ: return x == a;
    case GHB_FILTER_LE: return x <= a;
    case GHB_FILTER_GE: return x >= a;
    case GHB_FILTER_LT: return x < a;
    case GHB_FILTER_GT: return x > a;
    case GHB_FILTER_RANGE: return x > a && x < b;
    case GHB_FILTER_EQ_RANGE: return a <= x && x <= b;
    case GHB_FILTER_NOT_EQ: return x != a;
    case GHB_FILTER_NOT_RANGE: return x < a || x > b;
    case GHB_FILTER_NOT_EQ_RANGE: return x <= a || x >= b;
  }
  return false;
}

// Hive's StringExpr.compare: unsigned bytes, then length.
__device__ __forceinline__ int str_compare(const uint8_t* a, int la, const uint8_t* b, int lb) {
  const int m = la < lb ? la : lb;
  for (int k = 0; k < m; k++)
    if (a[k] != b[k]) return (int)a[k] - (int)b[k];
  return la - lb;
}

// A leaf on a STRING column (data: bytes, aux: int32 [start,end) per row,
// start < 0 = NULL), against the program's literals or another STRING column.
static __device__ __noinline__ bool eval_str_leaf(const PredProg& p, const ghb_pred_node& nd, const ColSet& cs,
                                           int64_t i) {
  const ghb_column& c = cs.c[nd.col];
  const int2 ix = ((const int2*)c.aux)[i];
  if (ix.x < 0) return false;
  if (nd.mode == GHB_FILTER_NOT_NULL) return true;
  const uint8_t* x = (const uint8_t*)c.data + ix.x;
  int ca, cb = 0;
  if (nd.col2 >= 0) {
    const ghb_column& c2 = cs.c[nd.col2];
    const int2 iy = ((const int2*)c2.aux)[i];
    if (iy.x < 0) return false;
    ca = str_compare(x, ix.y - ix.x, (const uint8_t*)c2.data + iy.x, iy.y - iy.x);
  } else {
    ca = str_compare(x, ix.y - ix.x, p.sbytes + nd.lit_i[0], nd.lit_s_len[0]);
    cb = str_compare(x, ix.y - ix.x, p.sbytes + nd.lit_i[1], nd.lit_s_len[1]);
  }
  switch (nd.mode) {
    case GHB_FILTER_EQ: return ca == 0;
    case GHB_FILTER_LE: return ca <= 0;
    case GHB_FILTER_GE: return ca >= 0;
    case GHB_FILTER_LT: return ca < 0;
    case GHB_FILTER_GT: return ca > 0;
    case GHB_FILTER_RANGE: return ca > 0 && cb < 0;
    case GHB_FILTER_EQ_RANGE: return ca >= 0 && cb <= 0;
    case GHB_FILTER_NOT_EQ: return ca != 0;
    case GHB_FILTER_NOT_RANGE: return ca < 0 || cb > 0;
    case GHB_FILTER_NOT_EQ_RANGE: return ca <= 0 || cb >= 0;
  }
  return false;
}

// A leaf against literals on a fixed-width column c, given row i's raw value x.
__device__ __forceinline__ bool leaf_on_raw(const ghb_pred_node& nd, const ghb_column& c, int64_t x, int64_t i) {
  if (raw_is_null(c, x, i)) return false;
  if (nd.mode == GHB_FILTER_NOT_NULL) return true;
  if (c.type == GHB_DOUBLE || nd.lit_is_double) {
    double a = nd.lit_is_double ? nd.lit_d[0] : (double)nd.lit_i[0];
    double b = nd.lit_is_double ? nd.lit_d[1] : (double)nd.lit_i[1];
    return cmp_mode<double>(nd.mode, raw_to_f64(c.type, x), a, b);
  }
  return cmp_mode<int64_t>(nd.mode, x, nd.lit_i[0], nd.lit_i[1]);
}

// One leaf of FilterPredicate (FilterPredicate.hpp:119-385 functors, with
// Hive's NULL rule: a NULL operand never passes).
__device__ __forceinline__ bool eval_leaf(const PredProg& p, const ghb_pred_node& nd, const ColSet& cs,
                                          int64_t i) {
  const ghb_column& c = cs.c[nd.col];
  if (p.has_str && c.type == GHB_STRING) return eval_str_leaf(p, nd, cs, i);
  int64_t x = ld_raw(c, i);
  if (nd.col2 < 0) return leaf_on_raw(nd, c, x, i);
  // against another column of the same row
  if (raw_is_null(c, x, i)) return false;
  if (nd.mode == GHB_FILTER_NOT_NULL) return true;
  const ghb_column& c2 = cs.c[nd.col2];
  int64_t y = ld_raw(c2, i);
  if (raw_is_null(c2, y, i)) return false;
  if (c.type == GHB_DOUBLE || c2.type == GHB_DOUBLE)
    return cmp_mode<double>(nd.mode, raw_to_f64(c.type, x), raw_to_f64(c2.type, y), 0.0);
  return cmp_mode<int64_t>(nd.mode, x, y, 0);
}

// Evaluates the whole tree for row i.  The program is in post-order, so each
// AND/OR reads its children's bits that were set earlier in the sweep.
__device__ __forceinline__ bool eval_pred(const PredProg& p, const ColSet& cs, int64_t i) {
  if (p.n_nodes == 0) return true;
  if (p.n_nodes == 1) return eval_leaf(p, p.nodes[0], cs, i);
  uint32_t bits = 0;
  for (int k = 0; k < p.n_nodes; k++) {
    const ghb_pred_node& nd = p.nodes[k];
    bool r;
    if (nd.mode == GHB_FILTER_AND)
      r = ((bits >> nd.child[0]) & (bits >> nd.child[1]) & 1u) != 0;
    else if (nd.mode == GHB_FILTER_OR)
      r = (((bits >> nd.child[0]) | (bits >> nd.child[1])) & 1u) != 0;
    else
      r = eval_leaf(p, nd, cs, i);
    bits |= (uint32_t)r << k;
  }
  return (bits >> (p.n_nodes - 1)) & 1u;
}

// ----------------------------------------------------------- transforms
// Order-preserving map of a signed value to unsigned (BinarySortable's sign
// flip, BinarySortableSerDe.java:921-935).
__device__ __host__ __forceinline__ uint64_t flip_i64(int64_t v) {
  return (uint64_t)v ^ 0x8000000000000000ull;
}
// IEEE double -> unsigned total order (BinarySortableSerDe.java:954-960).
__device__ __host__ __forceinline__ uint64_t flip_f64_bits(uint64_t b) {
  return (b & 0x8000000000000000ull) ? ~b : (b ^ 0x8000000000000000ull);
}
__device__ __host__ __forceinline__ uint64_t unflip_f64_bits(uint64_t u) {
  return (u & 0x8000000000000000ull) ? (u ^ 0x8000000000000000ull) : ~u;
}

// 64-bit finaliser of MurmurHash3 (Austin Appleby, public domain): a
// bijective mixer, so distinct keys never collide before the mask.
__device__ __host__ __forceinline__ uint64_t mix64(uint64_t k) {
  k ^= k >> 33;
  k *= 0xff51afd7ed558ccdull;
  k ^= k >> 33;
  k *= 0xc4ceb9fe1a85ec53ull;
  k ^= k >> 33;
  return k;
}

// ----------------------------------------------------------- bulk copies
// Bulk global->shared copies through the Tensor Memory Accelerator's
// non-tensor path (cp.async.bulk), completing on an mbarrier that tracks the
// bytes in flight.  Source and destination must be 16-byte aligned and the
// size a multiple of 16.
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
// Makes mbarrier initialisation visible to the async (bulk copy) proxy.
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
// Starts bringing `bytes` of global memory at `src` into L2 (no completion
// to wait for; later loads of the range hit L2).  16-byte aligned address,
// size a multiple of 16.
__device__ __forceinline__ void bulk_prefetch_l2(const void* src, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// As mbar_try_wait, but a thread whose phase is not complete is suspended
// until it completes or about kWaitHintNs pass, instead of returning at once:
// a waiting warp then issues nothing while the copy is in flight.
constexpr uint32_t kWaitHintNs = 20000;
__device__ __forceinline__ bool mbar_try_wait_hint(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity), "r"(kWaitHintNs)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ uint64_t globaltimer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}
// Bounded wait for phase `parity` of `bar`: false (and GHB_ERR_TIMEOUT raised)
// when it did not complete within about one second (or kSpinLimit * 16 polls,
// whichever ends first).
constexpr uint64_t kWaitLimitNs = 1000000000ull;
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int32_t* dev_status) {
  if (mbar_try_wait_hint(bar, parity)) return true;
  const uint64_t t0 = globaltimer_ns();
  for (int i = 0; i < kSpinLimit * 16; i++) {
    if (mbar_try_wait_hint(bar, parity)) return true;
    if (globaltimer_ns() - t0 > kWaitLimitNs) break;
  }
  raise_status(dev_status, kDevTimeout);
  return false;
}
// Orders this thread's generic-proxy shared-memory accesses before later
// async-proxy (bulk copy) writes to the same buffer.
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// ----------------------------------------------------------- look-back
// Tile status word for decoupled look-back (single-pass prefix scan):
//   bits 63..44  epoch (launch tag, so the array is never cleared per launch)
//   bits 43..42  flag: 1 = aggregate of this tile only, 2 = inclusive prefix
//   bits 41..0   count
constexpr int kEpochShift = 44;
constexpr uint64_t kEpochMask = (1ull << 20) - 1;
constexpr uint64_t kFlagAgg = 1ull << 42;
constexpr uint64_t kFlagPrefix = 2ull << 42;
constexpr uint64_t kCountMask = (1ull << 42) - 1;

__device__ __forceinline__ uint64_t lb_pack(uint32_t epoch, uint64_t flag, uint64_t count) {
  return ((uint64_t)(epoch & kEpochMask) << kEpochShift) | flag | (count & kCountMask);
}

__device__ __forceinline__ void lb_store(uint64_t* p, uint64_t v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ uint64_t lb_load(const uint64_t* p) {
  uint64_t v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

// Exclusive prefix of tile `tile` given its own `count`.  Called by one warp
// (all 32 lanes).  Publishes the tile's aggregate, walks back over earlier
// tiles 32 at a time, then publishes the inclusive prefix.  The words carry
// only counts (no tile reads another tile's output), so relaxed stores and
// loads suffice and no fence is needed.  Every wait is bounded: after
// `spin_limit` polls that find an earlier tile not ready it raises
// GHB_ERR_TIMEOUT and returns 0 (the results of that launch are then invalid
// and the host is told; every output position stays below the true one, so
// no write leaves its buffer).
__device__ __forceinline__ uint64_t lookback_exclusive(uint64_t* status_arr, uint32_t epoch,
                                                       int64_t tile, uint64_t count,
                                                       int32_t* dev_status, int spin_limit) {
  const int lane = threadIdx.x & 31;
  if (tile == 0) {
    if (lane == 0) lb_store(&status_arr[0], lb_pack(epoch, kFlagPrefix, count));
    return 0;
  }
  if (lane == 0) lb_store(&status_arr[tile], lb_pack(epoch, kFlagAgg, count));
  uint64_t exclusive = 0;
  int64_t base = tile - 1;  // highest tile index the warp examines this round
  int spins = 0;
  while (true) {
    int64_t t = base - lane;
    uint64_t v = 0;
    bool valid = false;
    if (t >= 0) {
      v = lb_load(&status_arr[t]);
      valid = ((v >> kEpochShift) & kEpochMask) == (epoch & kEpochMask) &&
              (v & (kFlagAgg | kFlagPrefix)) != 0;
    } else {
      valid = true;  // before tile 0: acts as an empty prefix
      v = lb_pack(epoch, kFlagPrefix, 0);
    }
    unsigned not_ready = __ballot_sync(0xffffffffu, !valid);
    if (not_ready) {
      // wait until the lanes up to the first prefix are all ready
      unsigned pref = __ballot_sync(0xffffffffu, valid && (v & kFlagPrefix));
      // lanes below the lowest not-ready lane: if one of them holds a prefix
      // the walk can finish with them alone
      int first_nr = __ffs(not_ready) - 1;
      unsigned below = (first_nr == 0) ? 0u : ((1u << first_nr) - 1u);
      if (!(pref & below)) {
        if (++spins >= spin_limit) {
          if (lane == 0) raise_status(dev_status, kDevTimeout);
          return 0;
        }
        continue;
      }
    }
    unsigned pref = __ballot_sync(0xffffffffu, valid && (v & kFlagPrefix));
    int stop = pref ? (__ffs(pref) - 1) : 32;  // lowest lane (nearest tile) with a prefix
    uint64_t c = (lane <= stop) ? (v & kCountMask) : 0;
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
    c = __shfl_sync(0xffffffffu, c, 0);
    exclusive += c;
    if (pref) break;
    base -= 32;
  }
  if (lane == 0) lb_store(&status_arr[tile], lb_pack(epoch, kFlagPrefix, exclusive + count));
  return exclusive;
}

// Tiles are claimed in launch order from a global counter, so a tile's
// predecessors are always owned by running CTAs and the look-back cannot
// wait on a CTA that never started.  A tile is claimed only when its CTA is
// ready to work on it: a claim held back behind another tile would make
// every later tile's look-back wait for it.
__device__ __forceinline__ void claim_tile(unsigned long long* counter, int64_t* s_cur) {
  if (threadIdx.x == 0) *s_cur = (int64_t)atomicAdd(counter, 1ull);
  __syncthreads();
}

// Called once by every CTA at exit: the last one resets the claim counter
// and the finish counter for the next launch.
__device__ __forceinline__ void claim_finish(unsigned long long* counters) {
  if (threadIdx.x == 0) {
    __threadfence();
    unsigned long long done = atomicAdd(&counters[1], 1ull);
    if (done == gridDim.x - 1) {
      counters[0] = 0;
      counters[1] = 0;
      __threadfence();
    }
  }
}

}  // namespace ghb
