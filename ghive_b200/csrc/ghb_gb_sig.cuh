// ghb_gb_sig.cuh — group-by folds specialised for one operator signature.
//
// fold_tile (ghb_groupby.cuh) interprets, for every row, the predicate
// program, the key column's type and NULL convention and each accumulator's
// kind and column type.  The signature of a call (the used columns' types and
// NULL modes, the predicate tree's shape, the key column and the accumulator
// plan) is fixed for the whole launch, so a kernel compiled for it carries
// none of those branches.  A signature is a type built from the templates
// below, e.g.
//
//   SigFolder<2, 0, true, ColT<0, GHB_INT, GHB_NULLS_NONE>,
//             PLeaf<0, GHB_FILTER_LT, ColT<3, GHB_INT, GHB_NULLS_NONE>, false>,
//             AccT<A_CNT_STAR, NoCol>, AccT<A_SUM_I, ColT<1, GHB_LONG, GHB_NULLS_NONE>>, ...>
//
// The literals stay run-time values (read from the predicate nodes in the
// kernel parameters), so one compiled kernel serves every literal.  The
// library writes the type for a call and compiles it with NVRTC
// (ghb_jit.cu); this header is compiled by NVRTC as well as nvcc.
#pragma once

#include "ghb_groupby.cuh"

namespace ghb {

// A used column: position, type and NULL convention fixed.
template <int COL, int TYPE, int NULLS>
struct ColT {
  static constexpr int col = COL;
  static constexpr int type = TYPE;
  __device__ __forceinline__ static int64_t raw(const GbParams& p, const unsigned char* stage, int r) {
    const unsigned char* b = stage + p.col_off[COL];
    if constexpr (TYPE == GHB_INT) return (int64_t)((const int32_t*)b)[r];
    else return ((const long long*)b)[r];
  }
  __device__ __forceinline__ static bool null(const GbParams& p, const unsigned char* stage, int r,
                                              int64_t v) {
    if constexpr (NULLS == GHB_NULLS_NONE) {
      return false;
    } else if constexpr (NULLS == GHB_NULLS_BYTEMAP) {
      return stage[p.null_off[COL] + r] != 0;
    } else if constexpr (TYPE == GHB_INT) {
      return v == (int64_t)INT32_MAX;
    } else if constexpr (TYPE == GHB_LONG) {
      return v == INT64_MAX;
    } else {
      double d = __longlong_as_double(v);
      return d != d;
    }
  }
};

struct NoCol {
  static constexpr int col = -1;
  static constexpr int type = GHB_LONG;
};

// ---------------------------------------------------------------- predicates
struct PTrue {
  __device__ __forceinline__ static bool eval(const GbParams&, const unsigned char*, int) { return true; }
};

// Column vs literal(s) of predicate node NODE; LITD: the literals are doubles.
template <int NODE, int MODE, class C, bool LITD>
struct PLeaf {
  __device__ __forceinline__ static bool eval(const GbParams& p, const unsigned char* stage, int r) {
    const int64_t x = C::raw(p, stage, r);
    if (C::null(p, stage, r, x)) return false;
    if constexpr (MODE == GHB_FILTER_NOT_NULL) {
      return true;
    } else {
      const ghb_pred_node& nd = p.pred.nodes[NODE];
      if constexpr (C::type == GHB_DOUBLE || LITD) {
        const double a = LITD ? nd.lit_d[0] : (double)nd.lit_i[0];
        const double b = LITD ? nd.lit_d[1] : (double)nd.lit_i[1];
        return cmp_mode<double>(MODE, raw_to_f64(C::type, x), a, b);
      } else {
        return cmp_mode<int64_t>(MODE, x, nd.lit_i[0], nd.lit_i[1]);
      }
    }
  }
};

// Column vs column.
template <int MODE, class C, class C2>
struct PCols {
  __device__ __forceinline__ static bool eval(const GbParams& p, const unsigned char* stage, int r) {
    const int64_t x = C::raw(p, stage, r);
    if (C::null(p, stage, r, x)) return false;
    const int64_t y = C2::raw(p, stage, r);
    if (C2::null(p, stage, r, y)) return false;
    if constexpr (C::type == GHB_DOUBLE || C2::type == GHB_DOUBLE)
      return cmp_mode<double>(MODE, raw_to_f64(C::type, x), raw_to_f64(C2::type, y), 0.0);
    else
      return cmp_mode<int64_t>(MODE, x, y, 0);
  }
};

template <class A, class B>
struct PAnd {
  __device__ __forceinline__ static bool eval(const GbParams& p, const unsigned char* stage, int r) {
    return A::eval(p, stage, r) && B::eval(p, stage, r);
  }
};

template <class A, class B>
struct POr {
  __device__ __forceinline__ static bool eval(const GbParams& p, const unsigned char* stage, int r) {
    return A::eval(p, stage, r) || B::eval(p, stage, r);
  }
};

// ---------------------------------------------------------------- accumulators
// How an accumulator is kept in the shared table.  The global table keeps
// every accumulator as one 64-bit word; a CTA's shared table uses the
// narrowest form whose shared atomics are fast (a B200 SM retires about six
// 32-bit shared atomics for each 64-bit one):
//   R_CNT    u32 count (the kernel flushes the table before a count can wrap)
//   R_PAIR   64-bit wrapping sum as a u32 low word and a u32 high word: the
//            low add returns the old word, a carry out goes to the high word
//   R_F64    double (sum, or its compensation word)
//   R_IMG32  u32 order image of an INT value (MAX; MIN stores its complement)
//   R_IMG64  u64 order image (MAX; MIN stores its complement)
enum AccRep : int { R_CNT = 0, R_PAIR = 1, R_F64 = 2, R_IMG32 = 3, R_IMG64 = 4 };

// One accumulator: kind fixed, input column fixed (NoCol for COUNT(*)).
template <int KIND, class C>
struct AccT {
  static constexpr int kind = KIND;
  static constexpr int rep = (KIND == A_CNT_STAR || KIND == A_CNT_NN) ? R_CNT
                             : KIND == A_SUM_I                         ? R_PAIR
                             : (KIND == A_SUM_F || KIND == A_COMP_F)   ? R_F64
                             : C::type == GHB_INT                      ? R_IMG32
                                                                       : R_IMG64;
  static constexpr int words = (rep == R_CNT || rep == R_IMG32) ? 1 : 2;   // u32 words per slot

  // The row's contribution as a global-table word (0 = none).
  __device__ __forceinline__ static uint64_t contrib(const GbParams& p, const unsigned char* stage, int r) {
    if constexpr (KIND == A_CNT_STAR) {
      return 1;
    } else if constexpr (KIND == A_COMP_F) {
      return 0;
    } else {
      const int64_t v = C::raw(p, stage, r);
      if (C::null(p, stage, r, v)) return 0;
      if constexpr (KIND == A_CNT_NN) return 1;
      else if constexpr (KIND == A_SUM_I) return (uint64_t)v;
      else if constexpr (KIND == A_SUM_F) return (uint64_t)__double_as_longlong(raw_to_f64(C::type, v));
      else if constexpr (KIND == A_MAX_O) return order_image(C::type, v);
      else return ~order_image(C::type, v);   // A_MIN_O
    }
  }

  // The row's contribution in the shared table's form (0 = none): a count,
  // a sum, double bits, or an order image (u32 for R_IMG32, complemented for
  // MIN).  A u32 image of 0 adds nothing to a maximum, which is what the
  // value it stands for (INT32_MIN for MAX, INT32_MAX for MIN) would add.
  __device__ __forceinline__ static uint64_t narrow(const GbParams& p, const unsigned char* stage, int r) {
    if constexpr (rep == R_IMG32) {
      const int64_t v = C::raw(p, stage, r);
      if (C::null(p, stage, r, v)) return 0;
      const uint32_t u = (uint32_t)(int32_t)v ^ 0x80000000u;
      return KIND == A_MAX_O ? u : (uint32_t)~u;
    } else {
      return contrib(p, stage, r);
    }
  }
};

// u32 image of an INT order value back to the global table's 64-bit image.
__device__ __forceinline__ uint64_t img32_to_64(uint32_t u) {
  return flip_i64((int64_t)(int32_t)(u ^ 0x80000000u));
}

template <bool B, class T, class F>
struct TypeIf {
  using type = T;
};
template <class T, class F>
struct TypeIf<false, T, F> {
  using type = F;
};

// Slot of a key image in the specialised folds' shared table of mask + 1
// slots: the low bits of the image folded to 32 bits and xor-shifted, so keys
// of a dense integer range (the common GROUP BY key) land in distinct slots,
// and keys that differ only in high bits still spread.
__device__ __forceinline__ int sslot(uint64_t u, int mask) {
  uint32_t x = (uint32_t)u ^ (uint32_t)(u >> 32);
  return (int)((x ^ (x >> 16)) & (uint32_t)mask);
}

// Find-or-insert of a non-zero key image (u32 or u64 words) in the shared
// table by linear probing from sslot; the slot, or -1 after max_probe probes.
template <class W>
__device__ __forceinline__ int sinsert(W* keys, int mask, W u, int max_probe) {
  int h = sslot((uint64_t)u, mask);
  for (int q = 0; q < max_probe; q++) {
    const W cur = keys[h];
    if (cur == u) return h;
    if (cur == 0) {
      const W prev = atomicCAS(keys + h, (W)0, u);
      if (prev == 0 || prev == u) return h;
    }
    h = (h + 1) & mask;
  }
  return -1;
}

// 64-bit wrapping add into a (low, high) pair of u32 words.
__device__ __forceinline__ void pair_add(uint32_t* lo, uint32_t* hi, uint64_t w) {
  const uint32_t l = (uint32_t)w;
  uint32_t h = (uint32_t)(w >> 32);
  if (l) {
    const uint32_t old = atomicAdd(lo, l);
    h += (old + l < old) ? 1u : 0u;
  }
  if (h) atomicAdd(hi, h);
}

// Error-free sum of (s, c) pairs across the lanes of a warp.
__device__ __forceinline__ void warp_sum_f64(double& s, double& c) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double so = __shfl_xor_sync(0xffffffffu, s, o);
    const double co = __shfl_xor_sync(0xffffffffu, c, o);
    const double t = __dadd_rn(s, so);
    c = __dadd_rn(__dadd_rn(c, co), two_sum_err(s, so, t));
    s = t;
  }
}

__device__ __forceinline__ uint64_t warp_sum_u64(uint64_t v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ uint64_t warp_max_u64(uint64_t v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = max(v, (uint64_t)__shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Folds one tile for one operator signature.  ROWS is the tile's rows per
// thread; WAGG selects combining equal keys within a warp before the shared
// atomics (few groups): 0 never, 1 always, 2 as p.warp_agg says (a batch whose
// instances differ in it).  Phase A: per row,
// predicate, key, slot (shared table, else global).  Phase B: per
// accumulator, each shared row's contribution in its narrow form.  Phase C
// (rare, skipped by a warp with no such row): rows whose key is not in the
// shared table merge every accumulator into their global record.  The shared
// table (S slots + the two side slots) is laid out as arrays: keys (u32 for an
// INT key column, else u64), then each accumulator's words in plan order.
template <int ROWS, int WAGG, bool KEYED, class KEY, class PRED, class... ACCS>
struct SigFolder {
  static_assert(ROWS >= 1 && ROWS <= kGbRows, "rows per thread");
  static constexpr bool kNarrow = true;
  static constexpr bool k32 = KEYED && KEY::type == GHB_INT;
  static constexpr int kKeyWords = k32 ? 1 : 2;
  static constexpr int kN = sizeof...(ACCS);
  static constexpr int kWords[kN] = {ACCS::words...};
  static constexpr int kKinds[kN] = {ACCS::kind...};
  static_assert(kKinds[0] == A_CNT_STAR, "accumulator 0 is COUNT(*)");

  // u32 word offset of accumulator I's array, in units of the slot stride.
  template <int I>
  __host__ __device__ static constexpr int off() {
    int s = kKeyWords;
    for (int k = 0; k < I; k++) s += kWords[k];
    return s;
  }
  static constexpr int kTableWords = off<kN>();   // u32 words per slot

  // A global aggregate keeps each thread's partial aggregates in registers
  // for the whole launch (sums, counts, extremes in the shared table's
  // narrow form; a double sum with its compensation word) and merges them
  // once, in drain, instead of reducing every row slot across the warp.
  struct Empty {};
  struct Partials {
    uint64_t w[kN];
  };
  using State = typename TypeIf<KEYED, Empty, Partials>::type;

  template <int... I>
  struct Seq {};
  template <int N, int... I>
  struct MakeSeq : MakeSeq<N - 1, N - 1, I...> {};
  template <int... I>
  struct MakeSeq<0, I...> {
    using type = Seq<I...>;
  };
  using Accs = typename MakeSeq<kN>::type;

  // Narrow update of shared slot s with a contribution w in the narrow form
  // (an SUM_F update also takes the compensation word wc).
  template <int I, class ACC>
  __device__ __forceinline__ static void shared_merge(uint32_t* tab, int sstride, int s, uint64_t w,
                                                      uint64_t wc) {
    uint32_t* a = tab + off<I>() * sstride;
    if constexpr (ACC::rep == R_CNT) {
      if (w) atomicAdd(a + s, (uint32_t)w);
    } else if constexpr (ACC::rep == R_PAIR) {
      pair_add(a + s, a + sstride + s, w);
    } else if constexpr (ACC::kind == A_SUM_F) {
      acc_merge(A_SUM_F, (uint64_t*)a + s, sstride, w, wc);
    } else if constexpr (ACC::rep == R_IMG32) {
      if (w) atomicMax(a + s, (uint32_t)w);
    } else if constexpr (ACC::rep == R_IMG64) {
      if (w) atomicMax((unsigned long long*)a + s, (unsigned long long)w);
    }
  }

  template <int I, class ACC>
  __device__ __forceinline__ static void acc_pass(const GbParams& p, const unsigned char* stage, const int* slot,
                                                  const bool* ins, const unsigned* peers, uint32_t* tab,
                                                  int sstride, uint64_t* wstage, State& st) {
    constexpr int kind = ACC::kind;
    if constexpr (kind == A_COMP_F) {
      return;
    } else {
#pragma unroll
      for (int j = 0; j < ROWS; j++) {
        const int r = j * blockDim.x + threadIdx.x;
        if constexpr (!KEYED) {
          // every live row is in the one group: into this thread's partials
          if (ins[j]) {
            if constexpr (kind == A_SUM_F) {
              const double x = __longlong_as_double(ACC::contrib(p, stage, r));
              const double s0 = __longlong_as_double(st.w[I]);
              const double t = __dadd_rn(s0, x);
              st.w[I + 1] = (uint64_t)__double_as_longlong(
                  __dadd_rn(__longlong_as_double(st.w[I + 1]), two_sum_err(s0, x, t)));
              st.w[I] = (uint64_t)__double_as_longlong(t);
            } else if constexpr (kind == A_MAX_O || kind == A_MIN_O) {
              st.w[I] = max(st.w[I], ACC::narrow(p, stage, r));
            } else {
              st.w[I] += ACC::contrib(p, stage, r);
            }
          }
        } else if (WAGG == 1 || (WAGG == 2 && p.warp_agg)) {
          // lanes of one shared slot combine first; the lowest applies it
          wstage[threadIdx.x & 31] = ins[j] ? ACC::narrow(p, stage, r) : 0;
          __syncwarp();
          if (ins[j] && (threadIdx.x & 31) == __ffs(peers[j]) - 1) {
            uint64_t tot = 0, comp = 0;
            double sf = 0.0, cf = 0.0;
            for (unsigned m = peers[j]; m; m &= m - 1) {
              const uint64_t x = wstage[__ffs(m) - 1];
              if constexpr (kind == A_SUM_F) {
                const double xv = __longlong_as_double(x);
                const double tt = __dadd_rn(sf, xv);
                cf = __dadd_rn(cf, two_sum_err(sf, xv, tt));
                sf = tt;
              } else if constexpr (kind == A_MAX_O || kind == A_MIN_O) {
                tot = max(tot, x);
              } else {
                tot += x;
              }
            }
            if constexpr (kind == A_SUM_F) {
              tot = (uint64_t)__double_as_longlong(sf);
              comp = (uint64_t)__double_as_longlong(cf);
            }
            shared_merge<I, ACC>(tab, sstride, slot[j], tot, comp);
          }
          __syncwarp();
        } else {
          if (ins[j]) shared_merge<I, ACC>(tab, sstride, slot[j], ACC::narrow(p, stage, r), 0);
        }
      }
    }
  }

  template <int... I>
  __device__ __forceinline__ static void all_accs(Seq<I...>, const GbParams& p, const unsigned char* stage,
                                                  const int* slot, const bool* ins, const unsigned* peers,
                                                  uint32_t* tab, int sstride, uint64_t* wstage, State& st) {
    (acc_pass<I, ACCS>(p, stage, slot, ins, peers, tab, sstride, wstage, st), ...);
  }

  // One accumulator of a global aggregate's partials: reduced across the
  // warp, merged by lane 0 into the one group's shared slot (or its global
  // record when there is no shared table), then cleared.
  template <int I, class ACC>
  __device__ __forceinline__ static void drain_one(const GbParams& p, uint32_t* tab, int sstride, State& st) {
    constexpr int kind = ACC::kind;
    if constexpr (!KEYED && kind != A_COMP_F) {
      uint64_t tot = 0, comp = 0;
      if constexpr (kind == A_SUM_F) {
        double sf = __longlong_as_double(st.w[I]), cf = __longlong_as_double(st.w[I + 1]);
        warp_sum_f64(sf, cf);
        tot = (uint64_t)__double_as_longlong(sf);
        comp = (uint64_t)__double_as_longlong(cf);
        st.w[I + 1] = 0;
      } else if constexpr (kind == A_MAX_O || kind == A_MIN_O) {
        tot = warp_max_u64(st.w[I]);
      } else {
        tot = warp_sum_u64(st.w[I]);
      }
      st.w[I] = 0;
      if ((threadIdx.x & 31) == 0) {
        const int S = p.smem_slots;
        if (S > 0) {
          shared_merge<I, ACC>(tab, sstride, S + 1, tot, comp);
        } else {
          // global record: extremes in the wide form (an untouched u32 word is
          // the neutral value, harmless to merge, as in flush)
          uint64_t w = tot;
          if constexpr (ACC::rep == R_IMG32) {
            const uint64_t img = img32_to_64(kind == A_MAX_O ? (uint32_t)tot : ~(uint32_t)tot);
            w = kind == A_MAX_O ? img : ~img;
          }
          acc_merge(kind, p.grec + (p.C + 1) * p.R + 1 + I, 1, w, comp);
        }
      }
    }
  }

  template <int... I>
  __device__ __forceinline__ static void drain_all(Seq<I...>, const GbParams& p, uint32_t* tab, int sstride,
                                                   State& st) {
    (drain_one<I, ACCS>(p, tab, sstride, st), ...);
  }

  // Merges this thread's partials (a global aggregate's) into the table; all
  // threads, before the barrier that precedes the flush.
  __device__ __forceinline__ static void drain(const GbParams& p, uint64_t* skeys, State& st) {
    if constexpr (!KEYED) drain_all(Accs{}, p, (uint32_t*)skeys, p.smem_slots + 2, st);
  }

  // Every accumulator of row r into global record g.
  template <int... I>
  __device__ __forceinline__ static void global_row(Seq<I...>, const GbParams& p, const unsigned char* stage,
                                                    int r, int64_t g) {
    uint64_t* rec = p.grec + g * p.R + 1;
    (acc_merge(ACCS::kind, rec + I, 1, ACCS::contrib(p, stage, r), 0), ...);
  }

  using KW = typename TypeIf<k32, uint32_t, unsigned long long>::type;

  // The key image of a non-NULL raw key: u32 for an INT key column (0 is
  // INT32_MIN), else flip_i64 (0 is INT64_MIN).
  __device__ __forceinline__ static KW image(int64_t raw) {
    if constexpr (k32) return (uint32_t)(int32_t)raw ^ 0x80000000u;
    else return (unsigned long long)flip_i64(raw);
  }

  __device__ __forceinline__ static void fold(const GbParams& p, const unsigned char* stage, int rows,
                                              uint64_t* skeys, uint64_t* wstage, State& st) {
    const int S = p.smem_slots;
    const int sstride = S + 2;
    uint32_t* tab = (uint32_t*)skeys;
    KW* keys = (KW*)skeys;
    const int mask = S - 1;
    int slot[ROWS];       // shared slot
    int64_t gslot[ROWS];  // global record of a live row without a shared slot
    bool ins[ROWS];       // live and in the shared table
    unsigned peers[ROWS];
    bool need[ROWS];      // live, and not found by the fast probe
    bool any_need = false, glob = false;
    // Phase A1: predicate, and a branch-free probe of the key's first two
    // slots (a key already in the table is there in almost every row).
#pragma unroll
    for (int j = 0; j < ROWS; j++) {
      const int r = j * blockDim.x + threadIdx.x;
      const bool lv = r < rows && PRED::eval(p, stage, r);
      int sl = -1;
      bool hit = false;
      if constexpr (KEYED) {
        const int64_t raw = KEY::raw(p, stage, r);
        const KW u = image(raw);
        if (S > 0) {
          const int h0 = sslot((uint64_t)u, mask), h1 = (h0 + 1) & mask;
          const KW c0 = keys[h0], c1 = keys[h1];
          hit = u != 0 && (c0 == u || c1 == u) && !KEY::null(p, stage, r, raw);
          sl = c0 == u ? h0 : h1;
        }
      } else {
        hit = S > 0;
        sl = S + 1;   // a global aggregate: the one group
      }
      slot[j] = sl;
      gslot[j] = -1;
      ins[j] = lv && hit;
      need[j] = lv && !hit;
      any_need |= need[j];
    }
    // Phase A2 (rows the fast probe missed): NULL key, INT64_MIN, a key new
    // to this CTA or further along its probe chain, or no room.
    if (__any_sync(0xffffffffu, any_need)) {
#pragma unroll
      for (int j = 0; j < ROWS; j++) {
        if (!need[j]) continue;
        const int r = j * blockDim.x + threadIdx.x;
        int sl = -1;
        int64_t g = -1;
        int side = -1;   // 0: key INT64_MIN, 1: NULL key / global aggregate
        if constexpr (KEYED) {
          const int64_t raw = KEY::raw(p, stage, r);
          if (KEY::null(p, stage, r, raw)) {
            side = 1;
          } else {
            const KW u = image(raw);
            if (u == 0 && !k32) {
              side = 0;
            } else {
              if (u != 0 && S > 0) sl = sinsert<KW>(keys, mask, u, 4);
              if (sl < 0) g = gtable_insert(p, flip_i64(raw));   // INT32_MIN keys too
            }
          }
        } else {
          side = 1;
        }
        if (side >= 0) {
          if (S > 0) sl = S + side;
          else g = p.C + side;
        }
        if (sl < 0 && g < 0) raise_status(p.status, kDevCapacity);   // the row is dropped
        slot[j] = sl;
        gslot[j] = g;
        ins[j] = sl >= 0;
        glob |= g >= 0;
      }
    }
#pragma unroll
    for (int j = 0; j < ROWS; j++) {
      peers[j] = 0;
      if (KEYED && (WAGG == 1 || (WAGG == 2 && p.warp_agg)))
        peers[j] = __match_any_sync(0xffffffffu, ins[j] ? slot[j] : -1);
    }
    all_accs(Accs{}, p, stage, slot, ins, peers, tab, sstride, wstage, st);
    if (__any_sync(0xffffffffu, glob)) {
#pragma unroll
      for (int j = 0; j < ROWS; j++)
        if (gslot[j] >= 0) global_row(Accs{}, p, stage, j * blockDim.x + threadIdx.x, gslot[j]);
    }
  }

  // The shared table of p fits the words the launch reserved.
  __device__ __forceinline__ static bool fits(const GbParams& p) {
    return (int64_t)(p.smem_slots + 2) * kTableWords <= 2 * (int64_t)p.table_words &&
           p.tile_rows == ROWS * (int)blockDim.x;
  }

  // Zeroes the shared table (all threads; the caller syncs after).
  __device__ __forceinline__ static void clear(const GbParams& p, uint64_t* skeys) {
    const int64_t words = (int64_t)(p.smem_slots + 2) * kTableWords / 2;
    for (int64_t i = threadIdx.x; i < words; i += blockDim.x) skeys[i] = 0;
  }

  template <int I, class ACC>
  __device__ __forceinline__ static void flush_one(const uint32_t* tab, int sstride, int s, uint64_t* rec) {
    const uint32_t* a = tab + off<I>() * sstride;
    if constexpr (ACC::rep == R_CNT) {
      if (a[s]) atomicAdd((unsigned long long*)rec, (unsigned long long)a[s]);
    } else if constexpr (ACC::rep == R_PAIR) {
      const uint64_t v = ((uint64_t)a[sstride + s] << 32) | a[s];
      if (v) atomicAdd((unsigned long long*)rec, (unsigned long long)v);
    } else if constexpr (ACC::kind == A_SUM_F) {
      acc_merge(A_SUM_F, rec, 1, ((const uint64_t*)a)[s], ((const uint64_t*)a)[sstride + s]);
    } else if constexpr (ACC::rep == R_IMG32) {
      // an untouched word stands for the value that leaves the extreme as it is
      const uint64_t img = img32_to_64(ACC::kind == A_MAX_O ? a[s] : ~a[s]);
      atomicMax((unsigned long long*)rec, (unsigned long long)(ACC::kind == A_MAX_O ? img : ~img));
    } else if constexpr (ACC::rep == R_IMG64) {
      const uint64_t v = ((const uint64_t*)a)[s];
      if (v) atomicMax((unsigned long long*)rec, (unsigned long long)v);
    }
  }

  template <int... I>
  __device__ __forceinline__ static void flush_all(Seq<I...>, const uint32_t* tab, int sstride, int s,
                                                   uint64_t* rec) {
    (flush_one<I, ACCS>(tab, sstride, s, rec + I), ...);
  }

  // Merges the shared table into the global one (all threads; the caller
  // syncs before and after).
  __device__ __forceinline__ static void flush(const GbParams& p, const uint64_t* skeys) {
    const int S = p.smem_slots;
    if (S == 0) return;
    const int sstride = S + 2;
    const uint32_t* tab = (const uint32_t*)skeys;
    const uint32_t* cnt = tab + off<0>() * sstride;
    for (int s = threadIdx.x; s < sstride; s += blockDim.x) {
      if (cnt[s] == 0) continue;
      int64_t g;
      if (s < S) {
        const uint64_t u = k32 ? flip_i64((int64_t)(int32_t)(tab[s] ^ 0x80000000u)) : ((const uint64_t*)tab)[s];
        g = gtable_insert(p, u);
        if (g < 0) {
          raise_status(p.status, kDevCapacity);
          continue;
        }
      } else {
        g = p.C + (s - S);
      }
      flush_all(Accs{}, tab, sstride, s, p.grec + g * p.R + 1);
    }
  }
};

}  // namespace ghb
