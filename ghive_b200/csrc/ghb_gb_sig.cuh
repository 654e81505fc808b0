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
//   SigFolder<true, ColT<0, GHB_INT, GHB_NULLS_NONE>,
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
// One accumulator word: kind fixed, input column fixed (NoCol for COUNT(*)).
template <int KIND, class C>
struct AccT {
  static constexpr int kind = KIND;
  // The row's contribution (0 = none).
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
};

// Folds one tile: phase A finds each row's slot as fold_tile does, phase B
// adds each accumulator's contribution with its kind known at compile time.
template <bool KEYED, class KEY, class PRED, class... ACCS>
struct SigFolder {
  template <int A, class ACC>
  __device__ __forceinline__ static void acc_pass(const GbParams& p, const unsigned char* stage, int rpt,
                                                  const int64_t* slot, const bool* live, const bool* in_s,
                                                  const unsigned* peers, uint64_t* sacc, int64_t sstride,
                                                  uint64_t* wstage) {
    constexpr int kind = ACC::kind;
    if constexpr (kind == A_COMP_F) {
      return;
    } else {
#pragma unroll
      for (int j = 0; j < kGbRows; j++) {
        if (j >= rpt) continue;
        const int r = j * blockDim.x + threadIdx.x;
        const uint64_t w = live[j] ? ACC::contrib(p, stage, r) : 0;
        if (p.warp_agg) {
          wstage[threadIdx.x & 31] = in_s[j] ? w : 0;
          __syncwarp();
          if (in_s[j] && (threadIdx.x & 31) == __ffs(peers[j]) - 1) {
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
            acc_merge(kind, sacc + A * sstride + slot[j], sstride, tot, comp);
          }
          __syncwarp();
          if (live[j] && !in_s[j]) acc_merge(kind, p.grec + slot[j] * p.R + 1 + A, 1, w, 0);
        } else if (live[j]) {
          if (in_s[j]) acc_merge(kind, sacc + A * sstride + slot[j], sstride, w, 0);
          else acc_merge(kind, p.grec + slot[j] * p.R + 1 + A, 1, w, 0);
        }
      }
    }
  }

  template <int... I>
  struct Seq {};
  template <int N, int... I>
  struct MakeSeq : MakeSeq<N - 1, N - 1, I...> {};
  template <int... I>
  struct MakeSeq<0, I...> {
    using type = Seq<I...>;
  };

  template <int... I>
  __device__ __forceinline__ static void all_accs(Seq<I...>, const GbParams& p, const unsigned char* stage,
                                                  int rpt, const int64_t* slot, const bool* live,
                                                  const bool* in_s, const unsigned* peers, uint64_t* sacc,
                                                  int64_t sstride, uint64_t* wstage) {
    (acc_pass<I, ACCS>(p, stage, rpt, slot, live, in_s, peers, sacc, sstride, wstage), ...);
  }

  __device__ __forceinline__ static void fold(const GbParams& p, const unsigned char* stage, int rows,
                                              uint64_t* skeys, uint64_t* wstage) {
    const int S = p.smem_slots;
    const int64_t sstride = S + 2;
    uint64_t* sacc = skeys + sstride;
    const int smask_shift = S > 0 ? 64 - __ffs(S) + 1 : 0;
    const int rpt = p.tile_rows / (int)blockDim.x;
    int64_t slot[kGbRows];
    bool live[kGbRows], in_s[kGbRows];
    unsigned peers[kGbRows];
#pragma unroll
    for (int j = 0; j < kGbRows; j++) {
      live[j] = in_s[j] = false;
      slot[j] = -1;
      peers[j] = 0;
      if (j >= rpt) continue;
      const int r = j * blockDim.x + threadIdx.x;
      bool lv = r < rows && PRED::eval(p, stage, r);
      uint64_t u = 0;
      int side = -1;
      if (lv) {
        if constexpr (KEYED) {
          const int64_t raw = KEY::raw(p, stage, r);
          if (KEY::null(p, stage, r, raw)) {
            side = 1;
          } else {
            u = flip_i64(raw);
            if (u == 0) side = 0;
          }
        } else {
          side = 1;
        }
      }
      int64_t ss = -1;
      if (lv && S > 0) ss = side >= 0 ? S + side : smem_insert(skeys, S - 1, smask_shift, u, 8);
      if (lv && ss < 0) {
        const int64_t g = side >= 0 ? p.C + side : gtable_insert(p, u);
        if (g < 0) {
          raise_status(p.status, kDevCapacity);
          lv = false;
        }
        slot[j] = g;
      } else {
        slot[j] = ss;
      }
      live[j] = lv;
      in_s[j] = lv && ss >= 0;
      if (p.warp_agg) peers[j] = __match_any_sync(0xffffffffu, in_s[j] ? ss : -1);
    }
    all_accs(typename MakeSeq<sizeof...(ACCS)>::type{}, p, stage, rpt, slot, live, in_s, peers, sacc, sstride,
             wstage);
  }
};

}  // namespace ghb
