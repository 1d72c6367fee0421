// edk_rankrows.cuh — the row-plan form of the flip-flop fast path for sectors
// whose target rows follow from colex ranks: translation (and translation +
// parity) sectors searched through their rank table, and complete
// fixed-charge sectors (ProjectedBasis without a predicate), where a state's
// row is its colex rank.
//
// The per-row work of the reference's colmn! (src/Operator.jl:417-465) with
// index() (TranslationalBasis.jl:310-341, TranslationalParityBasis.jl:192-234,
// ProjectedBasis.jl:52-81) becomes, for every exchange hit of a row state s:
//   rank(s') = rank(s) +- C(a, j)      (a, a+1 the exchanged sites, j set bits below a)
//   entry    = rankmap[rank(s')]       (row << shift | M << 5 | norm class)
//   y[row]  += conj(w C[M] R[t] / R[row]) x[t]
// through the row body the tile kernels use (ff_row_sum), so both give
// bit-identical H*x.
//
// What the plan removes from every product: the per-block sort of the rows by
// hit count (done once when the plan is built: rows are ordered inside each
// 256-row window, so the 32 lanes of a warp walk equally long hit lists), the
// per-row reads of the 8-byte state and the 8-byte norm (one 16-byte slot of
// state, rank, row word and wrap-around rank instead), and the walk over the
// set bits for the wrap-around bond.
#pragma once

#include <type_traits>

#include "edk_rows.cuh"

namespace edk {

// Resident blocks per SM asked of the compiler: the plan kernels are latency
// bound, so real vectors are held to 32 registers (all 64 warp slots of an SM
// filled), single-precision complex to 40 (48 warps), double complex to 64
// (32 warps).
template <int BK, class VT>
constexpr int plan_min_blocks() {
  return std::is_same<VT, double2>::value ? 4 : (std::is_same<VT, float2>::value ? 6 : 8);
}

// The operator is one nearest-neighbour bond family with equal exchange
// values (the plan kernels then compile only that loop: NN = 1; else NN = 2).
__host__ __device__ inline bool plan_nn(const FFParams& ff) {
  return ff.nfam == 1 && ff.d[0] == 1 && ff.same[0];
}

// One slot of the plan.  BK is BK_TRANS0_RANK, BK_TRANS_RANK,
// BK_TRANSPAR_RANK (rank table) or BK_PROJ_RANK (row = rank); `t` holds the
// block's tables (ff_tab_fill with the plan's binomials).
template <int BK, class VT, int NN = 0>
__device__ __forceinline__ void plan_row(const BasisDev& b, const OpDev& op, const FFParams& ff,
                                         const FFTab<BK>& t, int64_t slot,
                                         const VT* __restrict__ xk, VT* __restrict__ yk,
                                         int accumulate) {
  using A = typename VTraits<VT>::A;
  const RowPlanDev& pl = op.plan;
  const uint4 e = __ldg(pl.slot + slot);
  const uint32_t rw = e.x;
  if (rw == ~0u) return;
  const uint32_t st = e.y, rs = e.z, rkw = e.w;
  const int64_t i = (int64_t)(rw & kPlanRowMask);
  // 1 / R of the row, rounded as the tile form rounds it (coef[c].x = R_c)
  const A invRi = BK == BK_PROJ_RANK ? (A)1 : (A)(1.0 / t.coef[rw >> 27].x);
  const Cx<A> Y = ff_row_sum<BK, VT, 1, NN>(b, ff, t, st, rs, rkw, 0, xk);
  double dr = 0.0, di = 0.0;
  if (pl.dg) {
    dr = __ldg(pl.dg + slot);  // the same sums, taken when the plan was built
  } else {
    const uint32_t mask = (uint32_t)b.maskL;
    for (int f = 0; f < ff.nfam; ++f)
      ff_diag(ff, f, st, rotl_L(st, ff.d[f], b.L, mask), ff.valid[f], dr, di);
    term_diag(op, st, dr, di);
  }
  ff_row_store<VT>(Y, invRi, dr, di, xk, yk, i, accumulate);
}

}  // namespace edk
