// edk_spmm.cuh — H applied to a block of p right-hand-side vectors at once
// (SpMM), for one or many operators.
//
// EDKit's colmn! (src/Operator.jl:417-465) finds each nonzero's target index
// once and then loops over the RHS columns.  The GPU form keeps that order of
// work: one warp per row, the row's off-diagonal hits located by different
// lanes (canonicalisation and lookup done once per hit), then every hit
// applied to the p vectors with the lanes spread over the vectors.  Blocks are
// row-major (row i, vector c at i * p + c), so each hit reads one contiguous
// p-element row of X: coalesced, and reused from L2 across the rows that
// reach it.  The materialised form reads the sliced-ELL entries instead of
// recomputing them.
#pragma once

#include <algorithm>
#include <cstring>

#include "edk_rows.cuh"

namespace edk {

// One operator of an SpMM batch; operator q's blocks start at q * Dpad * p.
struct SpmmOp {
  BasisDev b;
  OpDev op;
  FFParams ff;
  int64_t D;
  int kind;  // 0: bond-family kernel, 1: materialised kernel, 2: neither
};

namespace spmm_detail {

template <class VT, int VPL>
__device__ __forceinline__ void acc_row(typename VTraits<VT>::A (&ar)[VPL],
                                        typename VTraits<VT>::A (&ai)[VPL],
                                        const VT* __restrict__ xr, int lane, int p, double cr,
                                        double ci) {
  using A = typename VTraits<VT>::A;
  constexpr bool CX = VTraits<VT>::cx;
  const A r = (A)cr, i = (A)ci;
#pragma unroll
  for (int v = 0; v < VPL; ++v) {
    const int c = lane + 32 * v;
    if (c < p) {
      const Cx<A> xv = ldv(xr + c);
      ar[v] += r * xv.r + i * xv.i;  // conj(coefficient) * x
      if constexpr (CX) ai[v] += r * xv.i - i * xv.r;
    }
  }
}

template <class VT, int VPL>
__device__ __forceinline__ void store_row(VT* __restrict__ yr, int lane, int p, int accumulate,
                                          typename VTraits<VT>::A (&ar)[VPL],
                                          typename VTraits<VT>::A (&ai)[VPL]) {
  using A = typename VTraits<VT>::A;
#pragma unroll
  for (int v = 0; v < VPL; ++v) {
    const int c = lane + 32 * v;
    if (c < p) {
      Cx<A> out{ar[v], ai[v]};
      if (accumulate) {
        const Cx<A> yo = ldout(yr + c);
        out.r += yo.r;
        out.i += yo.i;
      }
      stv(yr + c, out);
    }
  }
}

// Apply the nh hits held one per lane (ok, target row, coefficient) to the
// lane's columns, four hits at a time: their row gathers are all issued
// before the multiply-adds, so four rows are in flight per lane.
template <class VT, int VPL>
__device__ __forceinline__ void apply_hits(typename VTraits<VT>::A (&ar)[VPL],
                                           typename VTraits<VT>::A (&ai)[VPL],
                                           const VT* __restrict__ xb, int lane, int p, int nh,
                                           int ok, int64_t pos, double cr, double ci) {
  using A = typename VTraits<VT>::A;
  constexpr bool CX = VTraits<VT>::cx;
  const unsigned full = 0xffffffffu;
  int hh = 0;
  for (; hh + 4 <= nh; hh += 4) {
    int okq[4];
    int64_t pq[4];
    double crq[4], ciq[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      okq[u] = __shfl_sync(full, ok, hh + u);
      pq[u] = __shfl_sync(full, pos, hh + u);
      crq[u] = __shfl_sync(full, cr, hh + u);
      ciq[u] = __shfl_sync(full, ci, hh + u);
    }
    Cx<A> xv[4][VPL];
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int v = 0; v < VPL; ++v) {
        const int c = lane + 32 * v;
        xv[u][v] = (okq[u] && c < p) ? ldv(xb + pq[u] * p + c) : Cx<A>{0, 0};
      }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const A r = (A)crq[u], im = (A)ciq[u];
#pragma unroll
      for (int v = 0; v < VPL; ++v) {
        ar[v] += r * xv[u][v].r + im * xv[u][v].i;  // conj(coefficient) * x
        if constexpr (CX) ai[v] += r * xv[u][v].i - im * xv[u][v].r;
      }
    }
  }
  for (; hh < nh; ++hh) {
    if (!__shfl_sync(full, ok, hh)) continue;
    const int64_t ph = __shfl_sync(full, pos, hh);
    const double crh = __shfl_sync(full, cr, hh), cih = __shfl_sync(full, ci, hh);
    acc_row<VT, VPL>(ar, ai, xb + ph * p, lane, p, crh, cih);
  }
}

}  // namespace spmm_detail

template <int BK, class VT, int VPL>
__global__ void __launch_bounds__(256) k_spmm_ff(const SpmmOp* __restrict__ ops, int nops,
                                                 int64_t Dpad, int p,
                                                 const VT* __restrict__ X, VT* __restrict__ Y,
                                                 int accumulate) {
  using A = typename VTraits<VT>::A;
  __shared__ uint32_t s_binom[(BK == BK_PROJ_RANK) ? 32 * 33 : 1];
  if constexpr (BK == BK_PROJ_RANK) {
    fill_binom32(s_binom);
    __syncthreads();
  }
  const int lane = threadIdx.x & 31;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int64_t total = (int64_t)nops * Dpad;
  for (int64_t g = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; g < total; g += nw) {
    const int q = (int)(g / Dpad);
    const int64_t i = g - (int64_t)q * Dpad;
    const SpmmOp& o = ops[q];
    if (o.kind != 0 || i >= o.D) continue;  // warp-uniform
    const BasisDev& b = o.b;
    const FFParams& ff = o.ff;
    const uint32_t mask = (uint32_t)b.maskL;
    const uint32_t st = (BK == BK_TENSOR) ? (uint32_t)i : (uint32_t)__ldg(b.I + i);
    const double invRi = b.R ? 1.0 / __ldg(b.R + i) : 1.0;
    uint32_t hm[kMaxFF];
    int cnt[kMaxFF];
    int nhit = 0;
    double dr = 0.0, di = 0.0;
    for (int f = 0; f < ff.nfam; ++f) {
      const uint32_t Xb = st, Yb = rotl_L(st, ff.d[f], b.L, mask), V = ff.valid[f];
      const uint32_t m1 = ~Xb & Yb & V, m2 = Xb & ~Yb & V;
      const int c0 = __popc(~Xb & ~Yb & V), c1 = __popc(m1), c2 = __popc(m2),
                c3 = __popc(Xb & Yb & V);
      dr += ff.dval[f][0].x * c0 + ff.dval[f][1].x * c1 + ff.dval[f][2].x * c2 +
            ff.dval[f][3].x * c3;
      di += ff.dval[f][0].y * c0 + ff.dval[f][1].y * c1 + ff.dval[f][2].y * c2 +
            ff.dval[f][3].y * c3;
      hm[f] = m1 | m2;
      cnt[f] = __popc(hm[f]);
      nhit += cnt[f];
    }
    for (int t = 0; t < o.op.nterm; ++t) {  // diagonal-only terms
      const TermDev* T = o.op.term + t;
      int c = 0;
      for (int k = 0; k < T->nsites; ++k) c = (c << 1) | (int)((st >> T->bitpos[k]) & 1u);
      const double2 dv = __ldg(o.op.dval + T->diag_off + c);
      dr += dv.x;
      di += dv.y;
    }
    const VT* xb = X + (int64_t)q * Dpad * p;
    A ar[VPL], ai[VPL];
#pragma unroll
    for (int v = 0; v < VPL; ++v) ar[v] = ai[v] = 0;
    spmm_detail::acc_row<VT, VPL>(ar, ai, xb + i * p, lane, p, dr, di);  // conj(diag) x_i
    for (int base = 0; base < nhit; base += 32) {
      const int l = base + lane;
      int ok = 0;
      int64_t pos = 0;
      double cr = 0.0, ci = 0.0;
      if (l < nhit) {
        int f = 0, r = l;
        while (r >= cnt[f]) { r -= cnt[f]; ++f; }
        uint32_t m = hm[f];
        for (int k = 0; k < r; ++k) m &= m - 1;
        const int pb = __ffs(m) - 1;
        const int d = ff.d[f];
        const int qb = pb >= d ? pb - d : pb - d + b.L;
        HitCtx h;
        canon_ctx<BK>(b, st ^ (1u << pb) ^ (1u << qb), h);
        int64_t p1, p2;
        double r1, r2;
        bool ok1, ok2;
        locate2<BK>(b, s_binom, h.key, h.key, false, p1, r1, ok1, p2, r2, ok2);
        if (ok1) {
          const double2 w = ((st >> pb) & 1u) ? ff.v2[f] : ff.v1[f];
          const double ratio = r1 * invRi;
          cr = (w.x * h.pre - w.y * h.pim) * ratio;
          ci = (w.x * h.pim + w.y * h.pre) * ratio;
          pos = p1;
          ok = 1;
        }
      }
      const int nh = min(32, nhit - base);
      spmm_detail::apply_hits<VT, VPL>(ar, ai, xb, lane, p, nh, ok, pos, cr, ci);
    }
    spmm_detail::store_row<VT, VPL>(Y + (int64_t)q * Dpad * p + i * p, lane, p, accumulate, ar,
                                    ai);
  }
}

// materialised operators: one warp per sliced-ELL slot (= one row)
template <class VT, int VPL>
__global__ void __launch_bounds__(256) k_spmm_sell(const SpmmOp* __restrict__ ops, int nops,
                                                   int64_t smax, int64_t Dpad, int p,
                                                   const VT* __restrict__ X, VT* __restrict__ Y,
                                                   int accumulate) {
  using A = typename VTraits<VT>::A;
  const int lane = threadIdx.x & 31;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int64_t total = (int64_t)nops * smax;
  for (int64_t g = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; g < total; g += nw) {
    const int q = (int)(g / smax);
    const int64_t s = g - (int64_t)q * smax;
    const SpmmOp& o = ops[q];
    const SellDev& sd = o.op.sell;
    if (o.kind != 1 || s >= sd.nslices * 32) continue;
    const unsigned rc = __ldg(sd.rowid + s);
    if (rc == ~0u) continue;
    const int64_t row = rc & ((1u << sd.rbits) - 1u);
    const double invR = __ldg(sd.rinv + (rc >> sd.rbits));
    const int64_t slice = s >> 5;
    const int w = __ldg(sd.width + slice);
    const int64_t base = __ldg(sd.off + slice) + (s & 31);
    const double2 d = sd.diagc ? __ldg(sd.diagc + s) : make_double2(__ldg(sd.diag + s), 0.0);
    const VT* xb = X + (int64_t)q * Dpad * p;
    A ar[VPL], ai[VPL];
#pragma unroll
    for (int v = 0; v < VPL; ++v) ar[v] = ai[v] = 0;
    spmm_detail::acc_row<VT, VPL>(ar, ai, xb + row * p, lane, p, d.x, d.y);
    for (int kb = 0; kb < w; kb += 32) {
      const int k = kb + lane;
      int col = 0;
      double cr = 0.0, ci = 0.0;
      if (k < w && sd.val) {  // value mode: explicit coefficients, already divided by R[row]
        col = __ldg(sd.col + base + (int64_t)k * 32);
        const double2 v = __ldg(sd.val + base + (int64_t)k * 32);
        cr = v.x;
        ci = v.y;
      } else if (k < w) {
        int code;
        if (sd.packed) {
          const unsigned e =
              __ldg(reinterpret_cast<const unsigned*>(sd.col) + base + (int64_t)k * 32);
          col = (int)(e >> sd.packed);
          code = (int)(e & ((1u << sd.packed) - 1u));
        } else {
          col = __ldg(sd.col + base + (int64_t)k * 32);
          code = __ldg(sd.code + base + (int64_t)k * 32);
        }
        const double2 v = __ldg(sd.vt64 + code);
        cr = v.x * invR;
        ci = v.y * invR;
      }
      const int nh = min(32, w - kb);
      // padding entries carry a zero coefficient: applying them adds nothing
      spmm_detail::apply_hits<VT, VPL>(ar, ai, xb, lane, p, nh, 1, (int64_t)col, cr, ci);
    }
    spmm_detail::store_row<VT, VPL>(Y + (int64_t)q * Dpad * p + row * p, lane, p, accumulate,
                                    ar, ai);
  }
}

// Launch the SpMM for every operator of kind 0 (bond-family, lookup kind bk)
// and kind 1 (materialised, up to smax slots) of the batch; operators of kind
// 2 are left to the caller.  p <= 64.
template <class VT>
edk_status launch_spmm(const SpmmOp* d_ops, int nops, int bk_ff, int64_t smax, int64_t Dpad,
                       int p, const VT* X, VT* Y, int accumulate, cudaStream_t st) {
  const bool two = p > 32;
  if (bk_ff >= 0) {
    const int64_t nw = (int64_t)nops * Dpad;
    const int grid = (int)std::min<int64_t>((nw + 7) / 8, 148 * 64);
#define EDK_SPMM_FF(BK)                                                                          \
  case BK:                                                                                       \
    if (two) k_spmm_ff<BK, VT, 2><<<grid, 256, 0, st>>>(d_ops, nops, Dpad, p, X, Y, accumulate); \
    else k_spmm_ff<BK, VT, 1><<<grid, 256, 0, st>>>(d_ops, nops, Dpad, p, X, Y, accumulate);    \
    break;
    switch (bk_ff) {
      EDK_SPMM_FF(BK_TENSOR)
      EDK_SPMM_FF(BK_PROJ_RANK)
      EDK_SPMM_FF(BK_PROJ_HASH)
      EDK_SPMM_FF(BK_TRANS)
      EDK_SPMM_FF(BK_TRANSPAR)
      default:
        set_error("SpMM: unsupported basis kind for the bond-family kernel");
        return EDK_UNSUPPORTED;
    }
#undef EDK_SPMM_FF
    EDK_TRY_CUDA(cudaGetLastError());
  }
  if (smax > 0) {
    const int64_t nw = (int64_t)nops * smax;
    const int grid = (int)std::min<int64_t>((nw + 7) / 8, 148 * 64);
    if (two)
      k_spmm_sell<VT, 2><<<grid, 256, 0, st>>>(d_ops, nops, smax, Dpad, p, X, Y, accumulate);
    else
      k_spmm_sell<VT, 1><<<grid, 256, 0, st>>>(d_ops, nops, smax, Dpad, p, X, Y, accumulate);
    EDK_TRY_CUDA(cudaGetLastError());
  }
  return EDK_OK;
}

// Fill the SpMM description of one operator; returns its kind and, through
// bk / slots, the lookup kind of the bond-family kernel (translation sectors
// with and without phases share BK_TRANS) and its materialised slot count.
inline int spmm_describe(const edk_operator* op, SpmmOp& h, int& bk, int64_t& slots) {
  std::memset(&h, 0, sizeof(SpmmOp));
  h.b = op->b->dev;
  h.op = op->dev;
  h.D = op->b->D;
  bk = -1;
  slots = 0;
  if (op->sell_ok) {
    h.kind = 1;
    slots = op->dev.sell.nslices * 32;
  } else if (op->ff_ok && op->use_ff && op->b->dev.L <= 32) {
    h.kind = 0;
    std::memcpy(&h.ff, op->ff_params.data(), sizeof(FFParams));
    bk = op->b->dev.bk == BK_TRANS0 ? BK_TRANS : op->b->dev.bk;
    h.b.bk = bk;
  } else {
    h.kind = 2;
  }
  return h.kind;
}

}  // namespace edk
