// edk_batch.cu — Lanczos over many independent operators in lockstep
// (momentum sectors of one chain, disorder instances), and the single-operator
// ground state as a batch of one.
//
// Every kernel of a step covers all operators of the batch in one launch: a
// block owns a tile of one operator's rows (tile2op map) or, in the
// reorthogonalisation kernels, an equal share of all rows (RowSplit), reads
// that operator's basis/term descriptors from a device array, and works on
// its slice of the concatenated buffers.  The step index j, the recurrence
// coefficients alpha/beta, 1/beta and the per-operator stop flags live on the
// device, so a step has no host round trip: it is captured once into a CUDA
// graph and replayed.  The host looks at alpha/beta only every check_every
// steps (tridiagonal eigenvalues, convergence).  One step per operator q:
//   wt_q = H_q v_j                       (row-gather matvec)
//   s = V_q^H wt_q ; alpha_j = Re s_j     (CGS sweep 1, FP64 block partials)
//   w_q = wt_q - V_q s ; u = V_q^H w_q    (one pass: k_rupdate_dots)
//   w_q -= V_q u ; beta_j = ||w_q||       (sweep 2 + norm)
//   lucky breakdown beta <= sqrt(eps) max(1, |alpha|) stops operator q
//   v_{j+1} = w_q / beta_j
// (classical Gram-Schmidt twice, as _lanczos_build! in
// src/algorithms/TimeEvolution.jl:250-306, with its three-term recurrence
// folded into the first sweep).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstring>
#include <map>
#include <memory>
#include <vector>

#include "edk_rankrows.cuh"

namespace edk {

namespace {

constexpr int kTile = 256;          // rows per matvec / update tile
constexpr int kSplitBlocks = 4;         // resident reorthogonalisation blocks per SM (register cap)

template <class T> struct IsCx;
template <> struct IsCx<double> { static constexpr bool v = false; };
template <> struct IsCx<double2> { static constexpr bool v = true; };
template <> struct IsCx<float> { static constexpr bool v = false; };
template <> struct IsCx<float2> { static constexpr bool v = true; };

__device__ __forceinline__ double2 l2(const double* p) { return make_double2(*p, 0.0); }
__device__ __forceinline__ double2 l2(const double2* p) { return *p; }
__device__ __forceinline__ double2 l2(const float* p) { return make_double2((double)*p, 0.0); }
__device__ __forceinline__ double2 l2(const float2* p) {
  float2 v = *p;
  return make_double2((double)v.x, (double)v.y);
}
__device__ __forceinline__ void s2(double* p, double2 v) { *p = v.x; }
__device__ __forceinline__ void s2(double2* p, double2 v) { *p = v; }
__device__ __forceinline__ void s2(float* p, double2 v) { *p = (float)v.x; }
__device__ __forceinline__ void s2(float2* p, double2 v) { *p = make_float2((float)v.x, (float)v.y); }

__device__ __forceinline__ double wsum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

}  // namespace

// One operator of a batch, as the kernels see it.
struct __align__(16) BOp {
  BasisDev b;
  OpDev op;
  FFParams ff;
  int64_t D;
  int64_t voff;   // element offset of V_q (D x ncap, column-major)
  int64_t woff;   // element offset into w / wt
  int64_t tile0;  // first matvec tile
  int64_t sblk0;  // first block of the materialised-matrix product (8 slices each)
  int ntile;
};

// ---------------------------------------------------------------------------
// kernels (j = *step; operators with done[q] != 0 are skipped)
// ---------------------------------------------------------------------------
template <int BK, class VT>
__global__ void __launch_bounds__(256) k_bapply_ff(const BOp* __restrict__ ops,
                                                   const int* __restrict__ tile2op,
                                                   const VT* __restrict__ V, VT* __restrict__ wt,
                                                   const int* __restrict__ step,
                                                   const int* __restrict__ done) {
  const int q = tile2op[blockIdx.x];
  if (done[q]) return;
  const BOp& o = ops[q];
  const int j = *step;
  ff_tile<BK, VT>(o.b, o.op, o.ff, (blockIdx.x - o.tile0) * (int64_t)kTile,
                  V + o.voff + (int64_t)j * o.D, wt + o.woff, 0);
}

// the row-plan form of k_bapply_ff (rank-searched sectors whose operators all
// carry a plan): tile t of operator q is window t of q's plan
template <int BK, class VT, int NN>
__global__ void __launch_bounds__(256, plan_min_blocks<BK, VT>()) k_bapply_plan(const BOp* __restrict__ ops,
                                                     const int* __restrict__ tile2op,
                                                     int64_t ntiles,
                                                     const VT* __restrict__ V, VT* __restrict__ wt,
                                                     const int* __restrict__ step,
                                                     const int* __restrict__ done) {
  // a resident grid walks the tiles; the operator record and its tables are
  // loaded into shared memory again only when the operator changes
  __shared__ FFTab<BK> sm;
  __shared__ __align__(16) BOp s_op;  // the operator record, read from shared memory
  const int j = *step;
  int cur = -1;
  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int q = tile2op[tile];
    if (done[q]) continue;
    if (q != cur) {
      __syncthreads();  // the previous operator's rows no longer read the tables
      const int4* src = reinterpret_cast<const int4*>(ops + q);
      int4* dst = reinterpret_cast<int4*>(&s_op);
      for (int e = threadIdx.x; e < (int)(sizeof(BOp) / sizeof(int4)); e += blockDim.x) dst[e] = src[e];
      __syncthreads();
      ff_tab_fill<BK>(sm, s_op.b, s_op.op.plan.binom);
      __syncthreads();
      cur = q;
    }
    const BOp& o = s_op;
    plan_row<BK, VT, NN>(o.b, o.op, o.ff, sm, (tile - o.tile0) * (int64_t)kTile + threadIdx.x,
                         V + o.voff + (int64_t)j * o.D, wt + o.woff, 0);
  }
}

template <class VT>
__global__ void __launch_bounds__(256) k_bapply_sell(const BOp* __restrict__ ops,
                                                     const int* __restrict__ sblk2op,
                                                     const VT* __restrict__ V, VT* __restrict__ wt,
                                                     const int* __restrict__ step,
                                                     const int* __restrict__ done) {
  const int q = sblk2op[blockIdx.x];
  if (done[q]) return;
  const BOp& o = ops[q];
  const int64_t slice = (blockIdx.x - o.sblk0) * 8 + (threadIdx.x >> 5);
  if (slice >= o.op.sell.nslices) return;
  const int j = *step;
  sell_slice<VT>(o.b, o.op.sell, slice, threadIdx.x & 31, V + o.voff + (int64_t)j * o.D,
                 wt + o.woff, 0);
}

template <int BK, class VT>
__global__ void __launch_bounds__(256) k_bapply_gen(const BOp* __restrict__ ops,
                                                    const int* __restrict__ tile2op,
                                                    const VT* __restrict__ V,
                                                    VT* __restrict__ wt,
                                                    const int* __restrict__ step,
                                                    const int* __restrict__ done) {
  __shared__ uint32_t s_binom[32 * 33];
  if constexpr (BK == BK_PROJ_RANK) {
    fill_binom32(s_binom);
    __syncthreads();
  }
  const int q = tile2op[blockIdx.x];
  if (done[q]) return;
  const BOp& o = ops[q];
  const int64_t i = (blockIdx.x - o.tile0) * (int64_t)kTile + threadIdx.x;
  if (i >= o.D) return;
  const int j = *step;
  gen_row<BK, uint32_t, VT, true>(o.b, o.op, i, V + o.voff + (int64_t)j * o.D, wt + o.woff, 0,
                                  s_binom);
}

// Sum of eight values over a warp, one value index per lane group: three
// halving exchanges (offsets 16, 8, 4: a lane keeps half of its values and
// adds its partner's copy of that half) then two butterfly steps.  Nine
// shuffles for eight sums instead of forty; lane l ends with the total of
// value (l >> 2) & 7.
__device__ __forceinline__ double wsum8(const double (&a)[8], int lane) {
  double b[4], c[2];
  const bool h16 = lane & 16, h8 = lane & 8, h4 = lane & 4;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const double send = h16 ? a[i] : a[i + 4];
    b[i] = (h16 ? a[i + 4] : a[i]) + __shfl_xor_sync(0xffffffffu, send, 16);
  }
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    const double send = h8 ? b[i] : b[i + 2];
    c[i] = (h8 ? b[i + 2] : b[i]) + __shfl_xor_sync(0xffffffffu, send, 8);
  }
  double d = (h4 ? c[1] : c[0]) + __shfl_xor_sync(0xffffffffu, h4 ? c[0] : c[1], 4);
  d += __shfl_xor_sync(0xffffffffu, d, 2);
  d += __shfl_xor_sync(0xffffffffu, d, 1);
  return d;
}

// ---------------------------------------------------------------------------
// Reorthogonalisation kernels.  Their grid is G blocks that are all resident
// at once (G = SMs x blocks per SM), and block b owns rows
// [b T / G, (b + 1) T / G) of the concatenated rows of the operators still
// running (T rows in all, recomputed by k_bsplit at the start of every step):
// every block streams the same number of bytes, so no partly filled last
// wave of blocks holds the launch up and operators that have stopped leave
// no block idle.  A block whose rows run from one operator into the next
// handles each piece in turn; its slot among operator q's partial sums is
// b - bfirst_q (nslot_q slots in all).
// ---------------------------------------------------------------------------
struct SplitOp {
  int64_t off;    // first row among the running operators' rows
  int64_t pofs;   // offset of the dot-product partial sums (ncols x nslot)
  int64_t slot0;  // first norm partial sum
  int bfirst, nslot;
};

struct RowSplit {
  const SplitOp* sp;
  const int64_t* TG;  // rows of the running operators, blocks that share them
  int nops;
};

// exclusive prefix sum over the block (blockDim.x a multiple of 32, at most
// 1024); *total gets the sum
__device__ int64_t block_scan(int64_t v, int64_t* s_warp, int64_t* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  int64_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int64_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) s_warp[warp] = x;
  __syncthreads();
  if (warp == 0) {
    int64_t t = lane < nw ? s_warp[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int64_t y = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) t += y;
    }
    if (lane < nw) s_warp[lane] = t;  // inclusive over warps
  }
  __syncthreads();
  const int64_t before = (warp > 0 ? s_warp[warp - 1] : 0) + x - v;
  *total = s_warp[nw - 1];
  __syncthreads();
  return before;
}

// the block holding row r: the largest b with b T / G <= r
__device__ __forceinline__ int split_owner(int64_t r, int64_t T, int G) {
  int64_t b = r * G / T;
  while (b + 1 < G && (b + 1) * T / G <= r) ++b;
  while (b > 0 && b * T / G > r) --b;
  return (int)b;
}

// The running operators' row offsets, blocks and partial-sum slots, by one
// whole block.  The grid's first G' = min(G, ceil(T / 128)) blocks share the
// rows, so each has at least one and every slot of an operator is written.
// The stop flags are read past L1: in k_bfinish other blocks have just set
// them.
__device__ void split_rows_dev(const BOp* __restrict__ ops, int nops, int Gmax, int ncap,
                               const int* done, SplitOp* __restrict__ sp,
                               int64_t* __restrict__ TG) {
  __shared__ int64_t s_warp[32];
  const int per = (nops + (int)blockDim.x - 1) / (int)blockDim.x;
  const int q0 = min(nops, (int)threadIdx.x * per), q1 = min(nops, q0 + per);
  int64_t loc = 0;
  for (int q = q0; q < q1; ++q) loc += __ldcg(done + q) ? 0 : ops[q].D;
  int64_t T = 0;
  int64_t off = block_scan(loc, s_warp, &T);
  const int G = (int)max((int64_t)1, min((int64_t)Gmax, (T + 127) / 128));
  int64_t nsl = 0;
  for (int q = q0; q < q1; ++q) {
    const int64_t d = __ldcg(done + q) ? 0 : ops[q].D;
    SplitOp o;
    o.off = off;
    o.pofs = 0;
    o.slot0 = 0;
    if (d > 0) {
      o.bfirst = split_owner(off, T, G);
      o.nslot = split_owner(off + d - 1, T, G) - o.bfirst + 1;
    } else {
      o.bfirst = 0;
      o.nslot = 0;
    }
    sp[q] = o;
    nsl += o.nslot;
    off += d;
  }
  int64_t nslot_all = 0;
  int64_t s0 = block_scan(nsl, s_warp, &nslot_all);
  for (int q = q0; q < q1; ++q) {
    sp[q].slot0 = s0;
    sp[q].pofs = s0 * ncap;
    s0 += sp[q].nslot;
  }
  if (threadIdx.x == 0) {
    TG[0] = T;
    TG[1] = G;
  }
}

// the split before the first step (one block of 1024 threads); later steps
// get theirs from the last block of k_bfinish
__global__ void __launch_bounds__(1024) k_bsplit(const BOp* __restrict__ ops, int nops, int Gmax,
                                                 int ncap, const int* __restrict__ done,
                                                 SplitOp* __restrict__ sp, int64_t* __restrict__ TG) {
  split_rows_dev(ops, nops, Gmax, ncap, done, sp, TG);
}

template <class F>
__device__ __forceinline__ void for_block_rows(const BOp* __restrict__ ops, RowSplit rs, F&& f) {
  const int64_t T = rs.TG[0], G = rs.TG[1];
  if ((int64_t)blockIdx.x >= G) return;
  const int64_t gb = (int64_t)blockIdx.x * T / G;
  const int64_t ge = (int64_t)(blockIdx.x + 1) * T / G;
  if (gb >= ge) return;
  int lo = 0, hi = rs.nops - 1;  // the last operator starting at or before gb
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (rs.sp[mid].off <= gb) lo = mid;
    else hi = mid - 1;
  }
  for (int q = lo; q < rs.nops; ++q) {
    const SplitOp& s = rs.sp[q];
    if (s.off >= ge) break;
    if (s.nslot == 0) continue;  // stopped
    const BOp& o = ops[q];
    const int64_t a = max(gb, s.off), b = min(ge, s.off + o.D);
    if (a < b) f(q, o, a - s.off, b - s.off, (int)blockIdx.x - s.bfirst, s);
  }
}

// Rows per thread and pass of the reorthogonalisation kernels: a pass loads
// U columns (8 real, 4 complex) of R rows in one go, 128 bytes a thread.
template <class VV>
constexpr int pass_rows() {
  return 128 / ((IsCx<VV>::v ? 4 : 8) * (int)sizeof(VV));
}

// One pass of k_rdots: a += conj(V[rows, cols]) w[rows] for the U columns
// at Vc[u] and the R rows rb + 256 k (all in range when FULL).
template <bool FULL, int U, int R, bool CX, class VV, class WV>
__device__ __forceinline__ void dots_pass(const VV* const (&Vc)[U], const WV* __restrict__ wq,
                                          int64_t rb, int64_t r1, double (&a)[8]) {
  double2 wv[R], v[U][R];
#pragma unroll
  for (int k = 0; k < R; ++k) {
    const int64_t r = rb + (int64_t)k * 256;
    wv[k] = (FULL || r < r1) ? l2(wq + r) : make_double2(0.0, 0.0);
  }
#pragma unroll
  for (int u = 0; u < U; ++u)
#pragma unroll
    for (int k = 0; k < R; ++k) {
      const int64_t r = rb + (int64_t)k * 256;
      v[u][k] = (FULL || r < r1) ? l2(Vc[u] + r) : make_double2(0.0, 0.0);
    }
#pragma unroll
  for (int u = 0; u < U; ++u)
#pragma unroll
    for (int k = 0; k < R; ++k) {
      if constexpr (CX) {
        a[2 * u] += v[u][k].x * wv[k].x + v[u][k].y * wv[k].y;
        a[2 * u + 1] += v[u][k].x * wv[k].y - v[u][k].y * wv[k].x;
      } else {
        a[u] += v[u][k].x * wv[k].x;
      }
    }
}

// part[pofs_q + c * nslot_q + slot] = sum over the block's rows r of
// conj(V_q[r, c]) w_q[r], c <= j.  Columns go eight real (four complex)
// values at a time through one wsum8 after the thread has summed its rows;
// the columns of a last, partial group read the segment's last column again
// (their sums are not kept).  The per-warp sums of 64 columns at a time are
// added across warps in shared memory.
template <class VV, class WV>
__global__ void __launch_bounds__(256, kSplitBlocks) k_rdots(const BOp* __restrict__ ops, RowSplit rs,
                                               const VV* __restrict__ V,
                                               const WV* __restrict__ w,
                                               double2* __restrict__ part,
                                               const int* __restrict__ step,
                                               const int* __restrict__ done) {
  constexpr bool CX = IsCx<VV>::v || IsCx<WV>::v;
  constexpr int U = CX ? 4 : 8;  // columns per reduction
  constexpr int SEG = 64;        // columns per shared-memory flush
  constexpr int R = pass_rows<VV>();
  __shared__ double s_part[8][SEG][2];
  const int ncols = *step + 1;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for_block_rows(ops, rs, [&](int q, const BOp& o, int64_t r0, int64_t r1, int slot, const SplitOp& sq) {
    if (done[q]) return;
    const int64_t D = o.D;
    const VV* Vq = V + o.voff;
    const WV* wq = w + o.woff;
    for (int s0 = 0; s0 < ncols; s0 += SEG) {
      const int s1 = min(ncols, s0 + SEG);
      for (int c = s0; c < s1; c += U) {
        const VV* Vc[U];
#pragma unroll
        for (int u = 0; u < U; ++u) Vc[u] = Vq + (int64_t)min(c + u, s1 - 1) * D;
        double a[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) a[u] = 0.0;
        int64_t rb = r0 + threadIdx.x;
        for (; rb + (int64_t)(R - 1) * 256 < r1; rb += 256 * R)
          dots_pass<true, U, R, CX>(Vc, wq, rb, r1, a);
        if (rb < r1) dots_pass<false, U, R, CX>(Vc, wq, rb, r1, a);
        const double t = wsum8(a, lane);
        if ((lane & 3) == 0) {
          const int vi = lane >> 2;
          const int col = CX ? c + (vi >> 1) : c + vi;
          if (col < s1) s_part[warp][col - s0][CX ? (vi & 1) : 0] = t;
        }
      }
      __syncthreads();
      for (int c = threadIdx.x; c < s1 - s0; c += blockDim.x) {
        double sr = 0.0, si = 0.0;
#pragma unroll
        for (int ww = 0; ww < 8; ++ww) {
          sr += s_part[ww][c][0];
          if (CX) si += s_part[ww][c][1];
        }
        part[sq.pofs + (int64_t)(s0 + c) * sq.nslot + slot] = make_double2(sr, si);
      }
      __syncthreads();
    }
  });
}

// coef[q * ncap + c] = sum of operator q's slots: block (x, q) sums columns
// 8x .. 8x + 7 of operator q, one warp per column
__global__ void __launch_bounds__(256) k_breduce(const SplitOp* __restrict__ sp, int ncap,
                                                 const double2* __restrict__ part,
                                                 double2* __restrict__ coef,
                                                 const int* __restrict__ step,
                                                 const int* __restrict__ done) {
  const int q = blockIdx.y;
  const int c = blockIdx.x * 8 + (threadIdx.x >> 5);
  if (done[q] || c > *step) return;
  const int lane = threadIdx.x & 31;
  const SplitOp& o = sp[q];
  const double2* pc = part + o.pofs + (int64_t)c * o.nslot;
  // four independent loads in flight a lane (a large operator has hundreds
  // of slots and only j + 1 columns, so few warps carry the whole reduction)
  double2 a[4] = {make_double2(0.0, 0.0), make_double2(0.0, 0.0), make_double2(0.0, 0.0),
                  make_double2(0.0, 0.0)};
  int k = lane;
  for (; k + 96 < o.nslot; k += 128) {
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const double2 v = pc[k + 32 * u];
      a[u].x += v.x;
      a[u].y += v.y;
    }
  }
  for (; k < o.nslot; k += 32) {
    const double2 v = pc[k];
    a[0].x += v.x;
    a[0].y += v.y;
  }
  double sr = (a[0].x + a[1].x) + (a[2].x + a[3].x);
  double si = (a[0].y + a[1].y) + (a[2].y + a[3].y);
  sr = wsum(sr);
  si = wsum(si);
  if (lane == 0) coef[(int64_t)q * ncap + c] = make_double2(sr, si);
}

// acc[k] -= V[rows, cols] coef[cols] for the U columns at Vc[u] (coefficient
// zero past the last column) and the R rows rb + 256 k (all in range when
// FULL).
template <bool FULL, int U, int R, bool CX, class VV>
__device__ __forceinline__ void update_pass(const VV* const (&Vc)[U], const double2* kc,
                                            int64_t rb, int64_t r1, double2 (&acc)[R]) {
  double2 v[U][R];
#pragma unroll
  for (int u = 0; u < U; ++u)
#pragma unroll
    for (int k = 0; k < R; ++k) {
      const int64_t r = rb + (int64_t)k * 256;
      v[u][k] = (FULL || r < r1) ? l2(Vc[u] + r) : make_double2(0.0, 0.0);
    }
#pragma unroll
  for (int u = 0; u < U; ++u) {
    const double2 cu = kc[u];
#pragma unroll
    for (int k = 0; k < R; ++k) {
      acc[k].x -= v[u][k].x * cu.x;
      if (CX) {
        acc[k].x += v[u][k].y * cu.y;
        acc[k].y -= v[u][k].x * cu.y + v[u][k].y * cu.x;
      }
    }
  }
}

// wout_q = win_q - V_q[:, 0:ncols] coef_q over the block's rows;
// normpart[slot0_q + slot] = sum |wout|^2 over them.  ncols = *step + 1 (or 0
// with zero_cols).  Columns go U at a time (the coefficients are padded with
// zeros to a multiple of U, the missing columns read the last one again).
template <class VV, class WI, class WO>
__global__ void __launch_bounds__(256, kSplitBlocks) k_rupdate(const BOp* __restrict__ ops, RowSplit rs,
                                                 int ncap, const VV* __restrict__ V,
                                                 const double2* __restrict__ coef,
                                                 const WI* __restrict__ win, WO* __restrict__ wout,
                                                 double* __restrict__ normpart,
                                                 const int* __restrict__ step,
                                                 const int* __restrict__ done, int zero_cols) {
  extern __shared__ double2 s_coef[];  // ncap + 8
  __shared__ double s_n[8];
  constexpr bool CX = IsCx<VV>::v || IsCx<WI>::v;
  constexpr int U = CX ? 4 : 8;
  constexpr int R = pass_rows<VV>();
  const int ncols = zero_cols ? 0 : *step + 1;
  const int npad = (ncols + U - 1) / U * U;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for_block_rows(ops, rs, [&](int q, const BOp& o, int64_t r0, int64_t r1, int slot, const SplitOp& sq) {
    if (done[q]) return;
    __syncthreads();  // the previous piece's coefficients and norms are read
    for (int c = threadIdx.x; c < npad; c += blockDim.x)
      s_coef[c] = c < ncols ? coef[(int64_t)q * ncap + c] : make_double2(0.0, 0.0);
    __syncthreads();
    const int64_t D = o.D;
    const VV* Vq = V + o.voff;
    double nrm = 0.0;
    for (int64_t rb = r0 + threadIdx.x; rb < r1; rb += 256 * R) {
      const bool full = rb + (int64_t)(R - 1) * 256 < r1;
      double2 acc[R];
#pragma unroll
      for (int k = 0; k < R; ++k) {
        const int64_t r = rb + (int64_t)k * 256;
        acc[k] = r < r1 ? l2(win + o.woff + r) : make_double2(0.0, 0.0);
      }
      for (int c = 0; c < npad; c += U) {
        const VV* Vc[U];
#pragma unroll
        for (int u = 0; u < U; ++u) Vc[u] = Vq + (int64_t)min(c + u, ncols - 1) * D;
        if (full) update_pass<true, U, R, CX>(Vc, s_coef + c, rb, r1, acc);
        else update_pass<false, U, R, CX>(Vc, s_coef + c, rb, r1, acc);
      }
#pragma unroll
      for (int k = 0; k < R; ++k) {
        const int64_t r = rb + (int64_t)k * 256;
        if (r < r1) {
          s2(wout + o.woff + r, acc[k]);
          nrm += acc[k].x * acc[k].x + (CX ? acc[k].y * acc[k].y : 0.0);
        }
      }
    }
    if (normpart) {
      nrm = wsum(nrm);
      if (lane == 0) s_n[warp] = nrm;
      __syncthreads();
      if (threadIdx.x == 0) {
        double t = 0.0;
        for (int k = 0; k < 8; ++k) t += s_n[k];
        normpart[sq.slot0 + slot] = t;
      }
    }
  });
}

// The first sweep's update and the second sweep's dot products in one pass,
// 256 rows at a time.  Update: one thread per row, wout = win - V coef over
// all columns; the result (as stored) goes to shared memory.  Dot products:
// one warp per column (warps take every eighth column, newest first, so the
// columns the update read last, the most likely to be still in L2, are read
// again first), each lane over eight of the 256 rows, one warp reduction per
// column; the sums build up per column in shared memory and go to
// part[pofs_q + c * nslot_q + slot] at the end of the piece.
// Shared memory: ncap + 8 coefficients and ncap column sums (double2).
template <class VV, class WI, class WO>
__global__ void __launch_bounds__(256, kSplitBlocks) k_rupdate_dots(const BOp* __restrict__ ops, RowSplit rs,
                                                      int ncap, const VV* __restrict__ V,
                                                      const double2* __restrict__ coef,
                                                      const WI* __restrict__ win,
                                                      WO* __restrict__ wout,
                                                      double2* __restrict__ part,
                                                      const int* __restrict__ step,
                                                      const int* __restrict__ done) {
  extern __shared__ double2 s_dyn[];
  double2* s_coef = s_dyn;
  double2* s_acc = s_dyn + ncap + 8;
  __shared__ double2 s_w[256];
  constexpr bool CX = IsCx<VV>::v || IsCx<WI>::v || IsCx<WO>::v;
  constexpr int U = CX ? 4 : 8;
  const int ncols = *step + 1;
  const int npad = (ncols + U - 1) / U * U;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for_block_rows(ops, rs, [&](int q, const BOp& o, int64_t r0, int64_t r1, int slot, const SplitOp& sq) {
    if (done[q]) return;
    __syncthreads();  // the previous piece's column sums are written out
    for (int c = threadIdx.x; c < npad; c += blockDim.x)
      s_coef[c] = c < ncols ? coef[(int64_t)q * ncap + c] : make_double2(0.0, 0.0);
    for (int c = threadIdx.x; c < ncols; c += blockDim.x) s_acc[c] = make_double2(0.0, 0.0);
    __syncthreads();
    const int64_t D = o.D;
    const VV* Vq = V + o.voff;
    for (int64_t rb = r0; rb < r1; rb += 256) {
      const int64_t r = rb + threadIdx.x;
      const int nrow = (int)min((int64_t)256, r1 - rb);
      double2 acc[1] = {make_double2(0.0, 0.0)};
      if (r < r1) {
        acc[0] = l2(win + o.woff + r);
        for (int c = 0; c < npad; c += U) {
          const VV* Vc[U];
#pragma unroll
          for (int u = 0; u < U; ++u) Vc[u] = Vq + (int64_t)min(c + u, ncols - 1) * D;
          update_pass<true, U, 1, CX>(Vc, s_coef + c, r, r + 1, acc);
        }
        WO t;
        s2(&t, acc[0]);
        wout[o.woff + r] = t;
        acc[0] = l2(&t);  // the dot products see the stored value
      }
      s_w[threadIdx.x] = acc[0];
      __syncthreads();
      // two columns (c and c - 8) per pass: sixteen loads in flight a lane
      for (int c = ncols - 1 - warp; c >= 0; c -= 16) {
        const int c2 = c >= 8 ? c - 8 : c;
        const VV* Va = Vq + (int64_t)c * D + rb;
        const VV* Vb = Vq + (int64_t)c2 * D + rb;
        double ar = 0.0, ai = 0.0, br = 0.0, bi = 0.0;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          const int i = lane + 32 * k;
          if (i < nrow) {
            const double2 va = l2(Va + i), vb = l2(Vb + i), x = s_w[i];
            ar += va.x * x.x + va.y * x.y;
            br += vb.x * x.x + vb.y * x.y;
            if (CX) {
              ai += va.x * x.y - va.y * x.x;
              bi += vb.x * x.y - vb.y * x.x;
            }
          }
        }
        ar = wsum(ar);
        br = wsum(br);
        if (CX) {
          ai = wsum(ai);
          bi = wsum(bi);
        }
        if (lane == 0) {
          s_acc[c].x += ar;
          s_acc[c].y += ai;
          if (c2 != c) {
            s_acc[c2].x += br;
            s_acc[c2].y += bi;
          }
        }
      }
      __syncthreads();  // s_w is rewritten by the next rows
    }
    for (int c = threadIdx.x; c < ncols; c += blockDim.x)
      part[sq.pofs + (int64_t)c * sq.nslot + slot] = s_acc[c];
  });
}

// per operator: alpha_j, beta_j, breakdown, 1/beta (one block per operator).
// The last block to finish then closes the step: it splits the rows of the
// operators still running for the next step's reorthogonalisation kernels
// and advances the step counter (every block has read it by then).
__global__ void __launch_bounds__(256) k_bfinish(const BOp* __restrict__ ops, int nops, int Gmax,
                                                 SplitOp* __restrict__ sp,
                                                 int64_t* __restrict__ TG,
                                                 unsigned* __restrict__ nfinished, int ncap, int m,
                                                 const double* __restrict__ normpart,
                                                 const double2* __restrict__ coef1,
                                                 double* __restrict__ alpha,
                                                 double* __restrict__ beta,
                                                 double* __restrict__ invb,
                                                 int* __restrict__ nsteps,
                                                 int* __restrict__ step,
                                                 int* __restrict__ done, int setup) {
  const int q = blockIdx.x;
  const int j = *step;
  __shared__ double sh[8];
  __shared__ bool s_last;
  if (!done[q]) {
    const SplitOp o = sp[q];
    double s = 0.0;
    for (int k = threadIdx.x; k < o.nslot; k += blockDim.x) s += normpart[o.slot0 + k];
    s = wsum(s);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
      double n2 = 0.0;
      for (int k = 0; k < 8; ++k) n2 += sh[k];
      const double nrm = sqrt(n2);
      if (setup) {  // starting vector: zero or non-finite norm is an error for this operator
        if (!isfinite(nrm)) { done[q] = 4; invb[q] = 0.0; }
        else if (!(nrm > 0.0)) { done[q] = 3; invb[q] = 0.0; }
        else invb[q] = 1.0 / nrm;
      } else {
        const double a = coef1[(int64_t)q * ncap + j].x;
        alpha[(int64_t)q * m + j] = a;
        beta[(int64_t)q * m + j] = nrm;
        nsteps[q] = j + 1;
        const double seps = 1.4901161193847656e-08;  // sqrt(eps(Float64))
        if (nrm <= seps * fmax(1.0, fabs(a))) {
          beta[(int64_t)q * m + j] = 0.0;
          done[q] = 2;
          invb[q] = 0.0;
        } else {
          invb[q] = 1.0 / nrm;
        }
      }
    }
  }
  if (threadIdx.x == 0) {
    __threadfence();  // this block's stop flag before its count
    s_last = atomicAdd(nfinished, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  split_rows_dev(ops, nops, Gmax, ncap, done, sp, TG);
  if (threadIdx.x == 0) {
    *nfinished = 0;
    *step = j + 1;
  }
}

// V_q[:, j+1] = w_q / beta (skipped past the last column); k_bfinish has
// advanced the step counter to j + 1
template <class WV, class VV>
__global__ void __launch_bounds__(256) k_bscale(const BOp* __restrict__ ops,
                                                const int* __restrict__ tile2op, int ncap,
                                                const WV* __restrict__ w, VV* __restrict__ V,
                                                const double* __restrict__ invb,
                                                const int* __restrict__ step,
                                                const int* __restrict__ done) {
  const int q = tile2op[blockIdx.x];
  if (done[q]) return;
  const BOp& o = ops[q];
  const int col = *step;
  if (col >= ncap) return;
  const int64_t r = (blockIdx.x - o.tile0) * (int64_t)kTile + threadIdx.x;
  if (r >= o.D) return;
  const double sc = invb[q];
  const double2 v = l2(w + o.woff + r);
  s2(V + o.voff + (int64_t)col * o.D + r, make_double2(v.x * sc, v.y * sc));
}

// out_q = V_q[:, 0:nc_q] c_q (coefficients per operator, FP64 output)
template <class VV, class OV>
__global__ void __launch_bounds__(256) k_bcombine(const BOp* __restrict__ ops,
                                                  const int* __restrict__ tile2op, int ncap,
                                                  const VV* __restrict__ V,
                                                  const double2* __restrict__ c,
                                                  const int* __restrict__ ncols,
                                                  OV* __restrict__ out) {
  const int q = tile2op[blockIdx.x];
  const BOp& o = ops[q];
  const int64_t r = (blockIdx.x - o.tile0) * (int64_t)kTile + threadIdx.x;
  if (r >= o.D) return;
  const int nc = ncols[q];
  double ar = 0.0, ai = 0.0;
  for (int k = 0; k < nc; ++k) {
    const double2 v = l2(V + o.voff + (int64_t)k * o.D + r);
    const double2 ck = c[(int64_t)q * ncap + k];
    ar += v.x * ck.x - v.y * ck.y;
    ai += v.x * ck.y + v.y * ck.x;
  }
  s2(out + o.woff + r, make_double2(ar, ai));
}

namespace {

size_t esz(int dt) { return (dt == EDK_F64 || dt == EDK_C64) ? 8 : (dt == EDK_C128 ? 16 : 4); }

template <class F> edk_status with_vt(int dt, F&& f) {
  switch (dt) {
    case EDK_F64: return f((double*)nullptr);
    case EDK_C128: return f((double2*)nullptr);
    case EDK_F32: return f((float*)nullptr);
    case EDK_C64: return f((float2*)nullptr);
  }
  set_error("batch: unknown dtype");
  return EDK_INVALID_ARG;
}

double wall() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// A batch of operators sharing a lookup kind, kernel family and storage type.
struct BatchEngine {
  int nops = 0, vdt = EDK_F64, wdt = EDK_F64, ncap = 0, m = 0;
  int bk = 0;
  bool ff = false;
  bool plan = false;  // every operator carries a row plan (rank-searched sectors)
  bool plan_nn_all = false;  // ... and is one nearest-neighbour family of equal values
  bool sell = false;
  int64_t nsblk = 0;
  cudaStream_t st = nullptr;
  std::vector<BOp> hops;
  std::vector<int64_t> Ds;
  int64_t ntiles = 0, totalD = 0;
  int G = 1;             // blocks of the reorthogonalisation grid
  int nsm = 1;           // SMs of the device
  bool fused = false;    // first update and second dot products in one kernel
  DevBuf dops, tile2op, sblk2op, splitops, splitT, nfin, V, w, wt, part, coef1, coef2, normpart, alpha, beta, invb,
      done, step, nsteps, cbuf, cnc;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  bool graph_ok = false;

  ~BatchEngine() {
    if (gexec) cudaGraphExecDestroy(gexec);
    if (graph) cudaGraphDestroy(graph);
  }

  edk_status init(const std::vector<edk_operator*>& ops, int vdtype, int m_, int lookup_kind,
                  bool use_ff, cudaStream_t s) {
    nops = (int)ops.size();
    if (nops > 65535) {
      set_error("batch Lanczos: at most 65535 operators per batch");
      return EDK_UNSUPPORTED;
    }
    // row plans (built here, outside any capture) when the sectors are ranked
    plan = use_ff && (lookup_kind == BK_TRANS0_RANK || lookup_kind == BK_TRANS_RANK ||
                      lookup_kind == BK_TRANSPAR_RANK || lookup_kind == BK_PROJ_RANK);
    plan_nn_all = plan;
    for (auto* op : ops) {
      if (!plan) break;
      if (!plan_applies(op)) { plan = false; break; }
      EDK_RETURN_IF(plan_ensure(op));
      plan = op->plan_state == 1;
      plan_nn_all = plan_nn_all && plan_nn(*reinterpret_cast<const FFParams*>(op->ff_params.data()));
    }
    vdt = vdtype;
    wdt = (vdt == EDK_C128 || vdt == EDK_C64) ? EDK_C128 : EDK_F64;
    m = m_;
    ncap = m + 1;
    bk = lookup_kind;
    ff = use_ff;
    st = s;
    std::vector<int> t2o, s2o;
    int64_t voff = 0, woff = 0;
    sell = true;
    for (auto* op : ops) sell = sell && op->sell_ok;
    for (int q = 0; q < nops; ++q) {
      edk_operator* op = ops[q];
      BOp o{};
      o.b = op->b->dev;
      o.b.bk = bk;
      o.op = op->dev;
      if (use_ff) std::memcpy(&o.ff, op->ff_params.data(), sizeof(FFParams));
      o.D = op->b->D;
      o.ntile = (int)((o.D + kTile - 1) / kTile);
      o.voff = voff;
      o.woff = woff;
      o.tile0 = ntiles;
      o.sblk0 = nsblk;
      if (sell) {
        const int64_t nb = (op->dev.sell.nslices + 7) / 8;
        for (int64_t k = 0; k < nb; ++k) s2o.push_back(q);
        nsblk += nb;
      }
      for (int k = 0; k < o.ntile; ++k) t2o.push_back(q);
      ntiles += o.ntile;
      voff += o.D * ncap;
      woff += o.D;
      hops.push_back(o);
      Ds.push_back(o.D);
    }
    totalD = woff;
    EDK_RETURN_IF(split_rows());
    EDK_RETURN_IF(dops.alloc_async(hops.size() * sizeof(BOp), st));
    EDK_TRY_CUDA(cudaMemcpyAsync(dops.p, hops.data(), hops.size() * sizeof(BOp),
                                 cudaMemcpyHostToDevice, st));
    EDK_RETURN_IF(tile2op.alloc_async(t2o.size() * 4, st));
    EDK_TRY_CUDA(cudaMemcpyAsync(tile2op.p, t2o.data(), t2o.size() * 4, cudaMemcpyHostToDevice, st));
    if (sell) {
      EDK_RETURN_IF(sblk2op.alloc_async(std::max<size_t>(s2o.size(), 1) * 4, st));
      if (!s2o.empty())
        EDK_TRY_CUDA(cudaMemcpyAsync(sblk2op.p, s2o.data(), s2o.size() * 4,
                                     cudaMemcpyHostToDevice, st));
    }
    EDK_RETURN_IF(V.alloc_async((size_t)voff * esz(vdt), st));
    EDK_RETURN_IF(w.alloc_async((size_t)totalD * esz(wdt), st));
    EDK_RETURN_IF(wt.alloc_async((size_t)totalD * esz(vdt), st));
    // a block meets at most one operator more than it starts in: G + nops slots
    EDK_RETURN_IF(part.alloc_async((size_t)(G + nops) * ncap * sizeof(double2), st));
    EDK_RETURN_IF(splitops.alloc_async((size_t)nops * sizeof(SplitOp), st));
    EDK_RETURN_IF(splitT.alloc_async(2 * sizeof(int64_t), st));
    EDK_RETURN_IF(nfin.alloc_async(sizeof(unsigned), st));
    EDK_TRY_CUDA(cudaMemsetAsync(nfin.p, 0, sizeof(unsigned), st));
    EDK_RETURN_IF(coef1.alloc_async((size_t)nops * ncap * sizeof(double2), st));
    EDK_RETURN_IF(coef2.alloc_async((size_t)nops * ncap * sizeof(double2), st));
    EDK_RETURN_IF(normpart.alloc_async((size_t)(G + nops) * sizeof(double), st));
    EDK_RETURN_IF(alpha.alloc_async((size_t)nops * m * sizeof(double), st));
    EDK_RETURN_IF(beta.alloc_async((size_t)nops * m * sizeof(double), st));
    EDK_RETURN_IF(invb.alloc_async((size_t)nops * sizeof(double), st));
    EDK_RETURN_IF(done.alloc_async((size_t)nops * sizeof(int), st));
    EDK_RETURN_IF(nsteps.alloc_async((size_t)nops * sizeof(int), st));
    EDK_RETURN_IF(step.alloc_async(sizeof(int), st));
    EDK_RETURN_IF(cbuf.alloc_async((size_t)nops * ncap * sizeof(double2), st));
    EDK_RETURN_IF(cnc.alloc_async((size_t)nops * sizeof(int), st));
    EDK_TRY_CUDA(cudaMemsetAsync(done.p, 0, nops * sizeof(int), st));
    EDK_TRY_CUDA(cudaMemsetAsync(nsteps.p, 0, nops * sizeof(int), st));
    EDK_TRY_CUDA(cudaMemsetAsync(alpha.p, 0, (size_t)nops * m * sizeof(double), st));
    EDK_TRY_CUDA(cudaMemsetAsync(beta.p, 0, (size_t)nops * m * sizeof(double), st));
    return EDK_OK;
  }

  // Opt the reorthogonalisation kernels into the shared memory they need
  // (outside any capture) and size their grid to what is resident at once.
  edk_status split_rows() {
    const size_t us = (size_t)(ncap + 8) * sizeof(double2);
    if (us > 200 * 1024) {
      set_error("batch Lanczos: too many steps for the shared-memory coefficients (max 12791)");
      return EDK_UNSUPPORTED;
    }
    const size_t fs = us + (size_t)ncap * sizeof(double2);  // + column sums
    fused = fs <= 200 * 1024;
    int dev = 0;
    EDK_TRY_CUDA(cudaGetDevice(&dev));
    EDK_TRY_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    int per_sm = 0;
    edk_status s = with_vt(vdt, [&](auto vp) -> edk_status {
      using VV = std::remove_pointer_t<decltype(vp)>;
      return with_vt(wdt, [&](auto wp) -> edk_status {
        using WD = std::remove_pointer_t<decltype(wp)>;
        const auto attr = cudaFuncAttributeMaxDynamicSharedMemorySize;
        const auto ku1 = k_rupdate<VV, VV, WD>;
        const auto ku2 = k_rupdate<VV, WD, WD>;
        const auto kd1 = k_rdots<VV, VV>;
        const auto kd2 = k_rdots<VV, WD>;
        const auto kf = k_rupdate_dots<VV, VV, WD>;
        if (us > 48 * 1024) {
          EDK_TRY_CUDA(cudaFuncSetAttribute(ku1, attr, (int)us));
          EDK_TRY_CUDA(cudaFuncSetAttribute(ku2, attr, (int)us));
        }
        if (fused && fs > 48 * 1024) EDK_TRY_CUDA(cudaFuncSetAttribute(kf, attr, (int)fs));
        int n[5] = {0, 0, 0, 0, 0};
        EDK_TRY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n[0], ku1, 256, us));
        EDK_TRY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n[1], ku2, 256, us));
        EDK_TRY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n[2], kd1, 256, 0));
        EDK_TRY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n[3], kd2, 256, 0));
        if (fused) EDK_TRY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n[4], kf, 256, fs));
        per_sm = std::min({n[0], n[1], fused ? n[4] : n[2], n[2], n[3]});
        return EDK_OK;
      });
    });
    EDK_RETURN_IF(s);
    // at least 256 rows a block, at most the resident blocks
    const int64_t want = std::max<int64_t>(1, (totalD + 255) / 256);
    G = (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)nsm * std::max(per_sm, 1), want));
    return EDK_OK;
  }

  const BOp* d_ops() const { return dops.as<BOp>(); }

  edk_status launch_apply() {
    const int* t2o = tile2op.as<int>();
    const int* stp = step.as<int>();
    const int* dn = done.as<int>();
    return with_vt(vdt, [&](auto vp) -> edk_status {
      using VT = std::remove_pointer_t<decltype(vp)>;
      const VT* Vv = V.as<VT>();
      VT* wv = wt.as<VT>();
      if (sell) {
        if (nsblk > 0)
          k_bapply_sell<VT><<<(unsigned)nsblk, 256, 0, st>>>(d_ops(), sblk2op.as<int>(), Vv, wv,
                                                             stp, dn);
        return EDK_OK;
      }
      if (plan) {
        switch (bk) {
          case BK_PROJ_RANK:
            if (plan_nn_all)
              k_bapply_plan<BK_PROJ_RANK, VT, 1><<<plan_grid(plan_min_blocks<BK_PROJ_RANK, VT>()), 256, 0, st>>>(
                  d_ops(), t2o, ntiles, Vv, wv, stp, dn);
            else
              k_bapply_plan<BK_PROJ_RANK, VT, 2><<<plan_grid(plan_min_blocks<BK_PROJ_RANK, VT>()), 256, 0, st>>>(
                  d_ops(), t2o, ntiles, Vv, wv, stp, dn);
            return EDK_OK;
          case BK_TRANS0_RANK:
            if (plan_nn_all)
              k_bapply_plan<BK_TRANS0_RANK, VT, 1><<<plan_grid(plan_min_blocks<BK_TRANS0_RANK, VT>()), 256, 0, st>>>(
                  d_ops(), t2o, ntiles, Vv, wv, stp, dn);
            else
              k_bapply_plan<BK_TRANS0_RANK, VT, 2><<<plan_grid(plan_min_blocks<BK_TRANS0_RANK, VT>()), 256, 0, st>>>(
                  d_ops(), t2o, ntiles, Vv, wv, stp, dn);
            return EDK_OK;
          case BK_TRANS_RANK:
            if (plan_nn_all)
              k_bapply_plan<BK_TRANS_RANK, VT, 1><<<plan_grid(plan_min_blocks<BK_TRANS_RANK, VT>()), 256, 0, st>>>(
                  d_ops(), t2o, ntiles, Vv, wv, stp, dn);
            else
              k_bapply_plan<BK_TRANS_RANK, VT, 2><<<plan_grid(plan_min_blocks<BK_TRANS_RANK, VT>()), 256, 0, st>>>(
                  d_ops(), t2o, ntiles, Vv, wv, stp, dn);
            return EDK_OK;
          case BK_TRANSPAR_RANK:
            if (plan_nn_all)
              k_bapply_plan<BK_TRANSPAR_RANK, VT, 1><<<plan_grid(plan_min_blocks<BK_TRANSPAR_RANK, VT>()), 256, 0, st>>>(
                  d_ops(), t2o, ntiles, Vv, wv, stp, dn);
            else
              k_bapply_plan<BK_TRANSPAR_RANK, VT, 2><<<plan_grid(plan_min_blocks<BK_TRANSPAR_RANK, VT>()), 256, 0, st>>>(
                  d_ops(), t2o, ntiles, Vv, wv, stp, dn);
            return EDK_OK;
        }
      }
#define EDK_BAPPLY(BK)                                                                       \
  case BK:                                                                                   \
    if (ff) k_bapply_ff<BK, VT><<<(unsigned)ntiles, 256, 0, st>>>(d_ops(), t2o, Vv, wv, stp, dn); \
    else k_bapply_gen<BK, VT><<<(unsigned)ntiles, 256, 0, st>>>(d_ops(), t2o, Vv, wv, stp, dn);  \
    break;
      switch (bk) {
        EDK_BAPPLY(BK_TENSOR)
        EDK_BAPPLY(BK_PROJ_RANK)
        EDK_BAPPLY(BK_PROJ_HASH)
        EDK_BAPPLY(BK_TRANS0)
        case BK_TRANS0_RANK:  // bond-family fast path only (other paths keep the hash)
          k_bapply_ff<BK_TRANS0_RANK, VT><<<(unsigned)ntiles, 256, 0, st>>>(d_ops(), t2o, Vv, wv,
                                                                           stp, dn);
          break;
        case BK_TRANS_RANK:
          k_bapply_ff<BK_TRANS_RANK, VT><<<(unsigned)ntiles, 256, 0, st>>>(d_ops(), t2o, Vv, wv,
                                                                          stp, dn);
          break;
        case BK_TRANSPAR_RANK:
          k_bapply_ff<BK_TRANSPAR_RANK, VT><<<(unsigned)ntiles, 256, 0, st>>>(d_ops(), t2o, Vv,
                                                                             wv, stp, dn);
          break;
        EDK_BAPPLY(BK_TRANS)
        EDK_BAPPLY(BK_TRANSPAR)
        default:
          set_error("batch Lanczos: lookup kind not supported in batches");
          return EDK_UNSUPPORTED;
      }
#undef EDK_BAPPLY
      return EDK_OK;
    });
  }

  // resident grid of the row-plan matvec: per_sm blocks on every SM, at
  // most one block per tile
  unsigned plan_grid(int per_sm) const {
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>(ntiles, (int64_t)nsm * per_sm));
  }

  RowSplit rsplit() const {
    return RowSplit{splitops.as<SplitOp>(), splitT.as<int64_t>(), nops};
  }

  void launch_split() {
    k_bsplit<<<1, 1024, 0, st>>>(d_ops(), nops, G, ncap, done.as<int>(), splitops.as<SplitOp>(),
                                 splitT.as<int64_t>());
  }

  // alpha / beta / stop flags, then (last block) the next step's split and
  // the step counter
  void launch_finish(int setup) {
    k_bfinish<<<nops, 256, 0, st>>>(d_ops(), nops, G, splitops.as<SplitOp>(),
                                    splitT.as<int64_t>(), nfin.as<unsigned>(), ncap, m,
                                    normpart.as<double>(), coef1.as<double2>(),
                                    alpha.as<double>(), beta.as<double>(), invb.as<double>(),
                                    nsteps.as<int>(), step.as<int>(), done.as<int>(), setup);
  }

  template <class XT>
  edk_status launch_dots(const XT* x) {
    return with_vt(vdt, [&](auto vp) -> edk_status {
      using VV = std::remove_pointer_t<decltype(vp)>;
      k_rdots<VV, XT><<<(unsigned)G, 256, 0, st>>>(d_ops(), rsplit(), V.as<VV>(), x,
                                                   part.as<double2>(), step.as<int>(),
                                                   done.as<int>());
      return EDK_OK;
    });
  }

  template <class WI, class WO>
  edk_status launch_update(const double2* coef, const WI* win, WO* wout, bool norm, int zero) {
    const size_t smem = (size_t)(ncap + 8) * sizeof(double2);
    return with_vt(vdt, [&](auto vp) -> edk_status {
      using VV = std::remove_pointer_t<decltype(vp)>;
      k_rupdate<VV, WI, WO><<<(unsigned)G, 256, smem, st>>>(
          d_ops(), rsplit(), ncap, V.as<VV>(), coef, win, wout,
          norm ? normpart.as<double>() : nullptr, step.as<int>(), done.as<int>(), zero);
      return EDK_OK;
    });
  }

  template <class WI, class WO>
  edk_status launch_update_dots(const double2* coef, const WI* win, WO* wout) {
    const size_t smem = (size_t)(2 * ncap + 8) * sizeof(double2);
    return with_vt(vdt, [&](auto vp) -> edk_status {
      using VV = std::remove_pointer_t<decltype(vp)>;
      k_rupdate_dots<VV, WI, WO><<<(unsigned)G, 256, smem, st>>>(
          d_ops(), rsplit(), ncap, V.as<VV>(), coef, win, wout, part.as<double2>(),
          step.as<int>(), done.as<int>());
      return EDK_OK;
    });
  }

  // one Lanczos step for every live operator (graph-capturable)
  edk_status enqueue_step() {
    EDK_RETURN_IF(launch_apply());
    edk_status s = with_vt(vdt, [&](auto vp) -> edk_status {
      using VV = std::remove_pointer_t<decltype(vp)>;
      return with_vt(wdt, [&](auto wp) -> edk_status {
        using WD = std::remove_pointer_t<decltype(wp)>;
        EDK_RETURN_IF(launch_dots<VV>(wt.as<VV>()));
        k_breduce<<<dim3((ncap + 7) / 8, nops), 256, 0, st>>>(
            splitops.as<SplitOp>(), ncap, part.as<double2>(), coef1.as<double2>(), step.as<int>(),
            done.as<int>());
        if (fused) {
          EDK_RETURN_IF((launch_update_dots<VV, WD>(coef1.as<double2>(), wt.as<VV>(), w.as<WD>())));
        } else {
          EDK_RETURN_IF((launch_update<VV, WD>(coef1.as<double2>(), wt.as<VV>(), w.as<WD>(), false, 0)));
          EDK_RETURN_IF(launch_dots<WD>(w.as<WD>()));
        }
        k_breduce<<<dim3((ncap + 7) / 8, nops), 256, 0, st>>>(
            splitops.as<SplitOp>(), ncap, part.as<double2>(), coef2.as<double2>(), step.as<int>(),
            done.as<int>());
        EDK_RETURN_IF((launch_update<WD, WD>(coef2.as<double2>(), w.as<WD>(), w.as<WD>(), true, 0)));
        launch_finish(0);
        k_bscale<WD, VV><<<(unsigned)ntiles, 256, 0, st>>>(d_ops(), tile2op.as<int>(), ncap,
                                                           w.as<WD>(), V.as<VV>(),
                                                           invb.as<double>(), step.as<int>(),
                                                           done.as<int>());
        return EDK_OK;
      });
    });
    EDK_RETURN_IF(s);
    EDK_TRY_CUDA(cudaGetLastError());
    return EDK_OK;
  }

  // V[:, 0] = start / ||start||; start is FP64 (wdt) concatenated on the device
  edk_status setup(const void* start_dev) {
    int minus1 = -1;
    EDK_TRY_CUDA(cudaMemcpyAsync(step.p, &minus1, sizeof(int), cudaMemcpyHostToDevice, st));
    launch_split();
    edk_status s = with_vt(vdt, [&](auto vp) -> edk_status {
      using VV = std::remove_pointer_t<decltype(vp)>;
      return with_vt(wdt, [&](auto wp) -> edk_status {
        using WD = std::remove_pointer_t<decltype(wp)>;
        EDK_RETURN_IF((launch_update<WD, WD>(coef1.as<double2>(), (const WD*)start_dev,
                                             w.as<WD>(), true, 1)));
        launch_finish(1);
        k_bscale<WD, VV><<<(unsigned)ntiles, 256, 0, st>>>(d_ops(), tile2op.as<int>(), ncap,
                                                           w.as<WD>(), V.as<VV>(),
                                                           invb.as<double>(), step.as<int>(),
                                                           done.as<int>());
        return EDK_OK;
      });
    });
    EDK_RETURN_IF(s);
    EDK_TRY_CUDA(cudaGetLastError());
    return EDK_OK;
  }

  edk_status capture() {
    if (graph_ok) return EDK_OK;
    cudaError_t e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return EDK_OK;  // replay not available: launch directly
    edk_status s = enqueue_step();
    cudaError_t e2 = cudaStreamEndCapture(st, &graph);
    if (s != EDK_OK) return s;
    if (e2 != cudaSuccess || !graph) { cudaGetLastError(); return EDK_OK; }
    if (cudaGraphInstantiate(&gexec, graph, 0) != cudaSuccess) {
      cudaGetLastError();
      return EDK_OK;
    }
    graph_ok = true;
    return EDK_OK;
  }

  edk_status run_step() {
    if (graph_ok) {
      EDK_TRY_CUDA(cudaGraphLaunch(gexec, st));
      return EDK_OK;
    }
    return enqueue_step();
  }
};

// Run the batch until every operator is done or max steps.
edk_status run_batch(BatchEngine& E, int max_steps, int nev, double tol, int check_every,
                     std::vector<OpResult>& res, int* nchecks = nullptr) {
  const int nops = E.nops;
  res.assign(nops, OpResult{});
  std::vector<double> ha((size_t)nops * E.m), hb((size_t)nops * E.m);
  std::vector<int> hdone(nops), hsteps(nops);
  std::vector<std::vector<double>> prev(nops);
  EDK_RETURN_IF(E.capture());
  int every = check_every > 0 ? check_every : 10;
  for (int j = 0; j < max_steps; ++j) {
    EDK_RETURN_IF(E.run_step());
    bool last = (j + 1 == max_steps);
    if (!last && !((j + 1) % every == 0 && tol > 0)) continue;
    if (nchecks) ++*nchecks;
    EDK_TRY_CUDA(cudaMemcpyAsync(hdone.data(), E.done.p, nops * sizeof(int), cudaMemcpyDeviceToHost, E.st));
    EDK_TRY_CUDA(cudaMemcpyAsync(hsteps.data(), E.nsteps.p, nops * sizeof(int), cudaMemcpyDeviceToHost, E.st));
    EDK_TRY_CUDA(cudaMemcpyAsync(ha.data(), E.alpha.p, ha.size() * 8, cudaMemcpyDeviceToHost, E.st));
    EDK_TRY_CUDA(cudaMemcpyAsync(hb.data(), E.beta.p, hb.size() * 8, cudaMemcpyDeviceToHost, E.st));
    EDK_TRY_CUDA(cudaStreamSynchronize(E.st));
    bool all_done = true;
    bool changed = false;
    for (int q = 0; q < nops; ++q) {
      if (hdone[q]) continue;
      int mq = hsteps[q];
      if (tol > 0 && mq >= nev) {
        std::vector<double> w(mq);
        if (tridiag_eigvals(mq, ha.data() + (size_t)q * E.m, hb.data() + (size_t)q * E.m, w.data()) == 0) {
          bool conv = !prev[q].empty();
          for (int k = 0; k < nev && k < mq && conv; ++k)
            conv = std::fabs(w[k] - prev[q][k]) <= tol * std::max(1.0, std::fabs(w[k]));
          prev[q].assign(w.begin(), w.begin() + std::min(nev, mq));
          if (conv) { hdone[q] = 1; changed = true; continue; }
        }
      }
      all_done = false;
    }
    if (changed)
      EDK_TRY_CUDA(cudaMemcpyAsync(E.done.p, hdone.data(), nops * sizeof(int), cudaMemcpyHostToDevice, E.st));
    if (all_done) break;
  }
  EDK_TRY_CUDA(cudaMemcpyAsync(hdone.data(), E.done.p, nops * sizeof(int), cudaMemcpyDeviceToHost, E.st));
  EDK_TRY_CUDA(cudaMemcpyAsync(hsteps.data(), E.nsteps.p, nops * sizeof(int), cudaMemcpyDeviceToHost, E.st));
  EDK_TRY_CUDA(cudaMemcpyAsync(ha.data(), E.alpha.p, ha.size() * 8, cudaMemcpyDeviceToHost, E.st));
  EDK_TRY_CUDA(cudaMemcpyAsync(hb.data(), E.beta.p, hb.size() * 8, cudaMemcpyDeviceToHost, E.st));
  EDK_TRY_CUDA(cudaStreamSynchronize(E.st));
  for (int q = 0; q < nops; ++q) {
    OpResult& r = res[q];
    r.status = hdone[q];
    r.steps = hsteps[q];
    r.a.assign(ha.begin() + (size_t)q * E.m, ha.begin() + (size_t)q * E.m + r.steps);
    r.b.assign(hb.begin() + (size_t)q * E.m, hb.begin() + (size_t)q * E.m + r.steps);
    if (r.steps > 0) {
      std::vector<double> w(r.steps);
      tridiag_eigvals(r.steps, r.a.data(), r.b.data(), w.data());
      r.ev.assign(w.begin(), w.begin() + std::min(nev, r.steps));
    }
  }
  return EDK_OK;
}

// FP64 start vectors for the refinement of each operator into out (wdt
// layout): the sum of its `nev` lowest Ritz vectors, so the refined Krylov
// space holds every wanted eigenvector.
edk_status ritz_vectors(BatchEngine& E, const std::vector<OpResult>& res, void* out, int nev) {
  std::vector<double2> c((size_t)E.nops * E.ncap, make_double2(0.0, 0.0));
  std::vector<int> nc(E.nops, 0);
  for (int q = 0; q < E.nops; ++q) {
    int mq = res[q].steps;
    if (mq <= 0) continue;
    std::vector<double> w(mq), Q((size_t)mq * mq);
    if (tridiag_eigen(mq, res[q].a.data(), res[q].b.data(), w.data(), Q.data()) != 0) {
      set_error("tridiagonal eigensolver did not converge");
      return EDK_NOT_CONVERGED;
    }
    const int nk = std::min(nev, mq);
    for (int k = 0; k < mq; ++k) {
      double v = 0.0;
      for (int e = 0; e < nk; ++e) v += Q[k + (size_t)e * mq];
      c[(size_t)q * E.ncap + k] = make_double2(v, 0.0);
    }
    nc[q] = mq;
  }
  const size_t cb = c.size() * sizeof(double2), nb = nc.size() * sizeof(int);
  EDK_TRY_CUDA(cudaMemcpyAsync(E.cbuf.p, c.data(), cb, cudaMemcpyHostToDevice, E.st));
  EDK_TRY_CUDA(cudaMemcpyAsync(E.cnc.p, nc.data(), nb, cudaMemcpyHostToDevice, E.st));
  return with_vt(E.vdt, [&](auto vp) -> edk_status {
    using VV = std::remove_pointer_t<decltype(vp)>;
    return with_vt(E.wdt, [&](auto wp) -> edk_status {
      using WD = std::remove_pointer_t<decltype(wp)>;
      k_bcombine<VV, WD><<<(unsigned)E.ntiles, 256, 0, E.st>>>(
          E.d_ops(), E.tile2op.as<int>(), E.ncap, E.V.as<VV>(), E.cbuf.as<double2>(),
          E.cnc.as<int>(), (WD*)out);
      EDK_TRY_CUDA(cudaGetLastError());
      return EDK_OK;
    });
  });
}

// convert/copy concatenated start vectors into a device FP64 buffer of dtype wdt
template <class S, class D>
__global__ void k_cast(const S* __restrict__ src, int64_t n, D* __restrict__ dst) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    s2(dst + i, l2(src + i));
}

}  // namespace

// Group-level driver: FP64 or mixed (FP32 Krylov vectors + FP64 refinement).
edk_status batch_lanczos(const std::vector<edk_operator*>& ops, const edk_lanczos_opts& o,
                         const void* v0_dev, int v0_dt, cudaStream_t st,
                         std::vector<OpResult>& res, edk_lanczos_diag* diag, void* ritz_out) {
  double t0 = wall();
  const int nops = (int)ops.size();
  bool cx = o.complex_vectors != 0 || v0_dt == EDK_C128 || v0_dt == EDK_C64;
  for (auto* op : ops) cx |= op->is_complex;
  bool mixed = o.precision == EDK_PREC_MIXED;
  int vdt = mixed ? (cx ? EDK_C64 : EDK_F32) : (cx ? EDK_C128 : EDK_F64);
  int wdt = cx ? EDK_C128 : EDK_F64;
  // common lookup kind: translation sectors with and without phases share BK_TRANS
  int bk = ops[0]->b->dev.bk;
  bool all_mat = true;  // materialised operators run on the sliced-ELL kernel, whatever the basis
  for (auto* op : ops) all_mat = all_mat && op->sell_ok;
  bool ff = true;
  int64_t Dmin = INT64_MAX;
  for (auto* op : ops) {
    int k = op->b->dev.bk;
    if (k != bk) {
      if ((k == BK_TRANS0 || k == BK_TRANS) && (bk == BK_TRANS0 || bk == BK_TRANS)) bk = BK_TRANS;
      else if (!all_mat) {
        set_error("batch Lanczos: operators of different basis kinds");
        return EDK_UNSUPPORTED;
      }
    }
    ff = ff && op->ff_ok && op->use_ff;
    if (!op->gather) {
      set_error("batch Lanczos: an operator is not Hermitian in its basis");
      return EDK_NOT_HERMITIAN;
    }
    if (op->b->L > 32 && !op->sell_ok) {
      set_error("batch Lanczos: L > 32 runs only on materialised operators");
      return EDK_UNSUPPORTED;
    }
    Dmin = std::min<int64_t>(Dmin, op->b->D);
  }
  // translation sectors searched through their rank tables (with a phase:
  // every table must carry the shift M)
  bool ranked = (bk == BK_TRANS0 || bk == BK_TRANS || bk == BK_TRANSPAR) && ff;
  for (auto* op : ops)
    ranked = ranked && op->b->dev.search == 2 && (bk != BK_TRANS || op->b->dev.rank_shift == 10);
  if (ranked)
    bk = bk == BK_TRANS0 ? BK_TRANS0_RANK : (bk == BK_TRANS ? BK_TRANS_RANK : BK_TRANSPAR_RANK);
  if (bk == BK_ABELIAN && !all_mat) {
    set_error("batch Lanczos: symmetry-group (abelian) bases run one at a time unless materialised");
    return EDK_UNSUPPORTED;
  }
  (void)Dmin;  // operators smaller than max_steps stop by the breakdown rule
  BatchEngine E;
  double ts0 = wall();
  int nchecks = 0;
  EDK_RETURN_IF(E.init(ops, vdt, o.max_steps, bk, ff, st));
  // start vectors in FP64 working dtype
  DevBuf start;
  EDK_RETURN_IF(start.alloc_async((size_t)E.totalD * esz(wdt), st));
  edk_status s = with_vt(v0_dt, [&](auto sp) -> edk_status {
    using SV = std::remove_pointer_t<decltype(sp)>;
    return with_vt(wdt, [&](auto dp) -> edk_status {
      using DV = std::remove_pointer_t<decltype(dp)>;
      k_cast<SV, DV><<<1184, 256, 0, st>>>((const SV*)v0_dev, E.totalD, (DV*)start.p);
      return EDK_OK;
    });
  });
  EDK_RETURN_IF(s);
  EDK_RETURN_IF(E.setup(start.p));
  EDK_RETURN_IF(E.capture());
  EDK_TRY_CUDA(cudaStreamSynchronize(st));
  double ts1 = wall();
  // mixed stage 1 (FP32 vectors): its Ritz values move by rounding at ~1e-7,
  // so it stops well above that — a ground state needs only a good start for
  // the FP64 refinement (1e-5), several levels a better one (1e-7) — and, for
  // a few operators, it checks every 5 steps so that it stops early
  double tol1 = mixed ? std::max(o.tol, o.nev > 1 ? 1e-7 : 1e-5) : o.tol;
  // (a check solves every operator's tridiagonal problem on the host, so
  // large batches keep the caller's interval)
  const int check1 = (mixed && nops <= 8)
                         ? std::max(1, std::min(o.check_every > 0 ? o.check_every : 5, 5))
                         : o.check_every;
  EDK_RETURN_IF(run_batch(E, o.max_steps, o.nev, tol1, check1, res, &nchecks));
  double ts2 = wall();
  int rounds = 0;
  for (int q = 0; q < nops; ++q) {
    if (res[q].status == 4) {
      set_error("Initial state has non-finite entries (NaN or Inf)");
      return EDK_INVALID_ARG;
    }
    if (res[q].status == 3) {
      set_error("Initial state has zero norm");
      return EDK_ZERO_NORM;
    }
  }
  int steps_low = 0, mvs = 0, bd = 0;
  for (auto& r : res) { steps_low = std::max(steps_low, r.steps); mvs += r.steps; bd |= r.status == 2; }
  // global element offset of each operator in the concatenated layout
  std::vector<int64_t> goff(nops);
  for (int q = 0; q < nops; ++q) goff[q] = E.hops[q].woff;
  if (!mixed && ritz_out) EDK_RETURN_IF(ritz_vectors(E, res, ritz_out, 1));
  if (mixed) {
    // FP64 refinement restarted from the sum of the nev lowest Ritz vectors,
    // in one round that may run to max_steps (each operator stops when it
    // converges: a few steps for a ground state, more to separate close
    // levels).  Operators that reach the step limit unconverged are
    // restarted again, alone.
    const int mr = std::max(o.max_steps, o.refine_steps);
    std::vector<int> active(nops);
    for (int q = 0; q < nops; ++q) active[q] = q;
    DevBuf cur;  // start vectors of `active`, compact in that order
    EDK_RETURN_IF(ritz_vectors(E, res, start.p, o.nev));
    void* cur_p = start.p;
    for (int round = 0; round < 4 && !active.empty(); ++round) {
      std::vector<edk_operator*> sub;
      for (int q : active) sub.push_back(ops[q]);
      BatchEngine F;
      EDK_RETURN_IF(F.init(sub, wdt, mr, bk, ff, st));
      EDK_RETURN_IF(F.setup(cur_p));
      std::vector<OpResult> r2;
      ++rounds;
      EDK_RETURN_IF(run_batch(F, mr, o.nev, o.tol, std::min(5, mr), r2, &nchecks));
      std::vector<int> next;
      std::vector<int> keep;  // positions in `active` of the operators to restart
      for (size_t i = 0; i < active.size(); ++i) {
        const int q = active[i];
        bool still = r2[i].ev.size() == res[q].ev.size();
        for (size_t k = 0; k < r2[i].ev.size() && still; ++k) {
          const double a = r2[i].ev[k], b = res[q].ev[k];
          still = std::fabs(a - b) <= std::max(o.tol, 1e-14) * std::max(1.0, std::fabs(a));
        }
        mvs += r2[i].steps;
        res[q] = r2[i];
        if (r2[i].status == 0 && !still && o.tol > 0) {
          next.push_back(q);
          keep.push_back((int)i);
        }
      }
      if (ritz_out) {
        // lowest Ritz vectors of the operators this round finalises
        DevBuf gs;
        EDK_RETURN_IF(gs.alloc_async((size_t)F.totalD * esz(wdt), st));
        EDK_RETURN_IF(ritz_vectors(F, r2, gs.p, 1));
        size_t k = 0;
        const bool last_round = round == 3;  // restarts end here: every vector is final
        for (size_t i = 0; i < active.size(); ++i) {
          if (!last_round && k < keep.size() && keep[k] == (int)i) { ++k; continue; }
          const int q = active[i];
          EDK_TRY_CUDA(cudaMemcpyAsync((char*)ritz_out + goff[q] * esz(wdt),
                                       (char*)gs.p + F.hops[i].woff * esz(wdt),
                                       (size_t)F.Ds[i] * esz(wdt), cudaMemcpyDeviceToDevice, st));
        }
        EDK_TRY_CUDA(cudaStreamSynchronize(st));
      }
      if (next.empty()) break;
      // Ritz vectors of this round (F's layout), then the restarted subset
      DevBuf full;
      EDK_RETURN_IF(full.alloc_async((size_t)F.totalD * esz(wdt), st));
      EDK_RETURN_IF(ritz_vectors(F, r2, full.p, o.nev));
      int64_t tot = 0;
      for (int i : keep) tot += F.Ds[i];
      DevBuf nb;
      EDK_RETURN_IF(nb.alloc_async((size_t)std::max<int64_t>(tot, 1) * esz(wdt), st));
      int64_t dst = 0;
      for (int i : keep) {
        EDK_TRY_CUDA(cudaMemcpyAsync((char*)nb.p + dst * esz(wdt),
                                     (char*)full.p + F.hops[i].woff * esz(wdt),
                                     (size_t)F.Ds[i] * esz(wdt), cudaMemcpyDeviceToDevice, st));
        dst += F.Ds[i];
      }
      EDK_TRY_CUDA(cudaStreamSynchronize(st));
      std::swap(cur.p, nb.p);
      std::swap(cur.bytes, nb.bytes);
      std::swap(cur.pooled, nb.pooled);
      std::swap(cur.pool_stream, nb.pool_stream);
      cur_p = cur.p;
      active = next;
    }
  }
  EDK_TRY_CUDA(cudaStreamSynchronize(st));
  if (diag) {
    diag->steps = 0;
    for (auto& r : res) diag->steps = std::max(diag->steps, r.steps);
    diag->steps_low = mixed ? steps_low : diag->steps;
    diag->matvecs = mvs;
    diag->breakdown = bd;
    diag->seconds = wall() - t0;
    diag->seconds_matvec = NAN;
    diag->seconds_reorth = NAN;
    double resid = 0.0;
    for (auto& r : res) {
      int mm = r.steps;
      if (mm <= 0) continue;
      std::vector<double> w(mm), Q((size_t)mm * mm);
      if (tridiag_eigen(mm, r.a.data(), r.b.data(), w.data(), Q.data()) == 0)
        resid = std::max(resid, std::fabs(r.b[mm - 1] * Q[(size_t)mm - 1]));
    }
    diag->residual = resid;
    diag->seconds_setup = ts1 - ts0;
    diag->seconds_stage1 = ts2 - ts1;
    diag->seconds_refine = mixed ? wall() - ts2 : 0.0;
    diag->refine_rounds = rounds;
    diag->checks = nchecks;
  }
  return EDK_OK;
}

}  // namespace edk

using namespace edk;

extern "C" edk_status edk_batch_lanczos_e0(int32_t nops, edk_operator* const* ops,
                                           const edk_lanczos_opts* opts, const void* v0s,
                                           int32_t v0_dtype, double* evals,
                                           edk_lanczos_diag* diag) {
  EDK_CHECK_ARG(nops >= 1 && ops && opts && v0s && evals, "edk_batch_lanczos_e0: NULL argument");
  EDK_CHECK_ARG(v0_dtype == EDK_F64 || v0_dtype == EDK_C128,
                "edk_batch_lanczos_e0: v0s must be F64 or C128 (host)");
  EDK_CHECK_ARG(opts->max_steps >= 1 && opts->nev >= 1, "edk_batch_lanczos_e0: bad options");
  std::vector<edk_operator*> v(ops, ops + nops);
  int64_t tot = 0;
  for (auto* op : v) {
    EDK_CHECK_ARG(op != nullptr, "edk_batch_lanczos_e0: NULL operator");
    tot += op->b->D;
  }
  cudaStream_t st = v[0]->stream;
  size_t es = v0_dtype == EDK_F64 ? 8 : 16;
  DevBuf v0d;
  EDK_RETURN_IF(v0d.alloc((size_t)tot * es));
  EDK_TRY_CUDA(cudaMemcpyAsync(v0d.p, v0s, (size_t)tot * es, cudaMemcpyHostToDevice, st));
  std::vector<OpResult> res;
  EDK_RETURN_IF(batch_lanczos(v, *opts, v0d.p, v0_dtype, st, res, diag));
  for (int q = 0; q < nops; ++q)
    for (int k = 0; k < opts->nev; ++k)
      evals[(size_t)q * opts->nev + k] = k < (int)res[q].ev.size() ? res[q].ev[k] : NAN;
  return EDK_OK;
}
