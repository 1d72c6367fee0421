// edk_apply.cu — matrix-free H * x on the device.
//
// Reference semantics (src/Operator.jl:399-465): for every basis state j and
// every local term, each nonzero M[r, c] of the local column c = digits of j on
// the term's sites produces the target state s' (digits rewritten to r) and
//     H[pos, j] += M[r, c] * C(s') * R[pos] / R[j],    (C, pos) = index(b, s').
//
// Row-gather form (the default).  When every local term is Hermitian and the
// operator is invariant under the basis symmetries, H is Hermitian and
//     y[i] = sum_{nonzeros of column i}  conj(H[pos, i]) * x[pos],
// so one thread owns one output row: no atomics, no private copies, a
// deterministic summation order.  The column-scatter form (atomics) is kept
// for operators that are not Hermitian in the sector.
//
// Terms are compiled for the device into
//   * bond families: 2-site terms (i, i+d mod L) that share one 4x4 matrix,
//     evaluated on whole bit planes (X = s, Y = rotl(s, d), local column
//     c = 2X+Y), so the diagonal is four popcounts and the off-diagonal hits
//     are the set bits of one mask;
//   * generic terms: per-term local column, CSC list of XOR masks.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>

#include "edk_lookup.cuh"

namespace edk {

template <class VT> struct VTraits;
template <> struct VTraits<double> { using A = double; static constexpr bool cx = false; };
template <> struct VTraits<double2> { using A = double; static constexpr bool cx = true; };
template <> struct VTraits<float> { using A = float; static constexpr bool cx = false; };
template <> struct VTraits<float2> { using A = float; static constexpr bool cx = true; };

template <class A> struct Cx { A r, i; };
__device__ __forceinline__ Cx<double> ldv(const double* p) { return {__ldg(p), 0.0}; }
__device__ __forceinline__ Cx<double> ldv(const double2* p) { double2 v = __ldg(p); return {v.x, v.y}; }
__device__ __forceinline__ Cx<float> ldv(const float* p) { return {__ldg(p), 0.0f}; }
__device__ __forceinline__ Cx<float> ldv(const float2* p) { float2 v = __ldg(p); return {v.x, v.y}; }
__device__ __forceinline__ void stv(double* p, Cx<double> v) { *p = v.r; }
__device__ __forceinline__ void stv(double2* p, Cx<double> v) { *p = make_double2(v.r, v.i); }
__device__ __forceinline__ void stv(float* p, Cx<float> v) { *p = v.r; }
__device__ __forceinline__ void stv(float2* p, Cx<float> v) { *p = make_float2(v.r, v.i); }
__device__ __forceinline__ Cx<double> ldout(const double* p) { return {*p, 0.0}; }
__device__ __forceinline__ Cx<double> ldout(const double2* p) { double2 v = *p; return {v.x, v.y}; }
__device__ __forceinline__ Cx<float> ldout(const float* p) { return {*p, 0.0f}; }
__device__ __forceinline__ Cx<float> ldout(const float2* p) { float2 v = *p; return {v.x, v.y}; }
__device__ __forceinline__ void atv(double* p, Cx<double> v) { atomicAdd(p, v.r); }
__device__ __forceinline__ void atv(double2* p, Cx<double> v) {
  atomicAdd(&p->x, v.r); atomicAdd(&p->y, v.i);
}
__device__ __forceinline__ void atv(float* p, Cx<float> v) { atomicAdd(p, v.r); }
__device__ __forceinline__ void atv(float2* p, Cx<float> v) {
  atomicAdd(&p->x, v.r); atomicAdd(&p->y, v.i);
}

__device__ __forceinline__ void fill_binom32(uint32_t* s_binom) {
  for (int q = threadIdx.x; q < 32 * 33; q += blockDim.x) {
    int pp = q / 33, kk = q % 33;
    uint64_t c = 1;
    if (kk > pp) c = 0;
    else for (int r = 1; r <= kk; ++r) c = c * (uint64_t)(pp - kk + r) / (uint64_t)r;
    s_binom[q] = (uint32_t)c;
  }
}

// Visit every nonzero of column `s` of H: f_diag(dr, di) once with the summed
// diagonal, f_hit(hit, vr, vi) for each off-diagonal element found in the basis.
template <int BK, class S, class FHit>
__device__ __forceinline__ void expand_row(const BasisDev& b, const OpDev& op, S s,
                                           const uint32_t* s_binom, double& dr, double& di,
                                           FHit&& f_hit) {
  const S mask = (S)b.maskL;
  const int L = b.L;
  for (int f = 0; f < op.nfam; ++f) {
    const FamDev* F = op.fam + f;
    const int d = F->d;
    const S X = s, Y = rotl_L(s, d, L, mask);
    const S valid = (S)F->valid;
    S m[4];
    m[0] = (S)(~X & ~Y & valid);
    m[1] = (S)(~X & Y & valid);
    m[2] = (S)(X & ~Y & valid);
    m[3] = (S)(X & Y & valid);
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const double2 dv = F->dval[c];
      const int cnt = popc_s(m[c]);
      dr += dv.x * cnt;
      di += dv.y * cnt;
      const int nz = F->nnz[c];
      if (nz == 0) continue;
      S bits = m[c];
      while (bits) {
        const int p = ffs_s(bits);
        bits &= bits - 1;
        int pj = p - d;
        if (pj < 0) pj += L;
        for (int q = 0; q < nz; ++q) {
          const int xr = F->xr[c][q];
          const S flip = (S)((S)((xr >> 1) & 1) << p) | (S)((S)(xr & 1) << pj);
          Hit h;
          if (lookup<BK, S>(b, (S)(s ^ flip), s_binom, h)) {
            const double2 v = F->val[c][q];
            f_hit(h, v.x, v.y);
          }
        }
      }
    }
  }
  for (int t = 0; t < op.nterm; ++t) {
    const TermDev* T = op.term + t;
    const int ns = T->nsites;
    int c = 0;
    for (int k = 0; k < ns; ++k) c = (c << 1) | (int)((s >> T->bitpos[k]) & 1);
    const double2 dv = __ldg(op.dval + T->diag_off + c);
    dr += dv.x;
    di += dv.y;
    const int q0 = __ldg(op.colptr + T->col_off + c), q1 = __ldg(op.colptr + T->col_off + c + 1);
    for (int q = q0; q < q1; ++q) {
      Hit h;
      if (lookup<BK, S>(b, (S)(s ^ (S)__ldg(op.xmask + q)), s_binom, h)) {
        const double2 v = __ldg(op.val + q);
        f_hit(h, v.x, v.y);
      }
    }
  }
}

// y(:, k) (+)= H x(:, k); blockIdx.y = k.
template <int BK, class S, class VT, bool GATHER>
__global__ void __launch_bounds__(256) k_apply(BasisDev b, OpDev op, const VT* __restrict__ x,
                                               VT* __restrict__ y, int64_t ldx, int64_t ldy,
                                               int accumulate) {
  using A = typename VTraits<VT>::A;
  constexpr bool CX = VTraits<VT>::cx;
  __shared__ uint32_t s_binom[32 * 33];
  if constexpr (BK == BK_PROJ_RANK) {
    fill_binom32(s_binom);
    __syncthreads();
  }
  const VT* xk = x + (int64_t)blockIdx.y * ldx;
  VT* yk = y + (int64_t)blockIdx.y * ldy;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < b.D;
       i += (int64_t)gridDim.x * blockDim.x) {
    const S s = (BK == BK_TENSOR) ? (S)i : (S)__ldg(b.I + i);
    const A invRi = b.R ? (A)(1.0 / __ldg(b.R + i)) : (A)1;
    double dr = 0.0, di = 0.0;
    if constexpr (GATHER) {
      A ar = 0, ai = 0;
      expand_row<BK, S>(b, op, s, s_binom, dr, di, [&](const Hit& h, double vr, double vi) {
        const A pr = (A)h.pre, pi = (A)h.pim, v_r = (A)vr, v_i = (A)vi;
        const A ratio = (A)h.rpos * invRi;
        const A cr = (v_r * pr - v_i * pi) * ratio;
        const Cx<A> xv = ldv(xk + h.pos);
        if constexpr (CX) {
          const A ci = (v_r * pi + v_i * pr) * ratio;
          ar += cr * xv.r + ci * xv.i;   // conj(c) * x
          ai += cr * xv.i - ci * xv.r;
        } else {
          ar += cr * xv.r;
        }
      });
      const Cx<A> xi = ldv(xk + i);
      ar += (A)dr * xi.r + (A)di * xi.i;
      if constexpr (CX) ai += (A)dr * xi.i - (A)di * xi.r;
      Cx<A> out{ar, ai};
      if (accumulate) {
        const Cx<A> yo = ldout(yk + i);
        out.r += yo.r;
        out.i += yo.i;
      }
      stv(yk + i, out);
    } else {
      const Cx<A> xi = ldv(xk + i);
      const A xr_ = xi.r * invRi, xi_ = xi.i * invRi;  // coeff = v[j] / R[j]
      expand_row<BK, S>(b, op, s, s_binom, dr, di, [&](const Hit& h, double vr, double vi) {
        const A pr = (A)h.pre, pi = (A)h.pim, v_r = (A)vr, v_i = (A)vi;
        const A cr = (v_r * pr - v_i * pi) * (A)h.rpos;
        const A ci = (v_r * pi + v_i * pr) * (A)h.rpos;
        Cx<A> add{cr * xr_ - ci * xi_, cr * xi_ + ci * xr_};
        atv(yk + h.pos, add);
      });
      Cx<A> add{(A)dr * xi.r - (A)di * xi.i, (A)dr * xi.i + (A)di * xi.r};
      atv(yk + i, add);
    }
  }
}

// ---------------------------------------------------------------------------
// Fast path: every off-diagonal term is a flip-flop bond family (XXZ-like
// 2-site terms whose only off-diagonal entries swap the two digits), every
// other term is diagonal, L <= 32.  Each block owns 256 consecutive rows and
// first sorts them by their number of hits (a counting sort in shared
// memory), so the 32 lanes of a warp walk equally long hit lists; the hits
// are taken two at a time so the two canonicalisations overlap and their
// table probes and psi gathers are in flight together.
// ---------------------------------------------------------------------------
struct HitCtx {
  uint32_t key;     // canonical representative (or row for onsite kinds)
  double pre, pim;  // phase
};

template <int BK>
__device__ __forceinline__ void canon_ctx(const BasisDev& b, uint32_t s, HitCtx& c) {
  c.pre = 1.0;
  c.pim = 0.0;
  const uint32_t mask = (uint32_t)b.maskL;
  if constexpr (BK == BK_TRANS0) {
    c.key = b.runs_canon ? canon_runs32(s, b.L, mask) : canon_min32(s, b.L, b.A, b.len, mask);
  } else if constexpr (BK == BK_TRANS) {
    int M;
    c.key = canon_arg32(s, b.L, b.A, b.len, mask, M);
    const double2 ph = __ldg(b.phase + M);
    c.pre = ph.x;
    c.pim = ph.y;
  } else if constexpr (BK == BK_TRANSPAR) {
    uint32_t Iam, Ibm;
    int Rr, M;
    canon_par32(s, b.L, b.A, b.len, mask, Iam, Rr, Ibm, M);
    if (Ibm < Iam) { c.key = Ibm; c.pre = (double)b.P * __ldg(b.phase + M).x; }
    else { c.key = Iam; c.pre = __ldg(b.phase + Rr).x; }
  } else {
    c.key = s;
  }
}

__device__ __forceinline__ uint64_t first_slot(const BasisDev& b, uint32_t key) {
  return hslot32(key, b.hbits);
}
// finish a probe sequence whose first entry `e` (at `slot`) is already loaded
__device__ __forceinline__ bool probe_rest(const BasisDev& b, uint32_t key, unsigned long long e,
                                           uint64_t slot, uint32_t& val) {
  const unsigned long long* tab = reinterpret_cast<const unsigned long long*>(b.htab);
  for (uint64_t n = 0; n <= b.hmask; ++n) {
    if (e == ~0ull) return false;
    if ((uint32_t)(e >> 32) == key) { val = (uint32_t)e; return true; }
    slot = (slot + 1) & b.hmask;
    e = __ldg(tab + slot);
  }
  return false;
}

// (pos, rpos) of two canonical keys, both table probes issued together
template <int BK>
__device__ __forceinline__ void locate2(const BasisDev& b, const uint32_t* s_binom, uint32_t k1,
                                        uint32_t k2, bool two, int64_t& p1, double& r1,
                                        bool& ok1, int64_t& p2, double& r2, bool& ok2) {
  r1 = r2 = 1.0;
  if constexpr (BK == BK_TENSOR) {
    p1 = k1; p2 = k2; ok1 = true; ok2 = two;
  } else if constexpr (BK == BK_PROJ_RANK) {
    ok1 = __popc(k1) == b.K;
    ok2 = two && __popc(k2) == b.K;
    p1 = ok1 ? colex_rank(k1, s_binom) : 0;
    p2 = ok2 ? colex_rank(k2, s_binom) : 0;
  } else {
    const unsigned long long* tab = reinterpret_cast<const unsigned long long*>(b.htab);
    const uint64_t q1 = first_slot(b, k1), q2 = first_slot(b, k2);
    const unsigned long long e1 = __ldg(tab + q1);
    const unsigned long long e2 = two ? __ldg(tab + q2) : ~0ull;
    uint32_t v1 = 0, v2 = 0;
    ok1 = probe_rest(b, k1, e1, q1, v1);
    ok2 = two && probe_rest(b, k2, e2, q2, v2);
    if constexpr (BK == BK_PROJ_HASH) {
      p1 = b.packed ? (int64_t)(v1 >> 5) : (int64_t)v1;
      p2 = b.packed ? (int64_t)(v2 >> 5) : (int64_t)v2;
    } else {
      p1 = p2 = 0;
      if (ok1) decode_val(b, v1, p1, r1);
      if (ok2) decode_val(b, v2, p2, r2);
    }
  }
}

constexpr int kMaxFF = 4;
struct FFParams {
  int nfam;
  int d[kMaxFF];
  uint32_t valid[kMaxFF];
  double2 dval[kMaxFF][4];
  double2 v1[kMaxFF];  // M[2][1]: local column "01" -> row "10"
  double2 v2[kMaxFF];  // M[1][2]: local column "10" -> row "01"
};

template <int BK, class VT>
__global__ void __launch_bounds__(256) k_apply_ff(BasisDev b, OpDev op, FFParams ff,
                                                  const VT* __restrict__ x, VT* __restrict__ y,
                                                  int64_t ldx, int64_t ldy, int accumulate) {
  using A = typename VTraits<VT>::A;
  constexpr bool CX = VTraits<VT>::cx;
  __shared__ uint32_t s_binom[(BK == BK_PROJ_RANK) ? 32 * 33 : 1];
  __shared__ int s_hist[64];
  __shared__ unsigned short s_order[256];
  __shared__ uint32_t s_state[256];
  if constexpr (BK == BK_PROJ_RANK) fill_binom32(s_binom);
  const int t = threadIdx.x;
  if (t < 64) s_hist[t] = 0;
  __syncthreads();
  const uint32_t mask = (uint32_t)b.maskL;
  const int L = b.L;
  const int64_t r0 = (int64_t)blockIdx.x * 256;
  uint32_t s = 0;
  int key = 0;
  if (r0 + t < b.D) {
    s = (BK == BK_TENSOR) ? (uint32_t)(r0 + t) : (uint32_t)__ldg(b.I + r0 + t);
    for (int f = 0; f < ff.nfam; ++f)
      key += __popc((s ^ rotl_L(s, ff.d[f], L, mask)) & ff.valid[f]);
  }
  key = min(key, 63);
  s_state[t] = s;
  const int slot = atomicAdd(&s_hist[key], 1);
  __syncthreads();
  if (t < 32) {  // exclusive scan over the 64 bins
    const int a = s_hist[2 * t], c = s_hist[2 * t + 1];
    int sum = a + c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int v = __shfl_up_sync(0xffffffffu, sum, o);
      if (t >= o) sum += v;
    }
    const int excl = sum - (a + c);
    s_hist[2 * t] = excl;
    s_hist[2 * t + 1] = excl + a;
  }
  __syncthreads();
  s_order[s_hist[key] + slot] = (unsigned short)t;
  __syncthreads();
  const int tt = s_order[t];
  const int64_t i = r0 + tt;
  if (i >= b.D) return;
  const uint32_t st = s_state[tt];
  const VT* xk = x + (int64_t)blockIdx.y * ldx;
  VT* yk = y + (int64_t)blockIdx.y * ldy;
  const A invRi = b.R ? (A)(1.0 / __ldg(b.R + i)) : (A)1;
  double dr = 0.0, di = 0.0;
  A ar = 0, ai = 0;
  auto acc = [&](const HitCtx& c, double rpos, double vr, double vi, Cx<A> xv) {
    const A pr = (A)c.pre, pi = (A)c.pim, v_r = (A)vr, v_i = (A)vi;
    const A ratio = (A)rpos * invRi;
    const A cr = (v_r * pr - v_i * pi) * ratio;
    if constexpr (CX) {
      const A ci = (v_r * pi + v_i * pr) * ratio;
      ar += cr * xv.r + ci * xv.i;
      ai += cr * xv.i - ci * xv.r;
    } else {
      ar += cr * xv.r;
    }
  };
  for (int f = 0; f < ff.nfam; ++f) {
    const int d = ff.d[f];
    const uint32_t X = st, Y = rotl_L(st, d, L, mask), V = ff.valid[f];
    const uint32_t m1 = ~X & Y & V, m2 = X & ~Y & V;
    const int c0 = __popc(~X & ~Y & V), c1 = __popc(m1), c2 = __popc(m2), c3 = __popc(X & Y & V);
    dr += ff.dval[f][0].x * c0 + ff.dval[f][1].x * c1 + ff.dval[f][2].x * c2 + ff.dval[f][3].x * c3;
    di += ff.dval[f][0].y * c0 + ff.dval[f][1].y * c1 + ff.dval[f][2].y * c2 + ff.dval[f][3].y * c3;
    const double2 va = ff.v1[f], vb = ff.v2[f];
    uint32_t bits = m1 | m2;
    while (bits) {
      const int p1 = __ffs(bits) - 1;
      bits &= bits - 1;
      const bool two = bits != 0;
      const int p2 = two ? __ffs(bits) - 1 : p1;
      if (two) bits &= bits - 1;
      const int q1 = p1 >= d ? p1 - d : p1 - d + L, q2 = p2 >= d ? p2 - d : p2 - d + L;
      const uint32_t s1 = st ^ (1u << p1) ^ (1u << q1), s2 = st ^ (1u << p2) ^ (1u << q2);
      HitCtx h1, h2;
      canon_ctx<BK>(b, s1, h1);
      canon_ctx<BK>(b, s2, h2);
      int64_t pos1, pos2;
      double rp1, rp2;
      bool ok1, ok2;
      locate2<BK>(b, s_binom, h1.key, h2.key, two, pos1, rp1, ok1, pos2, rp2, ok2);
      const Cx<A> x1 = ok1 ? ldv(xk + pos1) : Cx<A>{0, 0};
      const Cx<A> x2 = ok2 ? ldv(xk + pos2) : Cx<A>{0, 0};
      const double2 w1 = ((st >> p1) & 1u) ? vb : va;
      const double2 w2 = ((st >> p2) & 1u) ? vb : va;
      if (ok1) acc(h1, rp1, w1.x, w1.y, x1);
      if (ok2) acc(h2, rp2, w2.x, w2.y, x2);
    }
  }
  for (int q = 0; q < op.nterm; ++q) {  // diagonal-only terms (fields, zz on other sites)
    const TermDev* T = op.term + q;
    int c = 0;
    for (int k = 0; k < T->nsites; ++k) c = (c << 1) | (int)((st >> T->bitpos[k]) & 1u);
    const double2 dv = __ldg(op.dval + T->diag_off + c);
    dr += dv.x;
    di += dv.y;
  }
  const Cx<A> xi = ldv(xk + i);
  ar += (A)dr * xi.r + (A)di * xi.i;
  if constexpr (CX) ai += (A)dr * xi.i - (A)di * xi.r;
  Cx<A> out{ar, ai};
  if (accumulate) {
    const Cx<A> yo = ldout(yk + i);
    out.r += yo.r;
    out.i += yo.i;
  }
  stv(yk + i, out);
}

namespace {

int apply_grid(int64_t D) {
  int64_t g = (D + 255) / 256;
  if (g < 1) g = 1;
  if (g > 148 * 64) g = 148 * 64;
  return (int)g;
}

template <class VT>
edk_status launch_apply_ff(const BasisDev& b, const OpDev& op, const FFParams& ff, const void* x,
                           void* y, int64_t nvec, int64_t ldx, int64_t ldy, int accumulate,
                           cudaStream_t st) {
  const VT* X = static_cast<const VT*>(x);
  VT* Y = static_cast<VT*>(y);
  for (int64_t k0 = 0; k0 < nvec; k0 += 65535) {
    int64_t nk = std::min<int64_t>(nvec - k0, 65535);
    dim3 grid((unsigned)((b.D + 255) / 256), (unsigned)nk);
    const VT* Xk = X + k0 * ldx;
    VT* Yk = Y + k0 * ldy;
#define EDK_FF(BK)                                                                         \
  case BK:                                                                                 \
    k_apply_ff<BK, VT><<<grid, 256, 0, st>>>(b, op, ff, Xk, Yk, ldx, ldy, accumulate);     \
    break;
    switch (b.bk) {
      EDK_FF(BK_TENSOR)
      EDK_FF(BK_PROJ_RANK)
      EDK_FF(BK_PROJ_HASH)
      EDK_FF(BK_TRANS0)
      EDK_FF(BK_TRANS)
      EDK_FF(BK_TRANSPAR)
      default:
        set_error("apply: fast path not available for this basis");
        return EDK_INVALID_ARG;
    }
#undef EDK_FF
    EDK_TRY_CUDA(cudaGetLastError());
  }
  return EDK_OK;
}

template <class VT, bool GATHER>
edk_status launch_apply(const BasisDev& b, const OpDev& op, const void* x, void* y, int64_t nvec,
                        int64_t ldx, int64_t ldy, int accumulate, cudaStream_t st) {
  const VT* X = static_cast<const VT*>(x);
  VT* Y = static_cast<VT*>(y);
  bool wide = b.L > 32;
  for (int64_t k0 = 0; k0 < nvec; k0 += 65535) {
    int64_t nk = std::min<int64_t>(nvec - k0, 65535);
    dim3 grid(apply_grid(b.D), (unsigned)nk);
    const VT* Xk = X + k0 * ldx;
    VT* Yk = Y + k0 * ldy;
#define EDK_APPLY(BK)                                                                       \
  case BK:                                                                                  \
    if (wide) k_apply<BK, uint64_t, VT, GATHER><<<grid, 256, 0, st>>>(b, op, Xk, Yk, ldx, ldy, \
                                                                       accumulate);         \
    else k_apply<BK, uint32_t, VT, GATHER><<<grid, 256, 0, st>>>(b, op, Xk, Yk, ldx, ldy,   \
                                                                  accumulate);              \
    break;
    switch (b.bk) {
      EDK_APPLY(BK_TENSOR)
      EDK_APPLY(BK_PROJ_RANK)
      EDK_APPLY(BK_PROJ_HASH)
      EDK_APPLY(BK_TRANS0)
      EDK_APPLY(BK_TRANS)
      EDK_APPLY(BK_TRANSPAR)
      EDK_APPLY(BK_ABELIAN)
      default:
        set_error("apply: unknown basis lookup kind");
        return EDK_INVALID_ARG;
    }
#undef EDK_APPLY
    EDK_TRY_CUDA(cudaGetLastError());
  }
  return EDK_OK;
}

size_t dtype_size(int dtype) {
  switch (dtype) {
    case EDK_F64: return 8;
    case EDK_C128: return 16;
    case EDK_F32: return 4;
    case EDK_C64: return 8;
  }
  return 0;
}

}  // namespace

edk_status apply_device(edk_operator* op, int dtype, const void* x, void* y, int64_t nvec,
                        int64_t ldx, int64_t ldy, int accumulate, cudaStream_t st) {
  const BasisDev& b = op->b->dev;
  if (nvec <= 0 || b.D == 0) return EDK_OK;
  EDK_RETURN_IF(check_basis_dev(b));
  if (!op->gather && !accumulate) {
    // column scatter accumulates with atomics: start from zero
    size_t es = dtype_size(dtype);
    EDK_TRY_CUDA(cudaMemset2DAsync(y, ldy * es, 0, b.D * es, nvec, st));
  }
  bool sc = !op->gather;
  if (op->ff_ok && !sc && op->use_ff) {
    const FFParams& ff = *reinterpret_cast<const FFParams*>(op->ff_params.data());
    switch (dtype) {
      case EDK_F64: return launch_apply_ff<double>(b, op->dev, ff, x, y, nvec, ldx, ldy, accumulate, st);
      case EDK_C128: return launch_apply_ff<double2>(b, op->dev, ff, x, y, nvec, ldx, ldy, accumulate, st);
      case EDK_F32: return launch_apply_ff<float>(b, op->dev, ff, x, y, nvec, ldx, ldy, accumulate, st);
      case EDK_C64: return launch_apply_ff<float2>(b, op->dev, ff, x, y, nvec, ldx, ldy, accumulate, st);
    }
  }
  switch (dtype) {
    case EDK_F64:
      return sc ? launch_apply<double, false>(b, op->dev, x, y, nvec, ldx, ldy, 1, st)
                : launch_apply<double, true>(b, op->dev, x, y, nvec, ldx, ldy, accumulate, st);
    case EDK_C128:
      return sc ? launch_apply<double2, false>(b, op->dev, x, y, nvec, ldx, ldy, 1, st)
                : launch_apply<double2, true>(b, op->dev, x, y, nvec, ldx, ldy, accumulate, st);
    case EDK_F32:
      return sc ? launch_apply<float, false>(b, op->dev, x, y, nvec, ldx, ldy, 1, st)
                : launch_apply<float, true>(b, op->dev, x, y, nvec, ldx, ldy, accumulate, st);
    case EDK_C64:
      return sc ? launch_apply<float2, false>(b, op->dev, x, y, nvec, ldx, ldy, 1, st)
                : launch_apply<float2, true>(b, op->dev, x, y, nvec, ldx, ldy, accumulate, st);
  }
  set_error("apply: unknown dtype");
  return EDK_INVALID_ARG;
}

// ---------------------------------------------------------------------------
// Operator compilation (host)
// ---------------------------------------------------------------------------
namespace {

struct HostTerm {
  std::vector<int> sites;           // 1-based
  int dim = 0;
  std::vector<double> re, im;       // dense, row-major M[r*dim + c]
};

double term_scale(const HostTerm& t) {
  double m = 0;
  for (size_t q = 0; q < t.re.size(); ++q) m = std::max(m, std::hypot(t.re[q], t.im[q]));
  return m;
}

bool term_hermitian(const HostTerm& t) {
  double tol = 1e-12 * std::max(1.0, term_scale(t));
  for (int r = 0; r < t.dim; ++r)
    for (int c = 0; c < t.dim; ++c) {
      double dr = t.re[r * t.dim + c] - t.re[c * t.dim + r];
      double di = t.im[r * t.dim + c] + t.im[c * t.dim + r];
      if (std::hypot(dr, di) > tol) return false;
    }
  return true;
}

// Canonical form: sites sorted ascending, tensor factors permuted to match.
HostTerm canonical(const HostTerm& t) {
  int ns = (int)t.sites.size();
  std::vector<int> order(ns);
  for (int k = 0; k < ns; ++k) order[k] = k;
  std::sort(order.begin(), order.end(), [&](int a, int b) { return t.sites[a] < t.sites[b]; });
  HostTerm o;
  o.dim = t.dim;
  o.sites.resize(ns);
  for (int k = 0; k < ns; ++k) o.sites[k] = t.sites[order[k]];
  o.re.assign(t.re.size(), 0.0);
  o.im.assign(t.im.size(), 0.0);
  // new local index bit (ns-1-k) holds old factor order[k] whose bit is (ns-1-order[k])
  auto remap = [&](int idx) {
    int out = 0;
    for (int k = 0; k < ns; ++k) {
      int bit = (idx >> (ns - 1 - order[k])) & 1;
      out |= bit << (ns - 1 - k);
    }
    return out;
  };
  for (int r = 0; r < t.dim; ++r)
    for (int c = 0; c < t.dim; ++c) {
      int nr = remap(r), nc = remap(c);
      o.re[nr * t.dim + nc] = t.re[r * t.dim + c];
      o.im[nr * t.dim + nc] = t.im[r * t.dim + c];
    }
  return o;
}

using TermMap = std::map<std::vector<int>, std::pair<std::vector<double>, std::vector<double>>>;

void add_term(TermMap& m, const HostTerm& t) {
  HostTerm c = canonical(t);
  auto it = m.find(c.sites);
  if (it == m.end()) {
    m[c.sites] = {c.re, c.im};
  } else {
    for (size_t q = 0; q < c.re.size(); ++q) {
      it->second.first[q] += c.re[q];
      it->second.second[q] += c.im[q];
    }
  }
}

// Is sum_t M_t invariant under (site permutation perm, inversion flags inv)?
bool invariant(const std::vector<HostTerm>& terms, const std::vector<int>& perm,
               const std::vector<uint8_t>& inv) {
  TermMap a, b;
  double scale = 0;
  for (auto& t : terms) {
    add_term(a, t);
    scale = std::max(scale, term_scale(t));
    HostTerm g;
    g.dim = t.dim;
    int ns = (int)t.sites.size();
    g.sites.resize(ns);
    int fmask = 0;
    for (int k = 0; k < ns; ++k) {
      g.sites[k] = perm[t.sites[k] - 1];
      if (inv[g.sites[k] - 1]) fmask |= 1 << (ns - 1 - k);
    }
    g.re.resize(t.re.size());
    g.im.resize(t.im.size());
    for (int r = 0; r < t.dim; ++r)
      for (int c = 0; c < t.dim; ++c) {
        g.re[(r ^ fmask) * t.dim + (c ^ fmask)] = t.re[r * t.dim + c];
        g.im[(r ^ fmask) * t.dim + (c ^ fmask)] = t.im[r * t.dim + c];
      }
    add_term(b, g);
  }
  double tol = 1e-12 * std::max(1.0, scale);
  auto cmp = [&](const TermMap& x, const TermMap& y) {
    for (auto& kv : x) {
      auto it = y.find(kv.first);
      for (size_t q = 0; q < kv.second.first.size(); ++q) {
        double yr = (it == y.end()) ? 0.0 : it->second.first[q];
        double yi = (it == y.end()) ? 0.0 : it->second.second[q];
        if (std::hypot(kv.second.first[q] - yr, kv.second.second[q] - yi) > tol) return false;
      }
    }
    return true;
  };
  return cmp(a, b) && cmp(b, a);
}

}  // namespace
}  // namespace edk

using namespace edk;

edk_operator::~edk_operator() {
  if (stream) cudaStreamDestroy(stream);
}

extern "C" edk_status edk_operator_create(edk_basis* b, int32_t nterms, const int32_t* nsites,
                                          const int32_t* sites, const int64_t* nnz,
                                          const int64_t* colptr, const int64_t* rowval,
                                          const double* nzval, edk_operator** out) {
  EDK_CHECK_ARG(out != nullptr, "edk_operator_create: out is NULL");
  *out = nullptr;
  EDK_CHECK_ARG(b != nullptr, "edk_operator_create: basis is NULL");
  EDK_CHECK_ARG(nterms >= 0, "edk_operator_create: nterms < 0");
  EDK_CHECK_ARG(nterms == 0 || (nsites && sites && nnz && colptr && rowval && nzval),
                "edk_operator_create: NULL term array");
  const int L = b->L;
  std::vector<HostTerm> terms;
  size_t so = 0, co = 0, no = 0;
  for (int t = 0; t < nterms; ++t) {
    int ns = nsites[t];
    EDK_CHECK_ARG(ns >= 1 && ns <= 8, "edk_operator_create: a term must act on 1..8 sites");
    HostTerm h;
    h.sites.assign(sites + so, sites + so + ns);
    so += ns;
    std::vector<int> seen(L + 1, 0);
    for (int s : h.sites) {
      EDK_CHECK_ARG(s >= 1 && s <= L, "edk_operator_create: site outside 1:L");
      EDK_CHECK_ARG(!seen[s], "edk_operator_create: repeated site in one term");
      seen[s] = 1;
    }
    h.dim = 1 << ns;
    h.re.assign(h.dim * h.dim, 0.0);
    h.im.assign(h.dim * h.dim, 0.0);
    int64_t nz = nnz[t];
    EDK_CHECK_ARG(nz >= 0, "edk_operator_create: nnz < 0");
    for (int c = 0; c < h.dim; ++c) {
      int64_t q0 = colptr[co + c], q1 = colptr[co + c + 1];
      EDK_CHECK_ARG(q0 >= 1 && q1 >= q0 && q1 - 1 <= nz, "edk_operator_create: bad colptr");
      for (int64_t q = q0; q < q1; ++q) {
        int64_t r = rowval[no + q - 1];
        EDK_CHECK_ARG(r >= 1 && r <= h.dim, "edk_operator_create: bad rowval");
        h.re[(r - 1) * h.dim + c] += nzval[2 * (no + q - 1)];
        h.im[(r - 1) * h.dim + c] += nzval[2 * (no + q - 1) + 1];
      }
    }
    co += h.dim + 1;
    no += nz;
    terms.push_back(std::move(h));
  }
  auto* op = new edk_operator;
  std::unique_ptr<edk_operator> guard(op);
  op->b = b;
  // properties
  bool cplx = b->phase_complex;
  for (auto& t : terms)
    for (double v : t.im) cplx |= v != 0.0;
  bool herm = true;
  for (auto& t : terms) herm &= term_hermitian(t);
  if (herm && b->kind != EDK_TENSOR && b->kind != EDK_PROJECTED) {
    std::vector<uint8_t> noinv(L, 0);
    if (b->kind == EDK_TRANSLATIONAL || b->kind == EDK_TRANSPARITY) {
      std::vector<int> tr(L);
      for (int i = 1; i <= L; ++i) tr[i - 1] = (i - 1 + b->A) % L + 1;
      herm &= invariant(terms, tr, noinv);
      if (b->kind == EDK_TRANSPARITY) {
        std::vector<int> rv(L);
        for (int i = 1; i <= L; ++i) rv[i - 1] = L - i + 1;
        herm &= invariant(terms, rv, noinv);
      }
    } else {
      for (size_t g = 0; g < b->gen_perm.size(); ++g)
        herm &= invariant(terms, b->gen_perm[g], b->gen_inv[g]);
    }
  }
  op->gather = herm;
  op->is_complex = cplx;
  if (const char* e = std::getenv("EDK_DISABLE_FAST")) op->use_ff = !(e[0] == '1');
  // families of 2-site terms with one shared matrix
  std::map<std::pair<int, std::vector<double>>, std::vector<int>> groups;
  for (size_t t = 0; t < terms.size(); ++t) {
    if (terms[t].sites.size() != 2) continue;
    int d = ((terms[t].sites[1] - terms[t].sites[0]) % L + L) % L;
    std::vector<double> key(terms[t].re);
    key.insert(key.end(), terms[t].im.begin(), terms[t].im.end());
    groups[{d, key}].push_back((int)t);
  }
  std::vector<char> in_family(terms.size(), 0);
  std::vector<FamDev> fams;
  for (auto& kv : groups) {
    if (kv.second.size() < 3) continue;
    FamDev F{};
    F.d = kv.first.first;
    const HostTerm& t0 = terms[kv.second[0]];
    for (int t : kv.second) {
      F.valid |= 1ull << (L - terms[t].sites[0]);
      in_family[t] = 1;
    }
    for (int c = 0; c < 4; ++c) {
      F.dval[c] = make_double2(t0.re[c * 4 + c], t0.im[c * 4 + c]);
      int n = 0;
      for (int r = 0; r < 4; ++r) {
        if (r == c) continue;
        double vr = t0.re[r * 4 + c], vi = t0.im[r * 4 + c];
        if (vr == 0.0 && vi == 0.0) continue;
        F.xr[c][n] = c ^ r;
        F.val[c][n] = make_double2(vr, vi);
        ++n;
      }
      F.nnz[c] = n;
    }
    fams.push_back(F);
  }
  std::vector<TermDev> tds;
  std::vector<int> cp;
  std::vector<uint64_t> xm;
  std::vector<double2> vals, dvals;
  for (size_t t = 0; t < terms.size(); ++t) {
    if (in_family[t]) continue;
    const HostTerm& h = terms[t];
    TermDev td{};
    int ns = (int)h.sites.size();
    td.nsites = ns;
    for (int k = 0; k < ns; ++k) td.bitpos[k] = L - h.sites[k];
    td.col_off = (int)cp.size();
    td.diag_off = (int)dvals.size();
    for (int c = 0; c < h.dim; ++c) {
      cp.push_back((int)xm.size());
      dvals.push_back(make_double2(h.re[c * h.dim + c], h.im[c * h.dim + c]));
      for (int r = 0; r < h.dim; ++r) {
        if (r == c) continue;
        double vr = h.re[r * h.dim + c], vi = h.im[r * h.dim + c];
        if (vr == 0.0 && vi == 0.0) continue;
        int x = c ^ r;
        uint64_t mask = 0;
        for (int k = 0; k < ns; ++k)
          if ((x >> (ns - 1 - k)) & 1) mask |= 1ull << td.bitpos[k];
        xm.push_back(mask);
        vals.push_back(make_double2(vr, vi));
      }
    }
    cp.push_back((int)xm.size());
    tds.push_back(td);
  }
  op->nfam = (int)fams.size();
  op->ngeneric = (int)tds.size();
  // flip-flop fast path eligibility
  {
    bool ok = L <= 32 && op->gather && b->dev.bk != BK_ABELIAN && !fams.empty() &&
              fams.size() <= (size_t)kMaxFF && xm.empty();
    for (const FamDev& F : fams)
      ok = ok && F.nnz[0] == 0 && F.nnz[3] == 0 && F.nnz[1] == 1 && F.nnz[2] == 1 &&
           F.xr[1][0] == 3 && F.xr[2][0] == 3;
    op->ff_ok = ok;
    if (ok) {
      FFParams ff{};
      ff.nfam = (int)fams.size();
      for (size_t f = 0; f < fams.size(); ++f) {
        ff.d[f] = fams[f].d;
        ff.valid[f] = (uint32_t)fams[f].valid;
        for (int c = 0; c < 4; ++c) ff.dval[f][c] = fams[f].dval[c];
        ff.v1[f] = fams[f].val[1][0];
        ff.v2[f] = fams[f].val[2][0];
      }
      op->ff_params.resize(sizeof(FFParams));
      std::memcpy(op->ff_params.data(), &ff, sizeof(FFParams));
    }
  }
  auto upload = [&](DevBuf& buf, const void* src, size_t bytes) -> edk_status {
    if (bytes == 0) return EDK_OK;
    EDK_RETURN_IF(buf.alloc(bytes));
    EDK_TRY_CUDA(cudaMemcpy(buf.p, src, bytes, cudaMemcpyHostToDevice));
    return EDK_OK;
  };
  EDK_RETURN_IF(upload(op->fam, fams.data(), fams.size() * sizeof(FamDev)));
  EDK_RETURN_IF(upload(op->term, tds.data(), tds.size() * sizeof(TermDev)));
  EDK_RETURN_IF(upload(op->colptr, cp.data(), cp.size() * sizeof(int)));
  EDK_RETURN_IF(upload(op->xmask, xm.data(), xm.size() * sizeof(uint64_t)));
  EDK_RETURN_IF(upload(op->val, vals.data(), vals.size() * sizeof(double2)));
  EDK_RETURN_IF(upload(op->dval, dvals.data(), dvals.size() * sizeof(double2)));
  op->dev.nfam = op->nfam;
  op->dev.fam = op->fam.as<FamDev>();
  op->dev.nterm = op->ngeneric;
  op->dev.term = op->term.as<TermDev>();
  op->dev.colptr = op->colptr.as<int>();
  op->dev.xmask = op->xmask.as<uint64_t>();
  op->dev.val = op->val.as<double2>();
  op->dev.dval = op->dval.as<double2>();
  EDK_TRY_CUDA(cudaStreamCreateWithFlags(&op->stream, cudaStreamNonBlocking));
  *out = guard.release();
  return EDK_OK;
}

extern "C" edk_status edk_operator_destroy(edk_operator* op) {
  delete op;
  return EDK_OK;
}

extern "C" edk_status edk_operator_info(const edk_operator* op, int32_t* gather,
                                        int32_t* is_complex, int32_t* n_families,
                                        int32_t* n_generic) {
  EDK_CHECK_ARG(op != nullptr, "edk_operator_info: NULL operator");
  if (gather) *gather = op->gather ? 1 : 0;
  if (is_complex) *is_complex = op->is_complex ? 1 : 0;
  if (n_families) *n_families = op->nfam;
  if (n_generic) *n_generic = op->ngeneric;
  return EDK_OK;
}

static edk_status check_dtype(const edk_operator* op, int dtype) {
  EDK_CHECK_ARG(dtype >= EDK_F64 && dtype <= EDK_C64, "apply: unknown dtype");
  if (op->is_complex && (dtype == EDK_F64 || dtype == EDK_F32)) {
    set_error("apply: the operator has complex matrix elements; use a complex dtype");
    return EDK_INVALID_ARG;
  }
  return EDK_OK;
}

extern "C" edk_status edk_apply_async(edk_operator* op, int32_t dtype, const void* x, void* y,
                                      int64_t nvec, int64_t ldx, int64_t ldy, int32_t accumulate,
                                      void* stream) {
  EDK_CHECK_ARG(op && x && y, "edk_apply_async: NULL argument");
  EDK_RETURN_IF(check_dtype(op, dtype));
  EDK_CHECK_ARG(nvec >= 0 && ldx >= op->b->D && ldy >= op->b->D, "edk_apply_async: bad ld");
  return apply_device(op, dtype, x, y, nvec, ldx, ldy, accumulate,
                      static_cast<cudaStream_t>(stream));
}

extern "C" edk_status edk_apply(edk_operator* op, int32_t dtype, const void* x, void* y,
                                int64_t nvec, int64_t ldx, int64_t ldy, int32_t accumulate,
                                int32_t ptr_kind) {
  EDK_CHECK_ARG(op && x && y, "edk_apply: NULL argument");
  EDK_RETURN_IF(check_dtype(op, dtype));
  const int64_t D = op->b->D;
  EDK_CHECK_ARG(nvec >= 0 && ldx >= D && ldy >= D, "edk_apply: ldx/ldy smaller than the dimension");
  std::lock_guard<std::mutex> lk(op->mu);
  cudaStream_t st = op->stream;
  if (ptr_kind == EDK_DEVICE) {
    EDK_RETURN_IF(apply_device(op, dtype, x, y, nvec, ldx, ldy, accumulate, st));
    EDK_TRY_CUDA(cudaStreamSynchronize(st));
    return EDK_OK;
  }
  EDK_CHECK_ARG(ptr_kind == EDK_HOST, "edk_apply: bad ptr_kind");
  if (nvec == 0 || D == 0) return EDK_OK;
  size_t es = dtype_size(dtype);
  DevBuf& dx = op->hx;
  DevBuf& dy = op->hy;
  size_t need = (size_t)D * nvec * es;
  if (dx.bytes < need) EDK_RETURN_IF(dx.alloc(need));
  if (dy.bytes < need) EDK_RETURN_IF(dy.alloc(need));
  EDK_TRY_CUDA(cudaMemcpy2DAsync(dx.p, D * es, x, ldx * es, D * es, nvec, cudaMemcpyHostToDevice, st));
  if (accumulate)
    EDK_TRY_CUDA(cudaMemcpy2DAsync(dy.p, D * es, y, ldy * es, D * es, nvec, cudaMemcpyHostToDevice, st));
  EDK_RETURN_IF(apply_device(op, dtype, dx.p, dy.p, nvec, D, D, accumulate, st));
  EDK_TRY_CUDA(cudaMemcpy2DAsync(y, ldy * es, dy.p, D * es, D * es, nvec, cudaMemcpyDeviceToHost, st));
  EDK_TRY_CUDA(cudaStreamSynchronize(st));
  return EDK_OK;
}
