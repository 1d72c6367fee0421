// edk_rows.cuh — per-row bodies of the matvec kernels, shared by the single
// operator kernels (edk_apply.cu) and the batched ones (edk_batch.cu).
#pragma once

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

// One output row of the general kernels: gather form y[i] (+)= sum conj(H[pos,i]) x[pos],
// or scatter form y[pos] += H[pos,i] x[i] (atomics).
template <int BK, class S, class VT, bool GATHER>
__device__ __forceinline__ void gen_row(const BasisDev& b, const OpDev& op, int64_t i,
                                        const VT* __restrict__ xk, VT* __restrict__ yk,
                                        int accumulate, const uint32_t* s_binom) {
  using A = typename VTraits<VT>::A;
  constexpr bool CX = VTraits<VT>::cx;
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
    uint32_t v1 = 0, v2 = 0;
    if (b.search == 1) {
      ok1 = sorted_find32(b, k1, v1);
      ok2 = two && sorted_find32(b, k2, v2);
    } else {
      const unsigned long long* tab = reinterpret_cast<const unsigned long long*>(b.htab);
      const uint64_t q1 = first_slot(b, k1), q2 = first_slot(b, k2);
      const unsigned long long e1 = __ldg(tab + q1);
      const unsigned long long e2 = two ? __ldg(tab + q2) : ~0ull;
      ok1 = probe_rest(b, k1, e1, q1, v1);
      ok2 = two && probe_rest(b, k2, e2, q2, v2);
    }
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

// Colex rank of s with the set bit and the empty bit at positions p, q
// exchanged, from the rank rs of s: the moving bit keeps its place among the
// set bits below min(p, q), the set bits strictly between the two positions
// shift their index by one.  Adjacent positions cost one table read; the
// wrap-around bond walks the set bits in between.  binom[p * 33 + k] = C(p, k).
__device__ __forceinline__ uint32_t rank_after_swap(uint32_t s, uint32_t rs, int p, int q,
                                                    const uint32_t* binom) {
  const int a = min(p, q), c = max(p, q);  // a < c <= 31
  const int j = __popc(s & ((1u << a) - 1u));
  uint32_t between = s & ((1u << c) - 1u) & ~((2u << a) - 1u);
  const int nb = __popc(between);
  // the bit at a moves up to c: C(c, j+1+nb) - C(a, j+1), and every bit in
  // between drops from index j+1+k to j+k
  uint32_t delta = binom[c * 33 + j + 1 + nb] - binom[a * 33 + j + 1];
  for (int k = 1; between; ++k) {
    const int r = __ffs(between) - 1;
    between &= between - 1;
    delta += binom[r * 33 + j + k] - binom[r * 33 + j + 1 + k];
  }
  return ((s >> a) & 1u) ? rs + delta : rs - delta;  // modulo 2^32: the result is a valid rank
}

// 256 / TPS consecutive rows r0.. of the flip-flop fast path (one block of
// 256 threads).  Rows are sorted by their number of off-diagonal hits so that
// the lanes of a warp loop equally long; TPS adjacent lanes share one row and
// take its pairs of hits in turn (threads per state, picked by the
// autotuner), then reduce with shuffles.
template <int BK, class VT, int TPS = 1>
__device__ __forceinline__ void ff_tile(const BasisDev& b, const OpDev& op, const FFParams& ff,
                                        int64_t r0, const VT* __restrict__ xk,
                                        VT* __restrict__ yk, int accumulate) {
  using A = typename VTraits<VT>::A;
  constexpr bool CX = VTraits<VT>::cx;
  // BK_TRANS0_RANK / BK_TRANS_RANK: a translation sector whose target rows
  // (and, with a momentum phase, shifts M) come from the rank table instead of
  // canonicalisation + hash probe
  constexpr bool PHASED = BK == BK_TRANS_RANK;
  constexpr bool SIGNED = BK == BK_TRANSPAR_RANK;  // translation + parity: coefficient +-1
  constexpr bool RANKED = BK == BK_TRANS0_RANK || PHASED || SIGNED;
  constexpr int BKL = BK == BK_TRANS0_RANK ? (int)BK_TRANS0
                      : (PHASED ? (int)BK_TRANS : (SIGNED ? (int)BK_TRANSPAR : BK));
  __shared__ uint32_t s_binom[(BK == BK_PROJ_RANK || RANKED) ? 32 * 33 : 1];
  __shared__ int s_hist[64];
  __shared__ unsigned short s_order[256];
  __shared__ uint32_t s_state[256];
  if constexpr (BK == BK_PROJ_RANK) fill_binom32(s_binom);
  if constexpr (RANKED)
    for (int q = threadIdx.x; q < 32 * 33; q += blockDim.x) s_binom[q] = __ldg(b.binom32 + q);
  constexpr int RT = 256 / TPS;  // rows per tile
  const int t = threadIdx.x;
  if (t < 64) s_hist[t] = 0;
  __syncthreads();
  const uint32_t mask = (uint32_t)b.maskL;
  const int L = b.L;
  uint32_t s = 0;
  int key = 0;
  if (t < RT && r0 + t < b.D) {
    s = (BK == BK_TENSOR) ? (uint32_t)(r0 + t) : (uint32_t)__ldg(b.I + r0 + t);
    for (int f = 0; f < ff.nfam; ++f)
      key += __popc((s ^ rotl_L(s, ff.d[f], L, mask)) & ff.valid[f]);
  }
  key = min(key, 63);
  int slot = 0;
  if (t < RT) {
    s_state[t] = s;
    slot = atomicAdd(&s_hist[key], 1);
  }
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
  if (t < RT) s_order[s_hist[key] + slot] = (unsigned short)t;
  __syncthreads();
  const int tt = s_order[t / TPS];
  const int sub = TPS > 1 ? t % TPS : 0;
  const int64_t i = r0 + tt;
  const bool valid = i < b.D;  // the TPS lanes of a row agree
  if (TPS == 1 && !valid) return;
  const uint32_t st = s_state[tt];  // 0 past the last row: no hits
  const A invRi = (b.R && valid) ? (A)(1.0 / __ldg(b.R + i)) : (A)1;
  // complete fixed-charge sector (BK_PROJ_RANK): a state's row is its colex
  // rank, so target rows follow from the row index by the same rank update
  constexpr bool DIRECT = BK == BK_PROJ_RANK;
  uint32_t rs = 0;  // colex rank of the row state (rank-table search)
  if constexpr (RANKED) rs = valid ? __ldg(b.rowrank + i) : 0u;
  if constexpr (DIRECT) rs = (uint32_t)i;
  int pc = 0;  // pairs of hits seen so far in this row
  double dr = 0.0, di = 0.0;
  A ar = 0, ai = 0;
  // bases whose index() coefficient has no phase (1 + 0i): the products with
  // the phase are skipped (equal values; only the sign of a zero may differ)
  // (translation + parity: a real +-1 phase, the imaginary products are skipped)
  constexpr bool UNIT_PHASE =
      BKL == BK_TENSOR || BKL == BK_PROJ_RANK || BKL == BK_PROJ_HASH || BKL == BK_TRANS0;
  constexpr bool REAL_PHASE = BKL == BK_TRANSPAR;
  auto acc = [&](const HitCtx& c, double rpos, double vr, double vi, Cx<A> xv) {
    const A pr = (A)c.pre, pi = (A)c.pim, v_r = (A)vr, v_i = (A)vi;
    const A ratio = (A)rpos * invRi;
    const A cr = UNIT_PHASE ? v_r * ratio
                 : REAL_PHASE ? (v_r * pr) * ratio : (v_r * pr - v_i * pi) * ratio;
    if constexpr (CX) {
      const A ci = UNIT_PHASE ? v_i * ratio
                   : REAL_PHASE ? (v_i * pr) * ratio : (v_r * pi + v_i * pr) * ratio;
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
      if (TPS > 1 && (pc++ % TPS) != sub) continue;
      const int q1 = p1 >= d ? p1 - d : p1 - d + L, q2 = p2 >= d ? p2 - d : p2 - d + L;
      HitCtx h1, h2;
      int64_t pos1, pos2;
      double rp1, rp2;
      bool ok1, ok2;
      if constexpr (RANKED || DIRECT) {
        h1 = h2 = HitCtx{0u, 1.0, 0.0};
        uint32_t k1, k2;
        if (d == 1 && p1 != 0) {
          // adjacent sites (p2 >= p1 > 0, no wrap-around): the bit at a = p - 1
          // moves by one place, rank change C(a, j) with j set bits below a
          const int a1 = p1 - 1, a2 = p2 - 1;
          const uint32_t e1 = s_binom[a1 * 33 + __popc(st & ((1u << a1) - 1u))];
          const uint32_t e2 = s_binom[a2 * 33 + __popc(st & ((1u << a2) - 1u))];
          k1 = ((st >> a1) & 1u) ? rs + e1 : rs - e1;
          k2 = ((st >> a2) & 1u) ? rs + e2 : rs - e2;
        } else {
          k1 = rank_after_swap(st, rs, p1, q1, s_binom);
          k2 = two ? rank_after_swap(st, rs, p2, q2, s_binom) : k1;
        }
        if constexpr (DIRECT) {  // the exchange keeps the charge: both targets are rows
          pos1 = (int64_t)k1;
          pos2 = (int64_t)k2;
          rp1 = rp2 = 1.0;
          ok1 = true;
          ok2 = two;
        } else {
          const uint32_t v1 = __ldg(b.rankmap + k1);
          const uint32_t v2 = two ? __ldg(b.rankmap + k2) : ~0u;
          ok1 = v1 != ~0u;
          ok2 = v2 != ~0u;
          pos1 = pos2 = 0;
          rp1 = rp2 = 1.0;
          int M1 = 0, M2 = 0;
          if (ok1) rank_decode(b, v1, pos1, rp1, M1);
          if (ok2) rank_decode(b, v2, pos2, rp2, M2);
          if constexpr (PHASED) {  // phase C[M] of the target, as index() gives it
            if (ok1) { const double2 c = __ldg(b.phase + M1); h1.pre = c.x; h1.pim = c.y; }
            if (ok2) { const double2 c = __ldg(b.phase + M2); h2.pre = c.x; h2.pim = c.y; }
          }
          if constexpr (SIGNED) {  // bit 5 of the entry: the coefficient is -1
            h1.pre = ((v1 >> 5) & 1u) ? -1.0 : 1.0;
            h2.pre = ((v2 >> 5) & 1u) ? -1.0 : 1.0;
          }
        }
      } else {
        const uint32_t s1 = st ^ (1u << p1) ^ (1u << q1), s2 = st ^ (1u << p2) ^ (1u << q2);
        canon_ctx<BKL>(b, s1, h1);
        canon_ctx<BKL>(b, s2, h2);
        locate2<BKL>(b, s_binom, h1.key, h2.key, two, pos1, rp1, ok1, pos2, rp2, ok2);
      }
      const Cx<A> x1 = ok1 ? ldv(xk + pos1) : Cx<A>{0, 0};
      const Cx<A> x2 = ok2 ? ldv(xk + pos2) : Cx<A>{0, 0};
      const double2 w1 = ((st >> p1) & 1u) ? vb : va;
      const double2 w2 = ((st >> p2) & 1u) ? vb : va;
      if (ok1) acc(h1, rp1, w1.x, w1.y, x1);
      if (ok2) acc(h2, rp2, w2.x, w2.y, x2);
    }
  }
  if constexpr (TPS > 1) {
#pragma unroll
    for (int o = 1; o < TPS; o <<= 1) {
      ar += __shfl_xor_sync(0xffffffffu, ar, o);
      if constexpr (CX) ai += __shfl_xor_sync(0xffffffffu, ai, o);
    }
    if (sub != 0 || !valid) return;
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


// One 32-row slice of the materialised matrix (one warp, one row per lane).
// The entry stream is read once (evict-first: it is not reused within the
// product, psi is), four entries ahead of their psi gathers.  PACKED selects
// the entry format at compile time (1: row << packed | code in one word,
// 0: separate row and code arrays, -1: read sd.packed).  The diagonal operands
// are loaded after the loop: hoisting them costs registers and occupancy.
template <class VT, int PACKED = -1>
__device__ __forceinline__ void sell_slice(const BasisDev& b, const SellDev& sd, int64_t slice,
                                           int lane, const VT* __restrict__ xk,
                                           VT* __restrict__ yk, int accumulate) {
  using A = typename VTraits<VT>::A;
  constexpr bool CX = VTraits<VT>::cx;
  const int64_t slot = slice * 32 + lane;
  const unsigned rc = __ldg(sd.rowid + slot);
  const int w = __ldg(sd.width + slice);
  const int64_t base = __ldg(sd.off + slice) + lane;
  A ar = 0, ai = 0;
  auto term = [&](int c, int code) {
    const Cx<A> xv = ldv(xk + c);
    if constexpr (CX) {
      A vr, vi;
      if constexpr (sizeof(A) == 8) {
        const double2 v = __ldg(sd.vt64 + code);
        vr = v.x; vi = v.y;
      } else {
        const float2 v = __ldg(sd.vt32 + code);
        vr = v.x; vi = v.y;
      }
      ar += vr * xv.r + vi * xv.i;  // conj(v) * x
      ai += vr * xv.i - vi * xv.r;
    } else {
      A vr;
      if constexpr (sizeof(A) == 8) vr = __ldg(reinterpret_cast<const double*>(sd.vt64) + 2 * code);
      else vr = __ldg(reinterpret_cast<const float*>(sd.vt32) + 2 * code);
      ar += vr * xv.r;
    }
  };
  int k = 0;
  if (PACKED == 2 || (PACKED < 0 && sd.val)) {  // value mode: explicit coefficients
    const int* cp = sd.col + base;
    const double2* vp = sd.val + base;
    auto vterm = [&](int c, double2 v) {
      const Cx<A> xv = ldv(xk + c);
      const A vr = (A)v.x, vi = (A)v.y;
      if constexpr (CX) {
        ar += vr * xv.r + vi * xv.i;  // conj(v) * x
        ai += vr * xv.i - vi * xv.r;
      } else {
        ar += vr * xv.r;
      }
    };
    for (; k + 2 <= w; k += 2) {
      const int c0 = __ldcs(cp + (k + 0) * 32), c1 = __ldcs(cp + (k + 1) * 32);
      const double2 v0 = __ldcs(vp + (k + 0) * 32), v1 = __ldcs(vp + (k + 1) * 32);
      vterm(c0, v0);
      vterm(c1, v1);
    }
    for (; k < w; ++k) vterm(__ldcs(cp + k * 32), __ldcs(vp + k * 32));
  } else if (PACKED == 1 || (PACKED < 0 && sd.packed)) {
    const unsigned* ep = reinterpret_cast<const unsigned*>(sd.col + base);
    const int sh = sd.packed;
    const unsigned cm = (1u << sh) - 1u;
    for (; k + 4 <= w; k += 4) {  // four independent entries in flight
      const unsigned e0 = __ldcs(ep + (k + 0) * 32), e1 = __ldcs(ep + (k + 1) * 32);
      const unsigned e2 = __ldcs(ep + (k + 2) * 32), e3 = __ldcs(ep + (k + 3) * 32);
      term((int)(e0 >> sh), (int)(e0 & cm));
      term((int)(e1 >> sh), (int)(e1 & cm));
      term((int)(e2 >> sh), (int)(e2 & cm));
      term((int)(e3 >> sh), (int)(e3 & cm));
    }
    for (; k < w; ++k) {
      const unsigned e = __ldcs(ep + k * 32);
      term((int)(e >> sh), (int)(e & cm));
    }
  } else if (PACKED <= 0) {
    const int* cp = sd.col + base;
    const uint16_t* kp = sd.code + base;
    for (; k + 4 <= w; k += 4) {
      const int c0 = __ldcs(cp + (k + 0) * 32), c1 = __ldcs(cp + (k + 1) * 32);
      const int c2 = __ldcs(cp + (k + 2) * 32), c3 = __ldcs(cp + (k + 3) * 32);
      const int k0 = __ldcs(kp + (k + 0) * 32), k1 = __ldcs(kp + (k + 1) * 32);
      const int k2 = __ldcs(kp + (k + 2) * 32), k3 = __ldcs(kp + (k + 3) * 32);
      term(c0, k0);
      term(c1, k1);
      term(c2, k2);
      term(c3, k3);
    }
    for (; k < w; ++k) term(__ldcs(cp + k * 32), __ldcs(kp + k * 32));
  }
  if (rc == ~0u) return;
  const int64_t row = rc & ((1u << sd.rbits) - 1u);
  const A invR = (A)__ldg(sd.rinv + (rc >> sd.rbits));
  const double2 d = sd.diagc ? __ldg(sd.diagc + slot) : make_double2(__ldg(sd.diag + slot), 0.0);
  const Cx<A> xi = ldv(xk + row);
  Cx<A> out{ar * invR + (A)d.x * xi.r + (A)d.y * xi.i, (A)0};
  if constexpr (CX) out.i = ai * invR + (A)d.x * xi.i - (A)d.y * xi.r;
  if (accumulate) {
    const Cx<A> yo = ldout(yk + row);
    out.r += yo.r;
    out.i += yo.i;
  }
  stv(yk + row, out);
}

}  // namespace edk
