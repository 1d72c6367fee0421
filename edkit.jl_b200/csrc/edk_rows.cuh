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

// Diagonal of bond family f on the bit planes X = s, Y = rotl(s, d), valid
// mask V: sum over the local columns c = 2 X_p + Y_p of M[c][c] times the
// number of bonds in column c, explicitly rounded.  Shared by every flip-flop
// row kernel and the row-plan builder, so all of them round the diagonal alike.
__device__ __forceinline__ void ff_diag(const FFParams& ff, int f, uint32_t X, uint32_t Y,
                                        uint32_t V, double& dr, double& di) {
  const double c0 = __popc(~X & ~Y & V), c1 = __popc(~X & Y & V), c2 = __popc(X & ~Y & V),
               c3 = __popc(X & Y & V);
  const double2* dv = ff.dval[f];
  dr = __dadd_rn(dr, __fma_rn(dv[3].x, c3, __fma_rn(dv[2].x, c2, __fma_rn(dv[1].x, c1,
                                                                          __dmul_rn(dv[0].x, c0)))));
  di = __dadd_rn(di, __fma_rn(dv[3].y, c3, __fma_rn(dv[2].y, c2, __fma_rn(dv[1].y, c1,
                                                                          __dmul_rn(dv[0].y, c0)))));
}

// diagonal-only generic terms (fields, zz on other sites) of row state st
__device__ __forceinline__ void term_diag(const OpDev& op, uint32_t st, double& dr, double& di) {
  for (int q = 0; q < op.nterm; ++q) {
    const TermDev* T = op.term + q;
    int c = 0;
    for (int k = 0; k < T->nsites; ++k) c = (c << 1) | (int)((st >> T->bitpos[k]) & 1u);
    const double2 dv = __ldg(op.dval + T->diag_off + c);
    dr = __dadd_rn(dr, dv.x);
    di = __dadd_rn(di, dv.y);
  }
}

// ---------------------------------------------------------------------------
// Row body of the flip-flop fast path, shared by the tile kernels (rows sorted
// per block at run time, any index search) and the row-plan kernels (rows
// sorted once, rank-searched sectors).  For row i with state s:
//   y_i = (1/R_i) sum_f conj(w_f) sum_hits conj(C_t) R_t x_t + diag_i x_i
// where a hit exchanges the two sites of a bond of family f (value w_f =
// M[2][1] = M[1][2]* of the local matrix), t is the target row, C_t the phase
// index() returns and R_t its norm (TranslationalBasis.jl:310-341,
// Operator.jl:426-465: H[t, i] = w C_t R_t / R_i; the product gathers the
// conjugate, y_i = sum_t conj(H[t, i]) x_t, for a Hermitian operator).  Per
// family the hits are summed first and multiplied by conj(w_f) once (per hit
// when the two exchange values differ); 1/R_i is applied once at the end.
// Every product is an explicitly rounded operation (no contraction left to the
// compiler), so the tile and row-plan kernels, which share this body, give
// bit-identical results.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double fma_(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float fma_(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double mul_(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mul_(float a, float b) { return __fmul_rn(a, b); }

// Shared-memory tables of the fast kernels: binomials (rank updates) and the
// coefficient table indexed by the low bits of a table value: coef[c] = R of
// norm class c; with the rank table's shift M (k != 0) coef[M << 5 | c] =
// C[M] R_c; with its sign bit (translation + parity) coef[sign << 5 | c] = +-R_c.
template <int BK> struct FFTabSize { static constexpr int n = BK == BK_TRANS_RANK ? 1024 : 64; };
template <int BK> struct FFTab {
  uint32_t binom[32 * 33];
  double2 coef[FFTabSize<BK>::n];
};

// binom_src: the 32 x 33 table in global memory, or null to compute it
template <int BK>
__device__ __forceinline__ void ff_tab_fill(FFTab<BK>& t, const BasisDev& b,
                                            const uint32_t* binom_src) {
  if (binom_src) {
    for (int q = threadIdx.x; q < 32 * 33; q += blockDim.x) t.binom[q] = __ldg(binom_src + q);
  } else {
    fill_binom32(t.binom);
  }
  for (int q = threadIdx.x; q < FFTabSize<BK>::n; q += blockDim.x) {
    const int c = q & 31;
    const double R = (b.packed && c < b.nclass) ? b.Rcls[c] : 1.0;
    double2 v = make_double2(R, 0.0);
    if constexpr (BK == BK_TRANS_RANK) {
      const int M = q >> 5;
      const double2 C = M < b.len ? __ldg(b.phase + M) : make_double2(0.0, 0.0);
      v = make_double2(C.x * R, C.y * R);
    } else if constexpr (BK == BK_TRANSPAR_RANK) {
      v = make_double2(((q >> 5) & 1) ? -R : R, 0.0);
    }
    t.coef[q] = v;
  }
}

// S += conj(T) x for the target coefficient T = tr + i ti (real when !CT)
template <class A, bool CX, bool CT>
__device__ __forceinline__ void acc_t(Cx<A>& S, A tr, A ti, Cx<A> x) {
  if constexpr (CT) {
    S.r = fma_(ti, x.i, fma_(tr, x.r, S.r));
    if constexpr (CX) S.i = fma_(-ti, x.r, fma_(tr, x.i, S.i));
  } else {
    S.r = fma_(tr, x.r, S.r);
    if constexpr (CX) S.i = fma_(tr, x.i, S.i);
  }
}
// Y += conj(w) S
template <class A, bool CX>
__device__ __forceinline__ void fold_w(Cx<A>& Y, double2 w, Cx<A> S) {
  const A wr = (A)w.x, wi = (A)w.y;
  if constexpr (CX) {
    Y.r = fma_(wi, S.i, fma_(wr, S.r, Y.r));
    Y.i = fma_(-wi, S.r, fma_(wr, S.i, Y.i));
  } else {
    Y.r = fma_(wr, S.r, Y.r);
  }
}

// (ok, pos, coefficient) of the targets k1, k2 of a pair of hits: ranks
// (rank table or complete sector) or states (tensor rows, canonicalise + probe).
template <int BK, class A>
__device__ __forceinline__ void ff_targets(const BasisDev& b, const FFTab<BK>& t, uint32_t k1,
                                           uint32_t k2, bool two, bool& ok1, int64_t& pos1,
                                           A& t1r, A& t1i, bool& ok2, int64_t& pos2, A& t2r,
                                           A& t2i) {
  constexpr bool RANKED = BK == BK_TRANS0_RANK || BK == BK_TRANS_RANK || BK == BK_TRANSPAR_RANK;
  t1r = t2r = (A)1;
  t1i = t2i = (A)0;
  if constexpr (RANKED) {
    constexpr uint32_t TM = FFTabSize<BK>::n - 1;
    const uint32_t v1 = __ldg(b.rankmap + k1);
    const uint32_t v2 = __ldg(b.rankmap + k2);
    ok1 = v1 != ~0u;
    ok2 = two && v2 != ~0u;
    const int sh = b.rank_shift;
    pos1 = ok1 ? (int64_t)(v1 >> sh) : 0;
    pos2 = ok2 ? (int64_t)(v2 >> sh) : 0;
    const double2 c1 = t.coef[v1 & TM], c2 = t.coef[v2 & TM];
    t1r = (A)c1.x; t1i = (A)c1.y;
    t2r = (A)c2.x; t2i = (A)c2.y;
  } else if constexpr (BK == BK_PROJ_RANK || BK == BK_TENSOR) {  // k = the target's row
    ok1 = true;
    ok2 = two;
    pos1 = (int64_t)k1;
    pos2 = (int64_t)k2;
  } else {  // k = the target state: canonicalise, then probe
    HitCtx h1, h2;
    canon_ctx<BK>(b, k1, h1);
    canon_ctx<BK>(b, k2, h2);
    double r1, r2;
    locate2<BK>(b, t.binom, h1.key, h2.key, two, pos1, r1, ok1, pos2, r2, ok2);
    if constexpr (BK != BK_PROJ_HASH) {
      t1r = (A)(h1.pre * r1);
      t1i = (A)(h1.pim * r1);
      t2r = (A)(h2.pre * r2);
      t2i = (A)(h2.pim * r2);
    }
  }
}

// Off-diagonal sum of one row (before the factor 1/R_i).  TPS lanes share the
// row and take its pairs of hits in turn (lane `sub`); rkw, when not ~0u, is
// the precomputed rank of the state with bits 0 and L-1 exchanged.
// NN: 0 test at run time for the single nearest-neighbour family of equal
// exchange values (and take its loop), 1 always take that loop (the caller
// has checked), 2 never.
template <int BK, class VT, int TPS, int NN = 0>
__device__ __forceinline__ Cx<typename VTraits<VT>::A> ff_row_sum(
    const BasisDev& b, const FFParams& ff, const FFTab<BK>& t, uint32_t st, uint32_t rs,
    uint32_t rkw, int sub, const VT* __restrict__ xk) {
  using A = typename VTraits<VT>::A;
  constexpr bool CX = VTraits<VT>::cx;
  constexpr bool RANKED = BK == BK_TRANS0_RANK || BK == BK_TRANS_RANK || BK == BK_TRANSPAR_RANK;
  constexpr bool BYRANK = RANKED || BK == BK_PROJ_RANK;
  constexpr bool CT = BK == BK_TRANS_RANK || BK == BK_TRANS;  // complex target coefficients
  const uint32_t mask = (uint32_t)b.maskL;
  const int L = b.L;
  Cx<A> Y{0, 0};
  if constexpr (BYRANK && TPS == 1 && NN != 2) {
    // one nearest-neighbour family with equal exchange values (XXZ, Heisenberg
    // chains): the same hits in the same order, without the per-hit tests of
    // the general loop; the wrap-around hit (bit 0) first, then pairs
    if (NN == 1 || (ff.nfam == 1 && ff.d[0] == 1 && ff.same[0])) {
      uint32_t bits = (st ^ rotl_L(st, 1, L, mask)) & ff.valid[0];
      Cx<A> S0{0, 0};
      auto pair = [&](uint32_t k1, uint32_t k2, bool two) {
        bool ok1, ok2;
        int64_t pos1, pos2;
        A t1r, t1i, t2r, t2i;
        ff_targets<BK, A>(b, t, k1, k2, two, ok1, pos1, t1r, t1i, ok2, pos2, t2r, t2i);
        const Cx<A> x1 = ldv(xk + pos1), x2 = ldv(xk + pos2);
        if (ok1) acc_t<A, CX, CT>(S0, t1r, t1i, x1);
        if (ok2) acc_t<A, CX, CT>(S0, t2r, t2i, x2);
      };
      auto adj = [&](int a) -> uint32_t {  // sites a, a + 1: rank change C(a, j)
        const uint32_t e = t.binom[a * 33 + __popc(st & ((1u << a) - 1u))];
        return ((st >> a) & 1u) ? rs + e : rs - e;
      };
      if (bits & 1u) {
        bits &= ~1u;
        const uint32_t k = rkw != ~0u ? rkw : rank_after_swap(st, rs, 0, L - 1, t.binom);
        pair(k, k, false);
      }
      if constexpr (NN == 1) {  // four hits per pass: their table reads and psi gathers in flight together
        while (bits) {
          int p[4];
          bool on[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            on[u] = bits != 0;
            p[u] = on[u] ? __ffs(bits) - 1 : (u ? p[u - 1] : 1);
            bits &= bits - 1;
          }
          // target ranks (a hit past the row's last one repeats the previous
          // position: a valid rank whose product is not accumulated)
          uint32_t v[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) v[u] = adj(p[u] - 1);
          if constexpr (RANKED) {  // rank -> table entry (row, shift, class)
#pragma unroll
            for (int u = 0; u < 4; ++u) v[u] = __ldg(b.rankmap + v[u]);
          }
          Cx<A> x[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            if constexpr (RANKED) {
              on[u] = on[u] && v[u] != ~0u;
              x[u] = ldv(xk + (on[u] ? (int64_t)(v[u] >> b.rank_shift) : 0));
            } else {  // complete sector: the rank is the row
              x[u] = ldv(xk + (int64_t)v[u]);
            }
          }
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            if constexpr (RANKED) {
              constexpr uint32_t TM = FFTabSize<BK>::n - 1;
              const double2 c = t.coef[v[u] & TM];
              if (on[u]) acc_t<A, CX, CT>(S0, (A)c.x, (A)c.y, x[u]);
            } else {
              if (on[u]) acc_t<A, CX, CT>(S0, (A)1, (A)0, x[u]);
            }
          }
        }
        fold_w<A, CX>(Y, ff.v1[0], S0);
        return Y;
      }
      while (bits) {
        const int p1 = __ffs(bits) - 1;
        bits &= bits - 1;
        const bool two = bits != 0;
        const int p2 = two ? __ffs(bits) - 1 : p1;
        bits &= bits - 1;
        pair(adj(p1 - 1), adj(p2 - 1), two);
      }
      fold_w<A, CX>(Y, ff.v1[0], S0);
      return Y;
    }
  }
  int pc = 0;  // pairs of hits seen so far in this row
  for (int f = 0; f < ff.nfam; ++f) {
    const int d = ff.d[f];
    uint32_t bits = (st ^ rotl_L(st, d, L, mask)) & ff.valid[f];
    const bool same = ff.same[f] != 0;
    Cx<A> S0{0, 0};  // sum of conj(T) x (values equal), or of conj(w T) x (values differ)
    // the target of hit p (sites p and p - d mod L): its rank, or its state
    auto target = [&](int p) -> uint32_t {
      const int q = p >= d ? p - d : p - d + L;
      if constexpr (BYRANK) {
        if (d == 1 && p != 0) {  // adjacent sites a = p - 1, a + 1: rank change C(a, j)
          const int a = p - 1;
          const uint32_t e = t.binom[a * 33 + __popc(st & ((1u << a) - 1u))];
          return ((st >> a) & 1u) ? rs + e : rs - e;
        }
        if (d == 1 && rkw != ~0u) return rkw;
        return rank_after_swap(st, rs, p, q, t.binom);
      } else {
        return st ^ (1u << p) ^ (1u << q);
      }
    };
    while (bits) {
      const int p1 = __ffs(bits) - 1;
      bits &= bits - 1;
      const bool two = bits != 0;
      const int p2 = two ? __ffs(bits) - 1 : p1;
      bits &= bits - 1;
      if (TPS > 1 && (pc++ % TPS) != sub) continue;
      const uint32_t k1 = target(p1), k2 = target(p2);
      bool ok1, ok2;
      int64_t pos1, pos2;
      A t1r, t1i, t2r, t2i;
      ff_targets<BK, A>(b, t, k1, k2, two, ok1, pos1, t1r, t1i, ok2, pos2, t2r, t2i);
      const Cx<A> x1 = ldv(xk + pos1), x2 = ldv(xk + pos2);  // row 0 for an absent target
      if (same) {
        if (ok1) acc_t<A, CX, CT>(S0, t1r, t1i, x1);
        if (ok2) acc_t<A, CX, CT>(S0, t2r, t2i, x2);
      } else if constexpr (CX) {  // the two exchange values differ: fold w per hit
        const double2 w1 = ((st >> p1) & 1u) ? ff.v2[f] : ff.v1[f];
        const double2 w2 = ((st >> p2) & 1u) ? ff.v2[f] : ff.v1[f];
        const A u1r = fma_(-(A)w1.y, t1i, mul_((A)w1.x, t1r)), u1i = fma_((A)w1.y, t1r, mul_((A)w1.x, t1i));
        const A u2r = fma_(-(A)w2.y, t2i, mul_((A)w2.x, t2r)), u2i = fma_((A)w2.y, t2r, mul_((A)w2.x, t2i));
        if (ok1) acc_t<A, CX, true>(S0, u1r, u1i, x1);
        if (ok2) acc_t<A, CX, true>(S0, u2r, u2i, x2);
      }
    }
    // (real vectors always see equal values: the two exchange elements of a
    // Hermitian bond are complex conjugates, and complex operators refuse
    // real vectors)
    fold_w<A, CX>(Y, same ? ff.v1[f] : make_double2(1.0, 0.0), S0);
  }
  return Y;
}

// y_i (+)= invRi Y + diag x_i
template <class VT>
__device__ __forceinline__ void ff_row_store(Cx<typename VTraits<VT>::A> Y,
                                             typename VTraits<VT>::A invRi, double dr, double di,
                                             const VT* __restrict__ xk, VT* __restrict__ yk,
                                             int64_t i, int accumulate) {
  using A = typename VTraits<VT>::A;
  constexpr bool CX = VTraits<VT>::cx;
  const Cx<A> xi = ldv(xk + i);
  Cx<A> out{fma_((A)dr, xi.r, mul_(invRi, Y.r)), (A)0};
  if constexpr (CX) {
    out.r = fma_((A)di, xi.i, out.r);
    out.i = fma_(-(A)di, xi.r, fma_((A)dr, xi.i, mul_(invRi, Y.i)));
  }
  if (accumulate) {
    const Cx<A> yo = ldout(yk + i);
    out.r += yo.r;
    out.i += yo.i;
  }
  stv(yk + i, out);
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
  constexpr bool RANKED = BK == BK_TRANS0_RANK || BK == BK_TRANS_RANK || BK == BK_TRANSPAR_RANK;
  __shared__ FFTab<BK> s_tab;
  __shared__ int s_hist[64];
  __shared__ unsigned short s_order[256];
  __shared__ uint32_t s_state[256];
  ff_tab_fill<BK>(s_tab, b, RANKED ? b.binom32 : nullptr);
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
  uint32_t rs = 0;  // colex rank of the row state (rank search), or the row (complete sector)
  if constexpr (RANKED) rs = valid ? __ldg(b.rowrank + i) : 0u;
  if constexpr (BK == BK_PROJ_RANK) rs = (uint32_t)i;
  Cx<A> Y = ff_row_sum<BK, VT, TPS>(b, ff, s_tab, st, rs, ~0u, sub, xk);
  if constexpr (TPS > 1) {
#pragma unroll
    for (int o = 1; o < TPS; o <<= 1) {
      Y.r += __shfl_xor_sync(0xffffffffu, Y.r, o);
      if constexpr (CX) Y.i += __shfl_xor_sync(0xffffffffu, Y.i, o);
    }
    if (sub != 0 || !valid) return;
  }
  double dr = 0.0, di = 0.0;
  for (int f = 0; f < ff.nfam; ++f)
    ff_diag(ff, f, st, rotl_L(st, ff.d[f], L, mask), ff.valid[f], dr, di);
  term_diag(op, st, dr, di);
  ff_row_store<VT>(Y, invRi, dr, di, xk, yk, i, accumulate);
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
