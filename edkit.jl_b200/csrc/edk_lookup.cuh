// edk_lookup.cuh — device-side index(b, dgt): orbit canonicalisation on
// bit-packed states followed by a table lookup.
//
// The canonicalisation restates, on integers, the loops of
//   TranslationalBasis index        src/Basis/TranslationalBasis.jl:310-341
//   TranslationParityBasis index    src/Basis/TranslationalParityBasis.jl:192-234
//   AbelianBasis shift_canonical    src/Basis/AbelianBasis.jl:428-445, 669-693
// with the same first-minimum tie rule (strict <, scan order 0,1,2,...), so the
// shift M, and hence the phase, is the reference's.  Instead of the
// reference's binary_search over the sorted I (ProjectedBasis.jl:71-81) the row
// is found with one open-addressing probe sequence (a state present in I maps
// to its position in I, an absent state reports "not found" exactly where
// binary_search returns 0).
#pragma once

#include "edk_internal.cuh"

namespace edk {

template <class S> struct StateBits;
template <> struct StateBits<uint32_t> { static constexpr int bits = 32; };
template <> struct StateBits<uint64_t> { static constexpr int bits = 64; };

template <class S>
__device__ __forceinline__ S rotr_L(S s, int a, int L, S mask) {
  return (S)(((s >> a) | (s << (L - a))) & mask);
}
template <class S>
__device__ __forceinline__ S rotl_L(S s, int a, int L, S mask) {
  return (S)(((s << a) | (s >> (L - a))) & mask);
}
__device__ __forceinline__ uint32_t rev_L(uint32_t s, int L) { return __brev(s) >> (32 - L); }
__device__ __forceinline__ uint64_t rev_L(uint64_t s, int L) { return __brevll(s) >> (64 - L); }
__device__ __forceinline__ int popc_s(uint32_t s) { return __popc(s); }
__device__ __forceinline__ int popc_s(uint64_t s) { return __popcll(s); }
__device__ __forceinline__ int ffs_s(uint32_t s) { return __ffs(s) - 1; }
__device__ __forceinline__ int ffs_s(uint64_t s) { return __ffsll((long long)s) - 1; }

// 32-bit key mix; callers take the TOP bits (hslot32), which the two
// multiplications mix best.
__host__ __device__ __forceinline__ uint32_t hmix32(uint32_t h) {
  h *= 0x9e3779b1u; h ^= h >> 15; h *= 0x85ebca77u;
  return h;
}
__host__ __device__ __forceinline__ uint64_t hmix64(uint64_t h) {
  h ^= h >> 33; h *= 0xff51afd7ed558ccdull; h ^= h >> 33; h *= 0xc4ceb9fe1a85ec53ull;
  h ^= h >> 33;
  return h;
}

// first slot of a 32-bit key in a table of hmask + 1 = 2^hbits slots
__host__ __device__ __forceinline__ uint64_t hslot32(uint32_t key, int hbits) {
  return hbits == 0 ? 0 : (uint64_t)(hmix32(key) >> (32 - hbits));
}

// Sorted-array search: the representatives are stored in ascending order, so
// the row of a key is its position in that array (the binary search of
// EDKit's index(), src/Basis/ProjectedBasis.jl:71-81 binary_search).  Level one
// searches every 32nd key (fence), level two the 32 keys of one 128-byte
// line.  The value returned is encoded like a hash value.
__device__ __forceinline__ uint32_t sorted_value(const BasisDev& b, int64_t row) {
  return b.packed ? ((uint32_t)row << 5) | (uint32_t)__ldg(b.rcls8 + row) : (uint32_t)row;
}
__device__ __forceinline__ bool sorted_find32(const BasisDev& b, uint32_t key, uint32_t& val) {
  int64_t n = b.nfence;
  if (n == 0 || __ldg(b.fence) > key) return false;
  int64_t lo = 0;  // invariant: fence[lo] <= key, answer in [lo, lo + n)
  while (n > 1) {
    const int64_t half = n >> 1;
    if (__ldg(b.fence + lo + half) <= key) { lo += half; n -= half; }
    else n = half;
  }
  int64_t r = lo * 32;
  n = b.D - r < 32 ? b.D - r : 32;
  while (n > 1) {
    const int64_t half = n >> 1;
    if (__ldg(b.keys32 + r + half) <= key) { r += half; n -= half; }
    else n = half;
  }
  if (__ldg(b.keys32 + r) != key) return false;
  val = sorted_value(b, r);
  return true;
}
__device__ __forceinline__ bool sorted_find64(const BasisDev& b, uint64_t key, uint32_t& val) {
  int64_t n = b.D;
  if (n == 0 || __ldg(reinterpret_cast<const unsigned long long*>(b.I)) > key) return false;
  int64_t lo = 0;
  while (n > 1) {
    const int64_t half = n >> 1;
    if (__ldg(reinterpret_cast<const unsigned long long*>(b.I) + lo + half) <= key) {
      lo += half;
      n -= half;
    } else {
      n = half;
    }
  }
  if (__ldg(reinterpret_cast<const unsigned long long*>(b.I) + lo) != key) return false;
  val = sorted_value(b, lo);
  return true;
}

// 32-bit keys: one 8-byte slot = key << 32 | value, empty = all ones.
__device__ __forceinline__ bool hash_find(const BasisDev& b, uint32_t key, uint32_t& val) {
  if (b.search == 1) return sorted_find32(b, key, val);
  const unsigned long long* tab = reinterpret_cast<const unsigned long long*>(b.htab);
  uint64_t slot = hslot32(key, b.hbits);
  for (uint64_t n = 0; n <= b.hmask; ++n) {
    unsigned long long e = __ldg(tab + slot);
    if (e == ~0ull) return false;
    if ((uint32_t)(e >> 32) == key) { val = (uint32_t)e; return true; }
    slot = (slot + 1) & b.hmask;
  }
  return false;
}
// 64-bit keys: 16-byte slots {key, value}, empty key = all ones.
__device__ __forceinline__ bool hash_find(const BasisDev& b, uint64_t key, uint32_t& val) {
  if (b.search == 1) return sorted_find64(b, key, val);
  const ulonglong2* tab = reinterpret_cast<const ulonglong2*>(b.htab);
  uint64_t slot = hmix64(key) & b.hmask;
  for (uint64_t n = 0; n <= b.hmask; ++n) {
    ulonglong2 e = __ldg(tab + slot);
    if (e.x == ~0ull) return false;
    if (e.x == key) { val = (uint32_t)e.y; return true; }
    slot = (slot + 1) & b.hmask;
  }
  return false;
}

// decode a hash value into (row, norm)
__device__ __forceinline__ void decode_val(const BasisDev& b, uint32_t v, int64_t& pos,
                                           double& rpos) {
  if (b.packed) {
    pos = (int64_t)(v >> 5);
    rpos = b.Rcls[v & 31u];
  } else {
    pos = (int64_t)v;
    rpos = __ldg(b.R + pos);
  }
}

// decode a rank-table entry into (row, norm, first-minimum shift M)
__device__ __forceinline__ void rank_decode(const BasisDev& b, uint32_t v, int64_t& pos,
                                            double& rpos, int& M) {
  pos = (int64_t)(v >> b.rank_shift);
  M = (int)((v >> 5) & 31u);
  rpos = b.packed ? b.Rcls[v & 31u] : __ldg(b.R + pos);
}

// colex rank of a fixed-popcount state (= its position among all states with
// that popcount in ascending order); binom[p*33 + k] = C(p, k), p < 32.
__device__ __forceinline__ int64_t colex_rank(uint32_t s, const uint32_t* binom) {
  uint32_t r = 0;
  int j = 1;
  while (s) {
    int p = __ffs(s) - 1;
    r += binom[p * 33 + j];
    s &= s - 1;
    ++j;
  }
  return (int64_t)r;
}
__device__ __forceinline__ int64_t colex_rank(uint64_t s, const uint32_t* binom) {
  return colex_rank((uint32_t)s, binom);  // rank mode is only enabled for L <= 32
}

// One odometer step over the generators — AbelianBasis.jl:292-299 / 405-414.
template <class S>
__device__ __forceinline__ S apply_gen(const GenDev& g, S s, int L, S mask) {
  switch (g.kind) {
    case GEN_ROTL: s = rotl_L(s, g.shift, L, mask); break;
    case GEN_REV: s = rev_L(s, L); break;
    case GEN_ID: break;
    default:
      for (int q = 0; q < g.nlayers; ++q) {
        S lm = (S)g.lmask[q];
        int sh = g.lshift[q];
        S delta = ((s >> sh) ^ s) & lm;
        s = s ^ delta ^ (S)(delta << sh);
      }
  }
  return (S)(s ^ (S)g.inv_mask);
}

// ---------------------------------------------------------------------------
// 32-bit canonicalisation (L <= 32).  The state is doubled into a 64-bit word
// w = s | s << L, so the rotation right by i is one funnel shift of (hi:lo)
// plus a mask: three instructions per candidate rotation, no branches.  Only
// the first strict minimum is kept, so M (the shift, hence the phase) is the
// one the reference's loop reports; its early exit on returning to the start
// state only skips rotations that repeat earlier ones.
// ---------------------------------------------------------------------------
struct Dbl32 { uint32_t lo, hi; };
__device__ __forceinline__ Dbl32 dbl32(uint32_t s, int L) {
  uint64_t w = (uint64_t)s | ((uint64_t)s << L);
  return {(uint32_t)w, (uint32_t)(w >> 32)};
}
__device__ __forceinline__ uint32_t rotr_dbl(Dbl32 d, int i, uint32_t mask) {
  return __funnelshift_r(d.lo, d.hi, i) & mask;
}
// Left-aligned doubling: V = (s | s << L) << (32 - L).  The 32-bit window
// funnelshift_r(V, i) holds the rotation right by i in its top L bits; its
// low 32 - L bits are other digits of the ring, which only matter when two
// rotations tie on the top L bits (then the states are equal).
__device__ __forceinline__ Dbl32 dbl32_top(uint32_t s, int L) {
  uint64_t w = ((uint64_t)s | ((uint64_t)s << L)) << (32 - L);
  return {(uint32_t)w, (uint32_t)(w >> 32)};
}
// min over translations by multiples of A (phase-free sectors): two
// instructions per rotation (funnel shift + min)
__device__ __forceinline__ uint32_t canon_min32(uint32_t s, int L, int A, int len, uint32_t mask) {
  const Dbl32 d = dbl32_top(s, L);
  uint32_t m = d.lo;
  int i = A;
#pragma unroll 4
  for (int q = 1; q < len; ++q) {
    m = min(m, __funnelshift_r(d.lo, d.hi, i));
    i += A;
  }
  (void)mask;
  return m >> (32 - L);
}
// Unit cell 1 only: the minimum rotation starts at the top of a run of zeros
// (a 0 digit whose left neighbour is 1), so only those rotations are
// compared: one per domain-wall pair instead of one per site.  For the top
// q of such a run the rotation is the right shift by q + 1 = ffs position.
__device__ __forceinline__ uint32_t canon_runs32(uint32_t s, int L, uint32_t mask) {
  const Dbl32 d = dbl32_top(s, L);
  uint32_t m = d.lo;
  uint32_t z = ~s & (((s >> 1) | (s << (L - 1))) & mask);
  while (z) {
    const int i = __ffs(z);
    z &= z - 1;
    m = min(m, __funnelshift_r(d.lo, d.hi, i));
  }
  return m >> (32 - L);
}

// first minimum and its translation count M
__device__ __forceinline__ uint32_t canon_arg32(uint32_t s, int L, int A, int len, uint32_t mask,
                                                int& M) {
  if (L <= 27) {
    // the spare low bits carry q, so min() keeps the smallest q on ties
    const Dbl32 d = dbl32_top(s, L);
    const uint32_t hi_mask = ~((1u << (32 - L)) - 1u);
    uint32_t m = d.lo & hi_mask;
    int i = A;
#pragma unroll 4
    for (int q = 1; q < len; ++q) {
      m = min(m, (__funnelshift_r(d.lo, d.hi, i) & hi_mask) | (uint32_t)q);
      i += A;
    }
    M = (int)(m & ~hi_mask);
    return m >> (32 - L);
  }
  const Dbl32 d = dbl32(s, L);
  uint32_t m = s;
  M = 0;
  int i = A;
#pragma unroll 4
  for (int q = 1; q < len; ++q) {
    const uint32_t r = rotr_dbl(d, i, mask);
    const bool lt = r < m;
    m = lt ? r : m;
    M = lt ? q : M;
    i += A;
  }
  return m;
}
// translations and reflected translations (TranslationParityBasis):
// rev(rotr(s, i)) = rotl(rev(s), i) = rotr(rev(s), L - i).
__device__ __forceinline__ void canon_par32(uint32_t s, int L, int A, int len, uint32_t mask,
                                            uint32_t& Iam, int& Rr, uint32_t& Ibm, int& M) {
  const uint32_t rs = __brev(s) >> (32 - L);
  if (L <= 27) {
    const Dbl32 d = dbl32_top(s, L), dr = dbl32_top(rs, L);
    const uint32_t hi_mask = ~((1u << (32 - L)) - 1u);
    uint32_t ma = d.lo & hi_mask, mb = dr.lo & hi_mask;
    int i = A;
#pragma unroll 2
    for (int q = 1; q < len; ++q) {
      ma = min(ma, (__funnelshift_r(d.lo, d.hi, i) & hi_mask) | (uint32_t)q);
      mb = min(mb, (__funnelshift_r(dr.lo, dr.hi, L - i) & hi_mask) | (uint32_t)q);
      i += A;
    }
    Rr = (int)(ma & ~hi_mask);
    M = (int)(mb & ~hi_mask);
    Iam = ma >> (32 - L);
    Ibm = mb >> (32 - L);
    return;
  }
  const Dbl32 d = dbl32(s, L);
  const Dbl32 dr = dbl32(rs, L);
  Iam = s; Rr = 0; Ibm = rs; M = 0;
  int i = A;
#pragma unroll 2
  for (int q = 1; q < len; ++q) {
    const uint32_t t = rotr_dbl(d, i, mask);
    const uint32_t tb = rotr_dbl(dr, L - i, mask);
    const bool lt = t < Iam, lb = tb < Ibm;
    Iam = lt ? t : Iam;
    Rr = lt ? q : Rr;
    Ibm = lb ? tb : Ibm;
    M = lb ? q : M;
    i += A;
  }
}

// Result of index(b, state) on the device.
struct Hit {
  int64_t pos;   // 0-based row
  double pre, pim;  // phase of the state relative to its representative
  double rpos;   // norm R[pos]
};

// index(b, s): returns false where EDKit returns (0, 1).
template <int BK, class S>
__device__ __forceinline__ bool lookup(const BasisDev& b, S s, const uint32_t* binom, Hit& h) {
  h.pre = 1.0; h.pim = 0.0; h.rpos = 1.0;
  const S mask = (S)b.maskL;
  if constexpr (BK == BK_TENSOR) {
    h.pos = (int64_t)s;
    return true;
  } else if constexpr (BK == BK_PROJ_RANK) {
    if (popc_s(s) != b.K) return false;
    h.pos = colex_rank(s, binom);
    return true;
  } else if constexpr (BK == BK_PROJ_HASH) {
    uint32_t v;
    if (!hash_find(b, s, v)) return false;
    h.pos = b.packed ? (int64_t)(v >> 5) : (int64_t)v;
    return true;
  } else if constexpr (BK == BK_TRANS0) {
    // trivial phase: the representative is the minimum over all rotations
    S m = s;
    if constexpr (sizeof(S) == 4) {
      m = canon_min32(s, b.L, b.A, b.len, mask);
    } else {
      S t = s;
      for (int i = 1; i < b.len; ++i) {
        t = rotr_L(t, b.A, b.L, mask);
        m = t < m ? t : m;
      }
    }
    uint32_t v;
    if (!hash_find(b, m, v)) return false;
    decode_val(b, v, h.pos, h.rpos);
    return true;
  } else if constexpr (BK == BK_TRANS) {
    // TranslationalBasis.jl:318-325: rotate right by A, stop on return,
    // keep the first strict minimum and its shift M.
    S Im = s;
    int M = 0;
    if constexpr (sizeof(S) == 4) {
      Im = canon_arg32(s, b.L, b.A, b.len, mask, M);
    } else {
      S I0 = s, t = s;
      for (int i = 1; i < b.len; ++i) {
        t = rotr_L(t, b.A, b.L, mask);
        if (t == I0) break;
        if (t < Im) { Im = t; M = i; }
      }
    }
    uint32_t v;
    if (!hash_find(b, Im, v)) return false;
    decode_val(b, v, h.pos, h.rpos);
    double2 c = __ldg(b.phase + M);
    h.pre = c.x; h.pim = c.y;
    return true;
  } else if constexpr (BK == BK_TRANSPAR) {
    // TranslationalParityBasis.jl:204-231
    S Iam, Ibm;
    int Rr = 0, M = 0;
    if constexpr (sizeof(S) == 4) {
      uint32_t a_, b_;
      canon_par32(s, b.L, b.A, b.len, mask, a_, Rr, b_, M);
      Iam = a_; Ibm = b_;
    } else {
      S Ia0 = s, t = s;
      Iam = Ia0; Ibm = rev_L(s, b.L);
      for (int i = 1; i < b.len; ++i) {
        t = rotr_L(t, b.A, b.L, mask);
        if (t == Ia0) break;
        if (t < Iam) { Iam = t; Rr = i; }
        S tb = rev_L(t, b.L);
        if (tb < Ibm) { Ibm = tb; M = i; }
      }
    }
    S key;
    double n;
    if (Ibm < Iam) { key = Ibm; n = (double)b.P * __ldg(b.phase + M).x; }
    else { key = Iam; n = __ldg(b.phase + Rr).x; }
    uint32_t v;
    if (!hash_find(b, key, v)) return false;
    decode_val(b, v, h.pos, h.rpos);
    h.pre = n;
    return true;
  } else {  // BK_ABELIAN: shift_canonical_int, AbelianBasis.jl:428-445
    int cnt[kMaxGen], best[kMaxGen];
#pragma unroll
    for (int g = 0; g < kMaxGen; ++g) { cnt[g] = 0; best[g] = 0; }
    int64_t order = 1;
    for (int g = 0; g < b.ngen; ++g) order *= b.gens[g].order;
    S cur = s, bst = s;
    for (int64_t t = 0; t < order; ++t) {
      for (int g = 0; g < b.ngen; ++g) {
        cur = apply_gen(b.gens[g], cur, b.L, mask);
        if (++cnt[g] >= b.gens[g].order) cnt[g] = 0; else break;
      }
      if (cur < bst) {
        bst = cur;
        for (int g = 0; g < b.ngen; ++g) best[g] = cnt[g];
      }
    }
    uint32_t v;
    if (!hash_find(b, bst, v)) return false;
    decode_val(b, v, h.pos, h.rpos);
    double pr = 1.0, pi = 0.0;
    for (int g = 0; g < b.ngen; ++g) {
      double2 c = __ldg(b.phase + b.gens[g].phase_off + best[g]);
      double nr = pr * c.x - pi * c.y, ni = pr * c.y + pi * c.x;
      pr = nr; pi = ni;
    }
    h.pre = pr; h.pim = pi;
    return true;
  }
}

}  // namespace edk
