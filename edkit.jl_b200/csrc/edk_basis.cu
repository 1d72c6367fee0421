// edk_basis.cu — basis tables on the device.
//
//   * construction on the GPU for base 2 (TensorBasis, ProjectedBasis with N,
//     TranslationalBasis, TranslationParityBasis, AbelianBasis via basis()):
//     candidates are enumerated in ascending order (colex unranking + Gosper's
//     next-permutation within a chunk), judged in parallel, and compacted with
//     an ordered two-pass count/scan/write, so I comes out sorted exactly like
//     the reference's ordered scans;
//   * upload of tables built by the Julia side (predicate bases);
//   * the row lookup table (open addressing, state -> row << 5 | norm class);
//   * batched index() and table export.
#include <cub/cub.cuh>

#include <algorithm>
#include <cstdlib>
#include <cmath>
#include <complex>
#include <map>
#include <set>
#include <unordered_map>

#include "edk_lookup.cuh"

namespace edk {

namespace {

constexpr int kChunk = 64;        // candidates per thread in the build kernels
constexpr int kMaxNormTab = 128;  // norm table entries (2 * len, len <= 64)

struct BuildParams {
  int kind;        // EDK_* basis kind
  int L, A, len;
  int Kmom;        // mod(-k, len) for TranslationalBasis
  int Kpar;        // +-1 for TranslationParityBasis
  int pairnorm;    // abelian (translation, Z2) group with TranslationFlipBasis norms
  int P;           // parity
  int full;        // 1: candidates are all 2^L states; 0: fixed popcount K
  int K;           // popcount of candidates
  uint64_t ncand;
  uint64_t maskL;
  const uint64_t* binom;   // (64 x 65) C(n, k), device
  // abelian
  int ngen;
  const GenDev* gens;
  const double2* gphase;
  const unsigned long long* allow;  // predicate bitmap (nullptr = no predicate)
};

__host__ __device__ inline uint64_t binom_at(const uint64_t* t, int n, int k) {
  return (k < 0 || k > n) ? 0ull : t[n * 65 + k];
}

// colex unranking of the t-th (0-based) state with K set bits below bit L
__device__ inline uint64_t unrank_colex(uint64_t t, int K, int L, const uint64_t* binom) {
  uint64_t s = 0;
  for (int p = L - 1; p >= 0 && K > 0; --p) {
    uint64_t c = binom_at(binom, p, K);
    if (t >= c) { s |= (1ull << p); t -= c; --K; }
  }
  return s;
}
// _gosper_next — AbelianBasis.jl:456-464
__device__ inline uint64_t gosper_next(uint64_t s) {
  uint64_t c = s & (~s + 1);
  uint64_t r = s + c;
  return r | (((r ^ s) >> 2) / c);
}

// TranslationJudge on integers — TranslationalBasis.jl:94-114.
// Returns the period (1..len) used to pick the norm, or 0 if rejected.
template <class S>
__device__ inline int judge_trans(S s, const BuildParams& p) {
  S mask = (S)p.maskL, t = s;
  for (int n = 1; n <= p.len - 1; ++n) {
    t = rotr_L(t, p.A, p.L, mask);
    if (t < s) return 0;
    if (t == s) return (((int64_t)n * p.Kmom) % p.len == 0) ? n : 0;
  }
  return p.len;
}
// TranslationParityJudge on integers — TranslationalParityBasis.jl:68-112.
// Returns 1 + norm-table index (Qp ? len + R - 1 : R - 1), 0 if rejected.
template <class S>
__device__ inline int judge_transpar(S s, const BuildParams& p) {
  S mask = (S)p.maskL;
  int R = p.len;
  bool Qp = false;
  S In = rev_L(s, p.L);
  if (In < s) return 0;
  if (In == s) { Qp = true; if (p.P != 1) return 0; }
  S t = s;
  for (int n = 1; n <= p.len - 1; ++n) {
    t = rotr_L(t, p.A, p.L, mask);
    S In1 = t, In2 = rev_L(t, p.L);
    if (In1 < s) return 0;
    if (In2 < s) return 0;
    bool even_or_k0 = (p.Kpar == 1) || (n % 2 == 0);
    if (In2 == s) {
      int Kn = even_or_k0 ? 1 : -1;
      if (p.P * Kn != 1) return 0;
      Qp = true;
    }
    if (In1 == s) {
      if (!even_or_k0) return 0;
      R = n;
      break;
    }
  }
  return 1 + (Qp ? p.len + R - 1 : R - 1);
}
// check_min_int — AbelianBasis.jl:399-418.  Returns the stabiliser size n
// (norm index n - 1) or 0 if rejected.
template <class S>
__device__ inline int judge_abelian(S s0, const BuildParams& p) {
  S mask = (S)p.maskL;
  int cnt[kMaxGen];
  for (int g = 0; g < kMaxGen; ++g) cnt[g] = 0;
  int64_t order = 1;
  for (int g = 0; g < p.ngen; ++g) order *= p.gens[g].order;
  S cur = s0;
  int N = 1;
  for (int64_t t = 2; t <= order; ++t) {
    for (int g = 0; g < p.ngen; ++g) {
      cur = apply_gen(p.gens[g], cur, p.L, mask);
      if (++cnt[g] >= p.gens[g].order) cnt[g] = 0; else break;
    }
    if (cur < s0) return 0;
    if (cur == s0) {
      double pr = 1.0, pi = 0.0;
      for (int g = 0; g < p.ngen; ++g) {
        double2 c = p.gphase[p.gens[g].phase_off + cnt[g]];
        double nr = pr * c.x - pi * c.y, ni = pr * c.y + pi * c.x;
        pr = nr; pi = ni;
      }
      // |phase - 1| < 1e-14 (hypot is the complex abs of the reference)
      if (!(hypot(pr - 1.0, pi) < 1e-14)) return 0;
      N += 1;
    }
  }
  return N;
}

// The same check for the (translation, flip) pair, returning the norm-table
// index of TranslationFlipBasis (TranslationalFlipBasis.jl:50-91): 1 +
// (Qp ? len + R - 1 : R - 1) with R the translation period and Qp whether a
// flipped translate returns the state.
template <class S>
__device__ inline int judge_abelian_pair(S s0, const BuildParams& p) {
  S mask = (S)p.maskL;
  int cnt[kMaxGen];
  for (int g = 0; g < kMaxGen; ++g) cnt[g] = 0;
  const int len = p.gens[0].order;
  const int64_t order = (int64_t)len * p.gens[1].order;
  S cur = s0;
  int R = len;
  bool Qp = false;
  for (int64_t t = 2; t <= order; ++t) {
    for (int g = 0; g < p.ngen; ++g) {
      cur = apply_gen(p.gens[g], cur, p.L, mask);
      if (++cnt[g] >= p.gens[g].order) cnt[g] = 0; else break;
    }
    if (cur < s0) return 0;
    if (cur == s0) {
      double pr = 1.0, pi = 0.0;
      for (int g = 0; g < p.ngen; ++g) {
        double2 c = p.gphase[p.gens[g].phase_off + cnt[g]];
        double nr = pr * c.x - pi * c.y, ni = pr * c.y + pi * c.x;
        pr = nr; pi = ni;
      }
      if (!(hypot(pr - 1.0, pi) < 1e-14)) return 0;
      if (cnt[1] == 0) R = min(R, cnt[0]);
      else Qp = true;
    }
  }
  return 1 + (Qp ? len + R - 1 : R - 1);
}

template <class S>
__device__ inline int judge(S s, const BuildParams& p) {
  if (p.allow && !((p.allow[(uint64_t)s >> 6] >> ((uint64_t)s & 63)) & 1ull)) return 0;
  switch (p.kind) {
    case EDK_PROJECTED: return 1;
    case EDK_TRANSLATIONAL: return judge_trans(s, p);
    case EDK_TRANSPARITY: return judge_transpar(s, p);
    default: return p.pairnorm ? judge_abelian_pair(s, p) : judge_abelian(s, p);
  }
}

template <class S>
__global__ void k_build_count(BuildParams p, uint64_t nchunks, uint32_t* counts) {
  uint64_t c = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nchunks) return;
  uint64_t t0 = c * kChunk;
  uint64_t t1 = min(t0 + (uint64_t)kChunk, p.ncand);
  uint64_t s = p.full ? t0 : unrank_colex(t0, p.K, p.L, p.binom);
  uint32_t n = 0;
  for (uint64_t t = t0; t < t1; ++t) {
    if (judge<S>((S)s, p) > 0) ++n;
    s = p.full ? s + 1 : gosper_next(s);
  }
  counts[c] = n;
}

template <class S>
__global__ void k_build_write(BuildParams p, uint64_t nchunks, const uint64_t* offsets,
                              uint64_t* I, uint8_t* cls) {
  uint64_t c = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nchunks) return;
  uint64_t t0 = c * kChunk;
  uint64_t t1 = min(t0 + (uint64_t)kChunk, p.ncand);
  uint64_t s = p.full ? t0 : unrank_colex(t0, p.K, p.L, p.binom);
  uint64_t o = offsets[c];
  for (uint64_t t = t0; t < t1; ++t) {
    int j = judge<S>((S)s, p);
    if (j > 0) {
      I[o] = s;
      if (cls) cls[o] = (uint8_t)(j - 1);
      ++o;
    }
    s = p.full ? s + 1 : gosper_next(s);
  }
}

__global__ void k_cls_hist(const uint8_t* cls, int64_t D, unsigned int* hist) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < D;
       i += (int64_t)gridDim.x * blockDim.x)
    atomicAdd(hist + cls[i], 1u);
}
// R[i] = norm_table[cls[i]]; cls[i] <- compact class id
__global__ void k_cls_apply(uint8_t* cls, int64_t D, const double* ntab, const int* remap,
                            double* R) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < D;
       i += (int64_t)gridDim.x * blockDim.x) {
    int c = cls[i];
    R[i] = ntab[c];
    cls[i] = (uint8_t)remap[c];
  }
}
// class of a host-provided R[i]: position of R[i] in the compact table
__global__ void k_cls_from_R(const double* R, int64_t D, BasisDev b, uint8_t* cls) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < D;
       i += (int64_t)gridDim.x * blockDim.x) {
    double r = R[i];
    int c = 0;
    for (int q = 0; q < b.nclass; ++q)
      if (b.Rcls[q] == r) c = q;
    cls[i] = (uint8_t)c;
  }
}

// Tables of the sorted-array search: 32-bit keys, the fence (every 32nd key)
// and a flag raised where the representatives are not strictly ascending.
__global__ void k_sorted_tables(const uint64_t* I, int64_t D, uint32_t* keys32, uint32_t* fence,
                                int* unsorted) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < D;
       i += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t s = I[i];
    if (i + 1 < D && !(s < I[i + 1])) *unsorted = 1;
    if (keys32) {
      keys32[i] = (uint32_t)s;
      if ((i & 31) == 0) fence[i >> 5] = (uint32_t)s;
    }
  }
}

__global__ void k_hash_insert32(const uint64_t* I, const uint8_t* cls, int64_t D, int packed,
                                unsigned long long* tab, uint64_t hmask, int hbits) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < D;
       i += (int64_t)gridDim.x * blockDim.x) {
    uint32_t key = (uint32_t)I[i];
    uint32_t val = packed ? (uint32_t)((i << 5) | (cls ? cls[i] : 0)) : (uint32_t)i;
    unsigned long long e = ((unsigned long long)key << 32) | val;
    uint64_t slot = hslot32(key, hbits);
    for (uint64_t n = 0; n <= hmask; ++n) {
      unsigned long long old = atomicCAS(tab + slot, ~0ull, e);
      if (old == ~0ull) break;
      slot = (slot + 1) & hmask;
    }
  }
}
__global__ void k_hash_insert64(const uint64_t* I, const uint8_t* cls, int64_t D, int packed,
                                ulonglong2* tab, uint64_t hmask) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < D;
       i += (int64_t)gridDim.x * blockDim.x) {
    uint64_t key = I[i];
    uint32_t val = packed ? (uint32_t)((i << 5) | (cls ? cls[i] : 0)) : (uint32_t)i;
    uint64_t slot = hmix64(key) & hmask;
    for (uint64_t n = 0; n <= hmask; ++n) {
      unsigned long long old =
          atomicCAS(reinterpret_cast<unsigned long long*>(&tab[slot].x), ~0ull,
                    (unsigned long long)key);
      if (old == ~0ull) { tab[slot].y = val; break; }
      slot = (slot + 1) & hmask;
    }
  }
}

// 1-based int64 (Julia) -> 0-based uint64
__global__ void k_to_states(const int64_t* I1, int64_t D, uint64_t* I) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < D;
       i += (int64_t)gridDim.x * blockDim.x)
    I[i] = (uint64_t)(I1[i] - 1);
}
__global__ void k_to_julia(const uint64_t* I, int64_t D, int64_t* I1) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < D;
       i += (int64_t)gridDim.x * blockDim.x)
    I1[i] = (int64_t)I[i] + 1;
}
template <int BK, class S>
__global__ void k_index(BasisDev b, int64_t n, const uint64_t* states, int64_t* pos,
                        double2* coeff) {
  __shared__ uint32_t s_binom[32 * 33];
  if (BK == BK_PROJ_RANK) {
    for (int q = threadIdx.x; q < 32 * 33; q += blockDim.x) {
      int pp = q / 33, kk = q % 33;
      uint64_t c = 1;
      if (kk > pp) c = 0;
      else for (int r = 1; r <= kk; ++r) c = c * (uint64_t)(pp - kk + r) / (uint64_t)r;
      s_binom[q] = (uint32_t)c;
    }
    __syncthreads();
  }
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    uint64_t st = states[i];
    Hit h;
    bool ok = (st <= b.maskL) && lookup<BK, S>(b, (S)st, s_binom, h);
    if (ok) {
      pos[i] = h.pos + 1;
      coeff[i] = make_double2(h.pre * h.rpos, h.pim * h.rpos);
    } else {
      pos[i] = 0;
      coeff[i] = make_double2(0.0, 0.0);
    }
  }
}

// every representative has popcount K (flag stays 0)
__global__ void k_popc_check(const uint64_t* I, int64_t D, int K, int* flag) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < D;
       i += (int64_t)gridDim.x * blockDim.x)
    if (__popcll(I[i]) != K) *flag = 1;
}
// Rank table of a phase-free translation sector: entry r belongs to the state
// of popcount K with colex rank r (colex unrank: the largest p with
// C(p, j) <= r for j = K..1), and holds the hash value of its orbit
// representative or ~0u.  `b` is passed with search = 0 (hash probes).
__global__ void k_rank_map(BasisDev b, int K, uint64_t n, uint32_t* out) {
  __shared__ uint32_t sb[32 * 33];
  for (int q = threadIdx.x; q < 32 * 33; q += blockDim.x) sb[q] = b.binom32[q];
  __syncthreads();
  const uint32_t mask = (uint32_t)b.maskL;
  for (uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n;
       r += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t rem = (uint32_t)r, s = 0;
    int p = b.L - 1;
    for (int j = K; j >= 1; --j) {
      while (sb[p * 33 + j] > rem) --p;
      s |= 1u << p;
      rem -= sb[p * 33 + j];
      --p;
    }
    uint32_t key, extra = 0;  // extra: M (BK_TRANS) or the sign bit (BK_TRANSPAR)
    if (b.bk == BK_TRANS) {
      int M = 0;
      key = canon_arg32(s, b.L, b.A, b.len, mask, M);
      extra = (uint32_t)M;
    } else if (b.bk == BK_TRANSPAR) {  // the coefficient rule of lookup<BK_TRANSPAR>
      uint32_t Iam, Ibm;
      int Rr, M;
      canon_par32(s, b.L, b.A, b.len, mask, Iam, Rr, Ibm, M);
      double n;
      if (Ibm < Iam) { key = Ibm; n = (double)b.P * __ldg(b.phase + M).x; }
      else { key = Iam; n = __ldg(b.phase + Rr).x; }
      extra = n < 0.0 ? 1u : 0u;
    } else {
      key = b.runs_canon ? canon_runs32(s, b.L, mask) : canon_min32(s, b.L, b.A, b.len, mask);
    }
    uint32_t v;
    if (!hash_find(b, key, v)) {
      out[r] = ~0u;
      continue;
    }
    const uint32_t row = b.packed ? v >> 5 : v, cls = b.packed ? v & 31u : 0u;
    out[r] = (row << b.rank_shift) | (b.rank_shift > 5 ? extra << 5 : 0u) | cls;
  }
}

// colex rank of every representative (the row states of the rank search)
__global__ void k_row_rank(const uint64_t* I, int64_t D, const uint32_t* binom, uint32_t* out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < D;
       i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (uint32_t)colex_rank((uint32_t)I[i], binom);
}

int grid_for(int64_t n, int block = 256, int cap = 148 * 32) {
  int64_t g = (n + block - 1) / block;
  if (g < 1) g = 1;
  if (g > cap) g = cap;
  return (int)g;
}

std::vector<uint64_t> host_binom64() {
  std::vector<uint64_t> t(64 * 65, 0);
  for (int n = 0; n < 64; ++n) {
    t[n * 65 + 0] = 1;
    for (int k = 1; k <= n; ++k)
      t[n * 65 + k] = t[(n - 1) * 65 + k - 1] + ((k <= n - 1) ? t[(n - 1) * 65 + k] : 0);
  }
  return t;
}

// Compile a 1-based site permutation into delta-swap layers on bit positions
// (same decomposition into transpositions as compile_benes, AbelianBasis.jl:28-69).
bool compile_perm(const std::vector<int>& perm, int L, GenDev& g) {
  std::vector<int> bit_perm(L), current(L), where_is(L), inv_perm(L);
  for (int i = 1; i <= L; ++i) bit_perm[L - i] = L - perm[i - 1];
  for (int i = 0; i < L; ++i) { current[i] = i; where_is[i] = i; }
  for (int s = 0; s < L; ++s) inv_perm[bit_perm[s]] = s;
  g.nlayers = 0;
  for (int dst = 0; dst < L; ++dst) {
    int src_bit = inv_perm[dst];
    int cur_pos = where_is[src_bit];
    if (cur_pos != dst) {
      int lo = std::min(dst, cur_pos), hi = std::max(dst, cur_pos);
      if (g.nlayers >= kMaxLayers) return false;
      g.lmask[g.nlayers] = 1ull << lo;
      g.lshift[g.nlayers] = hi - lo;
      ++g.nlayers;
      int other_bit = current[dst];
      std::swap(current[dst], current[cur_pos]);
      where_is[src_bit] = dst;
      where_is[other_bit] = cur_pos;
    }
  }
  return true;
}

edk_status validate_desc(const edk_basis_desc* d) {
  EDK_CHECK_ARG(d != nullptr, "edk_basis_create: desc is NULL");
  EDK_CHECK_ARG(d->kind >= EDK_TENSOR && d->kind <= EDK_TRANSFLIP, "edk_basis_create: bad kind");
  if (d->kind == EDK_TRANSFLIP) {
    EDK_CHECK_ARG(d->ngen == 2 && d->gen_order && d->gen_q && d->gen_perm && d->gen_inv,
                  "edk_basis_create: TranslationFlipBasis takes two generators (T^a, flip)");
    EDK_CHECK_ARG(d->gen_order[1] == 2 && d->gen_order[0] >= 1,
                  "edk_basis_create: TranslationFlipBasis generators: translation, then flip");
  }
  EDK_CHECK_ARG(d->L >= 1, "edk_basis_create: L must be >= 1");
  if (d->base != 2) {
    set_error("edk_basis_create: the GPU path supports base 2 (spin-1/2) only");
    return EDK_UNSUPPORTED;
  }
  if (d->L > 63) {
    set_error("edk_basis_create: L > 63 does not fit a 64-bit state");
    return EDK_UNSUPPORTED;
  }
  if (d->kind == EDK_TENSOR && d->L > 34) {
    set_error("edk_basis_create: TensorBasis with L > 34 does not fit one device");
    return EDK_UNSUPPORTED;
  }
  if (d->kind == EDK_TRANSLATIONAL || d->kind == EDK_TRANSPARITY) {
    EDK_CHECK_ARG(d->a >= 1 && d->L % d->a == 0, "Length of unit-cell incompatible with L");
    EDK_CHECK_ARG(d->L / d->a <= 64, "edk_basis_create: more than 64 translations");
  }
  return EDK_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// Norm classes and the row lookup table
// ---------------------------------------------------------------------------
static edk_status build_hash(edk_basis* b, const uint8_t* cls_dev, cudaStream_t st) {
  int64_t D = b->D;
  uint64_t slots = 1024;
  while (slots < (uint64_t)(2 * D)) slots <<= 1;
  bool wide = b->L > 32;
  size_t slot_bytes = wide ? 16 : 8;
  EDK_RETURN_IF(b->htab.alloc(slots * slot_bytes));
  EDK_TRY_CUDA(cudaMemsetAsync(b->htab.p, 0xFF, slots * slot_bytes, st));
  b->dev.htab = b->htab.p;
  b->dev.hmask = slots - 1;
  int hbits = 0;
  while ((1ull << hbits) < slots) ++hbits;
  b->dev.hbits = hbits;
  if (!wide && hbits > 32) {
    set_error("edk_basis_create: lookup table beyond 2^32 slots");
    return EDK_UNSUPPORTED;
  }
  if (D == 0) return EDK_OK;
  if (wide)
    k_hash_insert64<<<grid_for(D), 256, 0, st>>>(b->I.as<uint64_t>(), cls_dev, D, b->dev.packed,
                                                  b->htab.as<ulonglong2>(), slots - 1);
  else
    k_hash_insert32<<<grid_for(D), 256, 0, st>>>(b->I.as<uint64_t>(), cls_dev, D,
                                                  b->dev.packed,
                                                  b->htab.as<unsigned long long>(), slots - 1,
                                                  hbits);
  EDK_TRY_CUDA(cudaGetLastError());
  return EDK_OK;
}

// Choose packing from the distinct norms (host list) and build the table.
static edk_status finish_lookup_from_R(edk_basis* b, const std::vector<double>& distinct,
                                       cudaStream_t st) {
  DevBuf cls;
  b->dev.nclass = (int)distinct.size();
  b->dev.packed = (distinct.size() <= (size_t)kNormClasses && b->D < (int64_t(1) << 27)) ? 1 : 0;
  if (b->dev.packed) {
    for (size_t q = 0; q < distinct.size(); ++q) b->dev.Rcls[q] = distinct[q];
    EDK_RETURN_IF(cls.alloc(std::max<int64_t>(b->D, 1)));
    if (b->D > 0 && b->R.p)
      k_cls_from_R<<<grid_for(b->D), 256, 0, st>>>(b->R.as<double>(), b->D, b->dev,
                                                    cls.as<uint8_t>());
    else if (b->D > 0)
      EDK_TRY_CUDA(cudaMemsetAsync(cls.p, 0, b->D, st));
    EDK_TRY_CUDA(cudaGetLastError());
  }
  EDK_RETURN_IF(build_hash(b, b->dev.packed ? cls.as<uint8_t>() : nullptr, st));
  EDK_TRY_CUDA(cudaStreamSynchronize(st));
  return EDK_OK;
}

// ---------------------------------------------------------------------------
// GPU construction
// ---------------------------------------------------------------------------
static edk_status gpu_build(edk_basis* b, const edk_basis_desc& d, cudaStream_t st) {
  int L = b->L;
  BuildParams p{};
  p.kind = b->kind;
  p.L = L; p.A = b->A; p.len = b->len; p.Kmom = b->Kmom; p.P = b->P;
  p.maskL = (L == 64) ? ~0ull : ((1ull << L) - 1);
  // candidates: states with K set bits, or all 2^L
  int K = -1;
  bool charged = d.N >= 0;
  if (b->kind == EDK_ABELIAN) K = d.N;              // Gosper path counts set bits
  else if (charged) K = L * (d.base - 1) - d.N;     // sum(dgt) == L(base-1) - N
  std::vector<uint64_t> hb = host_binom64();
  DevBuf binom;
  EDK_RETURN_IF(binom.alloc(hb.size() * 8));
  EDK_TRY_CUDA(cudaMemcpyAsync(binom.p, hb.data(), hb.size() * 8, cudaMemcpyHostToDevice, st));
  p.binom = binom.as<uint64_t>();
  if (charged) {
    p.full = 0;
    p.K = (K >= 0 && K <= L) ? K : 0;
    p.ncand = (K >= 0 && K <= L) ? hb[L * 65 + K] : 0;  // no state carries that charge
  } else {
    if (L > 36) {
      set_error("edk_basis_create: a full 2^L scan beyond L = 36 is not supported; give N");
      return EDK_UNSUPPORTED;
    }
    p.full = 1; p.K = 0; p.ncand = 1ull << L;
  }
  if (b->kind == EDK_TRANSPARITY) p.Kpar = (b->Kmom == 0) ? 1 : -1;
  // norm table, built with the reference's expressions
  std::vector<double> ntab;
  if (b->kind == EDK_TRANSLATIONAL) {
    for (int i = 1; i <= b->len; ++i) ntab.push_back((double)b->len / std::sqrt((double)i));
  } else if (b->kind == EDK_TRANSPARITY) {
    std::vector<double> n2(b->len);
    for (int i = 1; i <= b->len; ++i) n2[i - 1] = (double)(2 * b->len) / std::sqrt((double)i);
    for (int i = 0; i < b->len; ++i) ntab.push_back(n2[i] / std::sqrt(2.0));
    for (int i = 0; i < b->len; ++i) ntab.push_back(n2[i]);
  } else if (b->kind == EDK_ABELIAN) {
    int64_t Ng = 1;
    for (int o : b->gen_order) Ng *= o;
    if (Ng > kMaxNormTab) {
      set_error("edk_basis_create: abelian group order above 128 is not supported");
      return EDK_UNSUPPORTED;
    }
    if (b->pairnorm) {  // TranslationFlipBasis: vcat(N1, N2), N2 = 2len/sqrt(i), N1 = N2/sqrt(2)
      const int len = b->gen_order[0];
      std::vector<double> n2(len);
      for (int i = 1; i <= len; ++i) n2[i - 1] = (double)(2 * len) / std::sqrt((double)i);
      for (int i = 0; i < len; ++i) ntab.push_back(n2[i] / std::sqrt(2.0));
      for (int i = 0; i < len; ++i) ntab.push_back(n2[i]);
      p.pairnorm = 1;
    } else {
      for (int64_t i = 1; i <= Ng; ++i)
        ntab.push_back((Ng % i == 0) ? std::sqrt((double)(Ng * i)) : 0.0);
    }
    p.ngen = (int)b->gens_host.size();
    p.gens = b->gens.as<GenDev>();
    p.gphase = b->phase.as<double2>();
  }
  DevBuf allow;
  if (d.allow) {
    if (L > 34) {
      set_error("edk_basis_create: a predicate bitmap needs L <= 34");
      return EDK_UNSUPPORTED;
    }
    size_t words = ((1ull << L) + 63) / 64;
    EDK_RETURN_IF(allow.alloc(words * 8));
    EDK_TRY_CUDA(cudaMemcpyAsync(allow.p, d.allow, words * 8, cudaMemcpyHostToDevice, st));
    p.allow = allow.as<unsigned long long>();
  }
  uint64_t nchunks = (p.ncand + kChunk - 1) / kChunk;
  DevBuf counts, offsets, cls, tmp;
  EDK_RETURN_IF(counts.alloc(std::max<uint64_t>(nchunks, 1) * 4));
  EDK_RETURN_IF(offsets.alloc((nchunks + 1) * 8));
  bool wide = L > 32;
  int nb = (int)((nchunks + 255) / 256);
  if (nchunks > 0) {
    if (wide) k_build_count<uint64_t><<<nb, 256, 0, st>>>(p, nchunks, counts.as<uint32_t>());
    else k_build_count<uint32_t><<<nb, 256, 0, st>>>(p, nchunks, counts.as<uint32_t>());
    EDK_TRY_CUDA(cudaGetLastError());
  }
  // exclusive scan of the chunk counts into 64-bit offsets (+ total)
  EDK_TRY_CUDA(cudaMemsetAsync(offsets.p, 0, 8, st));
  if (nchunks > 0) {
    size_t tb = 0;
    auto in = counts.as<uint32_t>();
    auto out = offsets.as<uint64_t>() + 1;
    cub::DeviceScan::InclusiveSum(nullptr, tb, in, out, (int64_t)nchunks, st);
    EDK_RETURN_IF(tmp.alloc(std::max<size_t>(tb, 16)));
    cub::DeviceScan::InclusiveSum(tmp.p, tb, in, out, (int64_t)nchunks, st);
    EDK_TRY_CUDA(cudaGetLastError());
  }
  uint64_t total = 0;
  EDK_TRY_CUDA(cudaMemcpyAsync(&total, offsets.as<uint64_t>() + nchunks, 8,
                               cudaMemcpyDeviceToHost, st));
  EDK_TRY_CUDA(cudaStreamSynchronize(st));
  b->D = (int64_t)total;
  EDK_RETURN_IF(b->I.alloc(std::max<uint64_t>(total, 1) * 8));
  bool symm = b->kind != EDK_PROJECTED;
  if (symm) EDK_RETURN_IF(cls.alloc(std::max<uint64_t>(total, 1)));
  if (nchunks > 0) {
    if (wide)
      k_build_write<uint64_t><<<nb, 256, 0, st>>>(p, nchunks, offsets.as<uint64_t>(),
                                                   b->I.as<uint64_t>(),
                                                   symm ? cls.as<uint8_t>() : nullptr);
    else
      k_build_write<uint32_t><<<nb, 256, 0, st>>>(p, nchunks, offsets.as<uint64_t>(),
                                                   b->I.as<uint64_t>(),
                                                   symm ? cls.as<uint8_t>() : nullptr);
    EDK_TRY_CUDA(cudaGetLastError());
  }
  if (!symm) {
    EDK_TRY_CUDA(cudaStreamSynchronize(st));
    return EDK_OK;
  }
  // compact the norm classes actually used and fill R
  DevBuf hist, dntab, dremap;
  EDK_RETURN_IF(hist.alloc(kMaxNormTab * 4));
  EDK_TRY_CUDA(cudaMemsetAsync(hist.p, 0, kMaxNormTab * 4, st));
  if (total > 0)
    k_cls_hist<<<grid_for(total), 256, 0, st>>>(cls.as<uint8_t>(), total, hist.as<unsigned>());
  std::vector<unsigned> hh(kMaxNormTab);
  EDK_TRY_CUDA(cudaMemcpyAsync(hh.data(), hist.p, kMaxNormTab * 4, cudaMemcpyDeviceToHost, st));
  EDK_TRY_CUDA(cudaStreamSynchronize(st));
  std::vector<int> remap(kMaxNormTab, 0);
  std::vector<double> used;
  for (int c = 0; c < (int)ntab.size(); ++c) {
    if (!hh[c]) continue;
    int q = -1;
    for (size_t u = 0; u < used.size(); ++u) if (used[u] == ntab[c]) q = (int)u;
    if (q < 0) { q = (int)used.size(); used.push_back(ntab[c]); }
    remap[c] = q;
  }
  ntab.resize(kMaxNormTab, 0.0);
  EDK_RETURN_IF(dntab.alloc(kMaxNormTab * 8));
  EDK_RETURN_IF(dremap.alloc(kMaxNormTab * 4));
  EDK_TRY_CUDA(cudaMemcpyAsync(dntab.p, ntab.data(), kMaxNormTab * 8, cudaMemcpyHostToDevice, st));
  EDK_TRY_CUDA(cudaMemcpyAsync(dremap.p, remap.data(), kMaxNormTab * 4, cudaMemcpyHostToDevice, st));
  EDK_RETURN_IF(b->R.alloc(std::max<uint64_t>(total, 1) * 8));
  if (total > 0)
    k_cls_apply<<<grid_for(total), 256, 0, st>>>(cls.as<uint8_t>(), total, dntab.as<double>(),
                                                 dremap.as<int>(), b->R.as<double>());
  EDK_TRY_CUDA(cudaGetLastError());
  b->dev.nclass = (int)used.size();
  b->dev.packed = (used.size() <= (size_t)kNormClasses && b->D < (int64_t(1) << 27)) ? 1 : 0;
  for (size_t q = 0; q < used.size() && q < (size_t)kNormClasses; ++q) b->dev.Rcls[q] = used[q];
  EDK_RETURN_IF(build_hash(b, b->dev.packed ? cls.as<uint8_t>() : nullptr, st));
  EDK_TRY_CUDA(cudaStreamSynchronize(st));
  return EDK_OK;
}

// upload Julia-held tables
static edk_status upload_tables(edk_basis* b, const edk_basis_desc& d, cudaStream_t st) {
  int64_t D = d.D;
  EDK_CHECK_ARG(D >= 0, "edk_basis_create: D < 0");
  const uint64_t lim = (b->L >= 64) ? ~0ull : (1ull << b->L);
  for (int64_t i = 0; i < D; ++i) {
    EDK_CHECK_ARG(d.I[i] >= 1 && (uint64_t)(d.I[i] - 1) < lim,
                  "edk_basis_create: I holds an index outside 1:base^L");
    if (i > 0) EDK_CHECK_ARG(d.I[i] > d.I[i - 1], "edk_basis_create: I must be strictly ascending");
  }
  b->D = D;
  EDK_RETURN_IF(b->I.alloc(std::max<int64_t>(D, 1) * 8));
  DevBuf tmp;
  EDK_RETURN_IF(tmp.alloc(std::max<int64_t>(D, 1) * 8));
  if (D > 0) {
    EDK_TRY_CUDA(cudaMemcpyAsync(tmp.p, d.I, D * 8, cudaMemcpyHostToDevice, st));
    k_to_states<<<grid_for(D), 256, 0, st>>>(tmp.as<int64_t>(), D, b->I.as<uint64_t>());
    EDK_TRY_CUDA(cudaGetLastError());
  }
  std::vector<double> distinct;
  if (b->kind != EDK_PROJECTED) {
    EDK_CHECK_ARG(d.R != nullptr, "edk_basis_create: symmetric bases need R with I");
    EDK_RETURN_IF(b->R.alloc(std::max<int64_t>(D, 1) * 8));
    if (D > 0)
      EDK_TRY_CUDA(cudaMemcpyAsync(b->R.p, d.R, D * 8, cudaMemcpyHostToDevice, st));
    std::set<double> ds;
    for (int64_t i = 0; i < D && ds.size() <= (size_t)kNormClasses; ++i) ds.insert(d.R[i]);
    distinct.assign(ds.begin(), ds.end());
  } else {
    distinct.push_back(1.0);
  }
  return finish_lookup_from_R(b, distinct, st);
}

}  // namespace edk

using namespace edk;

edk_basis::~edk_basis() {
  if (stream) cudaStreamDestroy(stream);
}

extern "C" edk_status edk_basis_create(const edk_basis_desc* desc, edk_basis** out) {
  EDK_CHECK_ARG(out != nullptr, "edk_basis_create: out is NULL");
  *out = nullptr;
  EDK_RETURN_IF(validate_desc(desc));
  auto* b = new edk_basis;
  std::unique_ptr<edk_basis> guard(b);
  b->desc = *desc;
  // TranslationFlipBasis: the generic symmetry-group path with its own norms
  b->pairnorm = desc->kind == EDK_TRANSFLIP;
  b->kind = b->pairnorm ? (int)EDK_ABELIAN : desc->kind;
  b->desc.kind = b->kind;
  b->L = desc->L;
  b->A = (desc->kind == EDK_TRANSLATIONAL || desc->kind == EDK_TRANSPARITY) ? desc->a : 1;
  b->len = b->L / b->A;
  b->desc.I = nullptr;  // host pointers are borrowed only for this call
  b->desc.R = nullptr;
  b->desc.gen_order = b->desc.gen_q = b->desc.gen_perm = nullptr;
  b->desc.gen_inv = nullptr;
  b->desc.allow = nullptr;
  EDK_TRY_CUDA(cudaGetDevice(&b->device));
  EDK_TRY_CUDA(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
  cudaStream_t st = b->stream;
  BasisDev& dv = b->dev;
  dv.L = b->L; dv.A = b->A; dv.len = b->len;
  dv.maskL = (b->L == 64) ? ~0ull : ((1ull << b->L) - 1);
  dv.P = 1;
  dv.phase_real = 1;
  // phase tables
  std::vector<double2> ph;
  if (b->kind == EDK_TRANSLATIONAL) {
    int len = b->len;
    int K = ((-desc->k) % len + len) % len;  // k = mod(-k, len)  TranslationalBasis.jl:247
    b->Kmom = K;
    const double twopi = 2.0 * M_PI;
    for (int i = 0; i < len; ++i) {  // phase_factor  TranslationalBasis.jl:277-285
      double re, im;
      if (K == 0) { re = 1.0; im = 0.0; }
      else if (2 * K == len) { re = (i % 2 == 0) ? 1.0 : -1.0; im = 0.0; }
      else {
        double th = ((-twopi / (double)len) * (double)K) * (double)i;
        if (i == 0) { re = 1.0; im = th; }
        else { re = std::cos(th); im = std::sin(th); }
      }
      ph.push_back(make_double2(re, im));
    }
    b->phase_complex = !(K == 0 || 2 * K == len);
  } else if (b->kind == EDK_TRANSPARITY) {
    int len = b->len, k = desc->k;
    int Kp;  // TranslationalParityBasis.jl:147-153
    if (((k % len) + len) % len == 0) Kp = 1;
    else if ((((2 * k) % len) + len) % len == 0) Kp = -1;
    else {
      set_error("Momentum " + std::to_string(k) + " incompatible with parity.");
      return EDK_INVALID_ARG;
    }
    EDK_CHECK_ARG(desc->p == 1 || desc->p == -1, "Invalid parity");
    b->Kmom = (Kp == 1) ? 0 : 1;
    b->P = desc->p;
    dv.P = desc->p;
    for (int i = 0; i < len; ++i)
      ph.push_back(make_double2((Kp == 1) ? 1.0 : ((i % 2 == 0) ? 1.0 : -1.0), 0.0));
  } else if (b->kind == EDK_ABELIAN) {
    EDK_CHECK_ARG(desc->ngen >= 1 && desc->ngen <= kMaxGen,
                  "edk_basis_create: abelian basis needs 1..8 generators");
    EDK_CHECK_ARG(desc->gen_order && desc->gen_q && desc->gen_perm && desc->gen_inv,
                  "edk_basis_create: abelian generator arrays are NULL");
    const double twopi = 2.0 * M_PI;
    int L = b->L;
    for (int g = 0; g < desc->ngen; ++g) {
      GenDev gd{};
      int order = desc->gen_order[g], q = desc->gen_q[g];
      EDK_CHECK_ARG(order >= 1, "edk_basis_create: generator order < 1");
      std::vector<int> perm(desc->gen_perm + (size_t)g * L, desc->gen_perm + (size_t)(g + 1) * L);
      std::vector<uint8_t> inv(desc->gen_inv + (size_t)g * L, desc->gen_inv + (size_t)(g + 1) * L);
      std::vector<int> seen(L + 1, 0);
      for (int i = 0; i < L; ++i) {
        EDK_CHECK_ARG(perm[i] >= 1 && perm[i] <= L && !seen[perm[i]],
                      "edk_basis_create: generator is not a permutation");
        seen[perm[i]] = 1;
      }
      gd.order = order;
      gd.phase_off = (int)ph.size();
      for (int j = 0; j < order; ++j) {  // AbelianOperator phases AbelianBasis.jl:167-176
        double re, im;
        if (q == 0) { re = 1.0; im = 0.0; }
        else if (2 * q == order) { re = (j % 2 == 0) ? 1.0 : -1.0; im = 0.0; }
        else {
          double th = ((twopi * (double)q) / (double)order) * (double)j;
          if (j == 0) { re = 1.0; im = th; }
          else { re = std::cos(th); im = std::sin(th); }
          b->phase_complex = true;
        }
        ph.push_back(make_double2(re, im));
      }
      for (int i = 1; i <= L; ++i) if (inv[i - 1]) gd.inv_mask |= 1ull << (L - i);
      // classify: identity, rotation (site i -> i - s mod L), reversal, generic
      bool ident = true, rev = true;
      for (int i = 1; i <= L; ++i) {
        ident &= perm[i - 1] == i;
        rev &= perm[i - 1] == L - i + 1;
      }
      int rot = -1;
      for (int s = 1; s < L && rot < 0; ++s) {
        bool ok = true;
        for (int i = 1; i <= L && ok; ++i) ok = perm[i - 1] == ((i - s - 1) % L + L) % L + 1;
        if (ok) rot = s;
      }
      if (ident) gd.kind = GEN_ID;
      else if (rot > 0) { gd.kind = GEN_ROTL; gd.shift = rot; }
      else if (rev) gd.kind = GEN_REV;
      else {
        gd.kind = GEN_PERM;
        if (!compile_perm(perm, L, gd)) {
          set_error("edk_basis_create: permutation network too deep");
          return EDK_UNSUPPORTED;
        }
      }
      b->gens_host.push_back(gd);
      b->gen_order.push_back(order);
      b->gen_q.push_back(q);
      b->gen_perm.push_back(perm);
      b->gen_inv.push_back(inv);
    }
    EDK_RETURN_IF(b->gens.alloc(b->gens_host.size() * sizeof(GenDev)));
    EDK_TRY_CUDA(cudaMemcpyAsync(b->gens.p, b->gens_host.data(),
                                 b->gens_host.size() * sizeof(GenDev), cudaMemcpyHostToDevice, st));
    dv.ngen = (int)b->gens_host.size();
    dv.gens = b->gens.as<GenDev>();
  }
  if (!ph.empty()) {
    EDK_RETURN_IF(b->phase.alloc(ph.size() * sizeof(double2)));
    EDK_TRY_CUDA(cudaMemcpyAsync(b->phase.p, ph.data(), ph.size() * sizeof(double2),
                                 cudaMemcpyHostToDevice, st));
    dv.phase = b->phase.as<double2>();
  }
  dv.phase_real = b->phase_complex ? 0 : 1;

  // tables
  if (b->kind == EDK_TENSOR) {
    b->D = int64_t(1) << b->L;
    dv.bk = BK_TENSOR;
  } else {
    if (desc->I) EDK_RETURN_IF(upload_tables(b, *desc, st));
    else EDK_RETURN_IF(gpu_build(b, *desc, st));
    if (b->kind == EDK_PROJECTED) {
      // exact colex rank when I is the complete fixed-popcount sector (L <= 32)
      bool rank = false;
      if (b->L <= 32 && b->D > 0) {
        uint64_t first = 0, last = 0;
        EDK_TRY_CUDA(cudaMemcpyAsync(&first, b->I.p, 8, cudaMemcpyDeviceToHost, st));
        EDK_TRY_CUDA(cudaMemcpyAsync(&last, b->I.as<uint64_t>() + b->D - 1, 8,
                                     cudaMemcpyDeviceToHost, st));
        EDK_TRY_CUDA(cudaStreamSynchronize(st));
        int K = __builtin_popcountll(first);
        std::vector<uint64_t> hb = host_binom64();
        uint64_t firstK = (K == 0) ? 0 : ((1ull << K) - 1);
        uint64_t lastK = (K == 0) ? 0 : (((1ull << K) - 1) << (b->L - K));
        // sorted + unique + correct count + matching endpoints + all popcount K
        // (popcount checked on the host copy when the tables came from Julia)
        bool allK = true;
        if (desc->I) for (int64_t i = 0; i < desc->D && allK; ++i)
          allK = __builtin_popcountll((uint64_t)(desc->I[i] - 1)) == K;
        else allK = desc->N >= 0 && desc->allow == nullptr;
        rank = allK && first == firstK && last == lastK && (uint64_t)b->D == hb[b->L * 65 + K];
        dv.K = K;
      }
      dv.bk = rank ? BK_PROJ_RANK : BK_PROJ_HASH;
      if (!rank && !b->htab.p) {
        // GPU-built projected tables without the complete-sector structure
        // (predicate bases) are looked up through the hash table
        std::vector<double> one(1, 1.0);
        EDK_RETURN_IF(finish_lookup_from_R(b, one, st));
      }
    } else if (b->kind == EDK_TRANSLATIONAL) {
      dv.bk = (b->Kmom == 0) ? BK_TRANS0 : BK_TRANS;
      const char* e = std::getenv("EDK_CANON_RUNS");
      dv.runs_canon = (dv.bk == BK_TRANS0 && b->A == 1 && b->L <= 32 && e && e[0] == '1') ? 1 : 0;
    } else if (b->kind == EDK_TRANSPARITY) {
      dv.bk = BK_TRANSPAR;
    } else {
      dv.bk = BK_ABELIAN;
    }
  }
  dv.D = b->D;
  dv.I = b->I.as<uint64_t>();
  dv.R = (b->kind == EDK_TENSOR || b->kind == EDK_PROJECTED) ? nullptr : b->R.as<double>();
  EDK_TRY_CUDA(cudaStreamSynchronize(st));
  *out = guard.release();
  return EDK_OK;
}

// Select the index search of a basis with a representative table: the hash
// table (default) or the two-level binary search over the sorted array.
namespace {
// EDK_SEARCH_RANK: build the rank table once (kept until the basis is freed)
edk_status build_rank_table(edk_basis* b) {
  if ((b->rankmap.p && b->rowrank.p) || b->D == 0) return EDK_OK;
  // a build that failed part-way (out of memory) starts again from nothing
  b->rankmap.release();
  b->rowrank.release();
  cudaStream_t st = b->stream;
  const int L = b->L;
  uint64_t s0 = 0;
  EDK_TRY_CUDA(cudaMemcpyAsync(&s0, b->I.p, sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
  EDK_TRY_CUDA(cudaStreamSynchronize(st));
  const int K = __builtin_popcountll(s0);
  DevBuf flag;
  EDK_RETURN_IF(flag.alloc(sizeof(int)));
  EDK_TRY_CUDA(cudaMemsetAsync(flag.p, 0, sizeof(int), st));
  k_popc_check<<<grid_for(b->D), 256, 0, st>>>(b->I.as<uint64_t>(), b->D, K, flag.as<int>());
  EDK_TRY_CUDA(cudaGetLastError());
  int mixed = 0;
  EDK_TRY_CUDA(cudaMemcpyAsync(&mixed, flag.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  EDK_TRY_CUDA(cudaStreamSynchronize(st));
  if (mixed) {
    set_error("edk_basis_set_search: the rank table needs a sector of fixed charge N");
    return EDK_UNSUPPORTED;
  }
  std::vector<uint32_t> binom(32 * 33, 0);
  for (int p = 0; p < 32; ++p) {
    binom[p * 33] = 1;
    for (int k = 1; k <= p; ++k)
      binom[p * 33 + k] = (p == 0) ? 0 : binom[(p - 1) * 33 + k - 1] + binom[(p - 1) * 33 + k];
  }
  uint64_t n = 1;  // C(L, K)
  for (int k = 1; k <= K; ++k) n = n * (uint64_t)(L - K + k) / (uint64_t)k;
  EDK_CHECK_ARG(n <= 0xFFFFFFFFull, "edk_basis_set_search: the sector has more than 2^32 states");
  EDK_RETURN_IF(b->binom32.alloc(binom.size() * sizeof(uint32_t)));
  EDK_TRY_CUDA(cudaMemcpyAsync(b->binom32.p, binom.data(), binom.size() * sizeof(uint32_t),
                               cudaMemcpyHostToDevice, st));
  EDK_RETURN_IF(b->rankmap.alloc(n * sizeof(uint32_t)));
  BasisDev tmp = b->dev;
  tmp.search = 0;
  tmp.binom32 = b->binom32.as<uint32_t>();
  tmp.rank_shift = b->dev.rank_shift;
  k_rank_map<<<grid_for((int64_t)n), 256, 0, st>>>(tmp, K, n, b->rankmap.as<uint32_t>());
  EDK_TRY_CUDA(cudaGetLastError());
  EDK_RETURN_IF(b->rowrank.alloc(b->D * sizeof(uint32_t)));
  k_row_rank<<<grid_for(b->D), 256, 0, st>>>(b->I.as<uint64_t>(), b->D, b->binom32.as<uint32_t>(),
                                             b->rowrank.as<uint32_t>());
  EDK_TRY_CUDA(cudaGetLastError());
  EDK_TRY_CUDA(cudaStreamSynchronize(st));
  return EDK_OK;
}
}  // namespace

extern "C" edk_status edk_basis_set_search(edk_basis* b, int32_t strategy) {
  EDK_CHECK_ARG(b != nullptr, "edk_basis_set_search: NULL basis");
  EDK_CHECK_ARG(strategy == EDK_SEARCH_HASH || strategy == EDK_SEARCH_SORTED ||
                    strategy == EDK_SEARCH_RANK,
                "edk_basis_set_search: unknown strategy");
  std::lock_guard<std::mutex> lk(b->mu);
  const int bk = b->dev.bk;
  if (bk == BK_TENSOR || bk == BK_PROJ_RANK) {
    set_error("edk_basis_set_search: this basis indexes rows directly (tensor product or "
              "complete fixed-charge sector), there is no representative search to choose");
    return EDK_UNSUPPORTED;
  }
  if (strategy == EDK_SEARCH_HASH) {
    b->dev.search = 0;
    return EDK_OK;
  }
  if (strategy == EDK_SEARCH_RANK) {
    // entries: row << 10 | M << 5 | class while rows fit 22 bits, else (k = 0
    // only, no phase needed) row << 5 | class
    const int shift = bk == BK_TRANSPAR ? 6 : (b->D < (1ll << 22) ? 10 : 5);
    if ((bk != BK_TRANS0 && bk != BK_TRANS && bk != BK_TRANSPAR) || b->L > 32 ||
        (bk == BK_TRANS && shift != 10) || b->D >= (1ll << (32 - shift))) {
      set_error("edk_basis_set_search: the rank table serves translation and "
                "translation-parity sectors of fixed N with L <= 32 (fewer than 2^22 rows "
                "when k has a phase, 2^26 with parity)");
      return EDK_UNSUPPORTED;
    }
    b->dev.rank_shift = shift;
    EDK_RETURN_IF(build_rank_table(b));
    b->dev.rankmap = b->rankmap.as<uint32_t>();
    b->dev.binom32 = b->binom32.as<uint32_t>();
    b->dev.rowrank = b->rowrank.as<uint32_t>();
    b->dev.search = 2;
    return EDK_OK;
  }
  if (!b->keys32.p && !b->fence.p && b->D > 0) {
    cudaStream_t st = b->stream;
    const bool narrow = b->L <= 32;
    DevBuf flag;
    EDK_RETURN_IF(flag.alloc(sizeof(int)));
    EDK_TRY_CUDA(cudaMemsetAsync(flag.p, 0, sizeof(int), st));
    const int64_t nf = (b->D + 31) / 32;
    if (narrow) {
      EDK_RETURN_IF(b->keys32.alloc(b->D * sizeof(uint32_t)));
      EDK_RETURN_IF(b->fence.alloc(nf * sizeof(uint32_t)));
    }
    k_sorted_tables<<<grid_for(b->D), 256, 0, st>>>(
        b->I.as<uint64_t>(), b->D, narrow ? b->keys32.as<uint32_t>() : nullptr,
        narrow ? b->fence.as<uint32_t>() : nullptr, flag.as<int>());
    EDK_TRY_CUDA(cudaGetLastError());
    if (b->dev.packed) {
      EDK_RETURN_IF(b->rcls8.alloc(b->D));
      if (b->R.p)
        k_cls_from_R<<<grid_for(b->D), 256, 0, st>>>(b->R.as<double>(), b->D, b->dev,
                                                      b->rcls8.as<uint8_t>());
      else
        EDK_TRY_CUDA(cudaMemsetAsync(b->rcls8.p, 0, b->D, st));
      EDK_TRY_CUDA(cudaGetLastError());
    }
    int unsorted = 0;
    EDK_TRY_CUDA(cudaMemcpyAsync(&unsorted, flag.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    EDK_TRY_CUDA(cudaStreamSynchronize(st));
    if (unsorted) {
      b->keys32.release(); b->fence.release(); b->rcls8.release();
      set_error("edk_basis_set_search: the representatives are not in ascending order");
      return EDK_INVALID_ARG;
    }
    b->dev.keys32 = narrow ? b->keys32.as<uint32_t>() : nullptr;
    b->dev.fence = narrow ? b->fence.as<uint32_t>() : nullptr;
    b->dev.nfence = narrow ? nf : 0;
    b->dev.rcls8 = b->dev.packed ? b->rcls8.as<uint8_t>() : nullptr;
  }
  b->dev.search = 1;
  return EDK_OK;
}

extern "C" edk_status edk_basis_get_search(const edk_basis* b, int32_t* strategy) {
  EDK_CHECK_ARG(b != nullptr && strategy != nullptr, "edk_basis_get_search: NULL argument");
  *strategy = b->dev.search == 2 ? EDK_SEARCH_RANK
               : (b->dev.search == 1 ? EDK_SEARCH_SORTED : EDK_SEARCH_HASH);
  return EDK_OK;
}

namespace edk {
// Host-side guard run before every kernel launch that reads the basis tables:
// a lookup kind is only launched with the tables it dereferences.
edk_status check_basis_dev(const BasisDev& b) {
  bool ok = true;
  switch (b.bk) {
    case BK_TENSOR: break;
    case BK_PROJ_RANK: ok = b.I != nullptr && b.L <= 32; break;
    case BK_PROJ_HASH: ok = b.I != nullptr && b.htab != nullptr; break;
    case BK_TRANS0:
    case BK_TRANS:
    case BK_TRANSPAR:
      ok = b.I != nullptr && b.R != nullptr && b.htab != nullptr && b.phase != nullptr &&
           b.len >= 1 && b.len <= 64;
      break;
    case BK_ABELIAN:
      ok = b.I != nullptr && b.R != nullptr && b.htab != nullptr && b.phase != nullptr &&
           b.gens != nullptr && b.ngen >= 1 && b.ngen <= kMaxGen;
      break;
    default: ok = false;
  }
  if (ok && b.search == 1 && b.bk != BK_TENSOR && b.bk != BK_PROJ_RANK)
    ok = (b.L <= 32) ? (b.keys32 != nullptr && b.fence != nullptr) : b.I != nullptr;
  if (ok && b.search == 1 && b.packed && b.bk != BK_TENSOR && b.bk != BK_PROJ_RANK)
    ok = b.rcls8 != nullptr;
  if (ok && b.search == 2)
    ok = ((b.bk == BK_TRANS0 && (b.rank_shift == 5 || b.rank_shift == 10)) ||
          (b.bk == BK_TRANS && b.rank_shift == 10) ||
          (b.bk == BK_TRANSPAR && b.rank_shift == 6)) &&
         b.L <= 32 && b.rankmap != nullptr && b.binom32 != nullptr && b.rowrank != nullptr;
  if (b.D > 0 && !ok) {
    set_error("internal: basis tables missing for its lookup kind");
    return EDK_INVALID_ARG;
  }
  return EDK_OK;
}
}  // namespace edk

extern "C" edk_status edk_basis_destroy(edk_basis* b) {
  delete b;
  return EDK_OK;
}

extern "C" edk_status edk_basis_dim(const edk_basis* b, int64_t* D) {
  EDK_CHECK_ARG(b && D, "edk_basis_dim: NULL argument");
  *D = b->D;
  return EDK_OK;
}

extern "C" edk_status edk_basis_export(const edk_basis* bc, int64_t* I, double* R) {
  EDK_CHECK_ARG(bc != nullptr, "edk_basis_export: NULL basis");
  edk_basis* b = const_cast<edk_basis*>(bc);
  std::lock_guard<std::mutex> lk(b->mu);
  cudaStream_t st = b->stream;
  int64_t D = b->D;
  if (D == 0) return EDK_OK;
  if (I) {
    if (b->kind == EDK_TENSOR) {
      for (int64_t i = 0; i < D; ++i) I[i] = i + 1;
    } else {
      DevBuf tmp;
      EDK_RETURN_IF(tmp.alloc(D * 8));
      k_to_julia<<<grid_for(D), 256, 0, st>>>(b->I.as<uint64_t>(), D, tmp.as<int64_t>());
      EDK_TRY_CUDA(cudaGetLastError());
      EDK_TRY_CUDA(cudaMemcpyAsync(I, tmp.p, D * 8, cudaMemcpyDeviceToHost, st));
      EDK_TRY_CUDA(cudaStreamSynchronize(st));
    }
  }
  if (R) {
    if (b->R.p) {
      EDK_TRY_CUDA(cudaMemcpyAsync(R, b->R.p, D * 8, cudaMemcpyDeviceToHost, st));
      EDK_TRY_CUDA(cudaStreamSynchronize(st));
    } else {
      for (int64_t i = 0; i < D; ++i) R[i] = 1.0;
    }
  }
  return EDK_OK;
}

namespace edk {
// launch index() for n device-resident states on stream st (no allocation);
// used by edk_basis_index_noalloc
edk_status index_device(const BasisDev& dv, int64_t n, const uint64_t* s_d, int64_t* p_d,
                        double2* c_d, cudaStream_t st) {
  EDK_RETURN_IF(check_basis_dev(dv));
  if (n <= 0) return EDK_OK;
  bool wide = dv.L > 32;
  int g = grid_for(n);
#define EDK_IDX(BK)                                                                 \
  case BK:                                                                          \
    if (wide) k_index<BK, uint64_t><<<g, 256, 0, st>>>(dv, n, s_d, p_d, c_d);       \
    else k_index<BK, uint32_t><<<g, 256, 0, st>>>(dv, n, s_d, p_d, c_d);            \
    break;
  switch (dv.bk) {
    EDK_IDX(BK_TENSOR)
    EDK_IDX(BK_PROJ_RANK)
    EDK_IDX(BK_PROJ_HASH)
    EDK_IDX(BK_TRANS0)
    EDK_IDX(BK_TRANS)
    EDK_IDX(BK_TRANSPAR)
    EDK_IDX(BK_ABELIAN)
  }
#undef EDK_IDX
  EDK_TRY_CUDA(cudaGetLastError());
  return EDK_OK;
}
}  // namespace edk

extern "C" edk_status edk_basis_index(const edk_basis* bc, int64_t n, const uint64_t* states,
                                      int64_t* pos, double* coeff, int32_t ptr_kind) {
  EDK_CHECK_ARG(bc && states && pos && coeff, "edk_basis_index: NULL argument");
  EDK_CHECK_ARG(n >= 0, "edk_basis_index: n < 0");
  edk_basis* b = const_cast<edk_basis*>(bc);
  std::lock_guard<std::mutex> lk(b->mu);
  if (n == 0) return EDK_OK;
  cudaStream_t st = b->stream;
  DevBuf ds, dp, dc;
  const uint64_t* s_d = states;
  int64_t* p_d = pos;
  double2* c_d = reinterpret_cast<double2*>(coeff);
  if (ptr_kind == EDK_HOST) {
    EDK_RETURN_IF(ds.alloc(n * 8));
    EDK_RETURN_IF(dp.alloc(n * 8));
    EDK_RETURN_IF(dc.alloc(n * 16));
    EDK_TRY_CUDA(cudaMemcpyAsync(ds.p, states, n * 8, cudaMemcpyHostToDevice, st));
    s_d = ds.as<uint64_t>(); p_d = dp.as<int64_t>(); c_d = dc.as<double2>();
  }
  const BasisDev& dv = b->dev;
  EDK_RETURN_IF(check_basis_dev(dv));
  bool wide = dv.L > 32;
  int g = grid_for(n);
#define EDK_IDX(BK)                                                                 \
  case BK:                                                                          \
    if (wide) k_index<BK, uint64_t><<<g, 256, 0, st>>>(dv, n, s_d, p_d, c_d);       \
    else k_index<BK, uint32_t><<<g, 256, 0, st>>>(dv, n, s_d, p_d, c_d);            \
    break;
  switch (dv.bk) {
    EDK_IDX(BK_TENSOR)
    EDK_IDX(BK_PROJ_RANK)
    EDK_IDX(BK_PROJ_HASH)
    EDK_IDX(BK_TRANS0)
    EDK_IDX(BK_TRANS)
    EDK_IDX(BK_TRANSPAR)
    EDK_IDX(BK_ABELIAN)
  }
#undef EDK_IDX
  EDK_TRY_CUDA(cudaGetLastError());
  if (ptr_kind == EDK_HOST) {
    EDK_TRY_CUDA(cudaMemcpyAsync(pos, p_d, n * 8, cudaMemcpyDeviceToHost, st));
    EDK_TRY_CUDA(cudaMemcpyAsync(coeff, c_d, n * 16, cudaMemcpyDeviceToHost, st));
  }
  EDK_TRY_CUDA(cudaStreamSynchronize(st));
  return EDK_OK;
}
