// edk_oracle.cpp — CPU restatement of EDKit.jl's basis tables, `index`, and
// matrix-free `Operator` application (column scatter, thread-private outputs).
//
// TEST INFRASTRUCTURE ONLY.  This file is the parity oracle and the timed CPU
// baseline.  Only tests/, __graft_entry__.smoke() and bench.py's CPU legs may
// load it; the product library (libedk.so) never links or calls it.
//
// Conventions follow the Julia reference exactly:
//   * digit strings are big-endian: dgt[0] is the most significant digit
//     (src/Basis/AbstractBasis.jl:285-298);
//   * tables hold 1-based indices `I` (Julia `Vector{Int}`), norms `R`;
//   * `index(b, dgt)` returns (coefficient, 1-based position), absent -> (0, 1).
//
// Every function cites the reference file:line it restates.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>
#include <omp.h>

using cplx = std::complex<double>;

namespace {

thread_local std::string g_err;

typedef int (*orc_pred)(const int64_t* dgt, int L, void* ud);

int64_t ipow(int64_t b, int e) { int64_t r = 1; while (e-- > 0) r *= b; return r; }

// index(dgt; base) — AbstractBasis.jl:285-298 (returns 1-based)
inline int64_t index_dgt(const int64_t* dgt, int L, int64_t base) {
  int64_t N = 0;
  if (base == 2) { for (int i = 0; i < L; ++i) N = (N << 1) | dgt[i]; }
  else { for (int i = 0; i < L; ++i) { N *= base; N += dgt[i]; } }
  return N + 1;
}
// index(dgt, sites; base) — AbstractBasis.jl:318-331 (sites 1-based)
inline int64_t index_sites(const int64_t* dgt, const int* sites, int ns, int64_t base) {
  int64_t N = 0;
  if (base == 2) { for (int i = 0; i < ns; ++i) N = (N << 1) | dgt[sites[i] - 1]; }
  else { for (int i = 0; i < ns; ++i) { N *= base; N += dgt[sites[i] - 1]; } }
  return N + 1;
}
// change!(dgt, ind; base) — AbstractBasis.jl:348-360
inline void change_dgt(int64_t* dgt, int L, int64_t ind, int64_t base) {
  int64_t N = ind - 1;
  if (base == 2) { for (int i = L - 1; i >= 0; --i) { dgt[i] = N & 1; N >>= 1; } }
  else { for (int i = L - 1; i >= 0; --i) { dgt[i] = N % base; N /= base; } }
}
// change!(dgt, sites, ind; base) — AbstractBasis.jl:380-392
inline void change_sites(int64_t* dgt, const int* sites, int ns, int64_t ind, int64_t base) {
  int64_t N = ind - 1;
  if (base == 2) { for (int i = ns - 1; i >= 0; --i) { dgt[sites[i] - 1] = N & 1; N >>= 1; } }
  else { for (int i = ns - 1; i >= 0; --i) { dgt[sites[i] - 1] = N % base; N /= base; } }
}
// rindex(dgt; base) — TranslationalParityBasis.jl:40-42 (evalpoly = reversed digits)
inline int64_t rindex_dgt(const int64_t* dgt, int L, int64_t base) {
  int64_t N = 0;
  for (int i = L - 1; i >= 0; --i) { N *= base; N += dgt[i]; }
  return N + 1;
}
// circshift!(dgt, A): new[j] = old[j - A mod L] (Julia Base semantics)
inline void circshift(int64_t* dgt, int L, int A, int64_t* tmp) {
  for (int j = 0; j < L; ++j) tmp[j] = dgt[j];
  for (int j = 0; j < L; ++j) dgt[((j + A) % L + L) % L] = tmp[j];
}
// _int_translate — AbstractBasis.jl:405-408
inline int64_t int_translate(int64_t state, int64_t pow_shift, int64_t base_shift) {
  int64_t tail = state % base_shift;
  return tail * pow_shift + state / base_shift;
}
// _int_reverse — AbstractBasis.jl:417-425
inline int64_t int_reverse(int64_t state, int L, int64_t base) {
  int64_t r = 0, v = state;
  for (int i = 0; i < L; ++i) { r = r * base + v % base; v /= base; }
  return r;
}
// binary_search — ProjectedBasis.jl:71-81 (1-based result, 0 if absent)
inline int64_t binary_search(const std::vector<int64_t>& list, int64_t i) {
  int64_t n = (int64_t)list.size();
  if (n == 0) return 0;
  int64_t l = 1, r = n, c = (l + r) / 2;
  while (true) {
    int64_t t = list[c - 1];
    if (i < t) r = c - 1; else if (i > t) l = c + 1; else break;
    if (l > r) { c = 0; break; } else c = (l + r) / 2;
  }
  return c;
}

// _gosper_next — AbelianBasis.jl:456-464
inline uint64_t gosper_next(uint64_t s) {
  uint64_t c = s & (~s + 1);
  uint64_t r = s + c;
  uint64_t diff = r ^ s;
  diff = (diff >> 2) / c;
  return r | diff;
}

enum Kind { K_TENSOR = 0, K_PROJECTED = 1, K_TRANS = 2, K_TRANSPAR = 3, K_ABELIAN = 4 };

struct Gen {  // one cyclic factor of an AbelianOperator (AbelianBasis.jl:143-193)
  int order;
  std::vector<cplx> c;            // phase table
  std::vector<int> perm;          // 1-based site permutation
  std::vector<uint8_t> inv;       // inversion flags
  std::vector<std::pair<uint64_t, int>> layers;  // delta-swap network
  uint64_t inv_mask = 0;
};

struct OBasis {
  int kind = K_TENSOR;
  int L = 0;
  int64_t base = 2;
  int A = 1, len = 1;
  std::vector<int64_t> I;
  std::vector<double> R;
  std::vector<cplx> C;
  int P = 1, Kpar = 1;   // TranslationParity: parity, K = +-1
  std::vector<Gen> gens; // AbelianBasis
  int64_t order() const { int64_t o = 1; for (auto& g : gens) o *= g.order; return o; }
  int64_t dim() const {
    if (kind == K_TENSOR) return ipow(base, L);
    return (int64_t)I.size();
  }
};

// ---------------------------------------------------------------------------
// Benes / delta-swap compilation — AbelianBasis.jl:28-69, apply :80-87
// ---------------------------------------------------------------------------
std::vector<std::pair<uint64_t, int>> compile_benes(const std::vector<int>& perm, int L) {
  std::vector<int> bit_perm(L), current(L), where_is(L), inv_perm(L);
  for (int i = 1; i <= L; ++i) bit_perm[L - i] = L - perm[i - 1];
  for (int i = 0; i < L; ++i) { current[i] = i; where_is[i] = i; }
  for (int s = 0; s < L; ++s) inv_perm[bit_perm[s]] = s;
  std::vector<std::pair<int, int>> swaps;
  for (int dst = 0; dst < L; ++dst) {
    int src_bit = inv_perm[dst];
    int cur_pos = where_is[src_bit];
    if (cur_pos != dst) {
      swaps.push_back({std::min(dst, cur_pos), std::max(dst, cur_pos)});
      int other_bit = current[dst];
      std::swap(current[dst], current[cur_pos]);
      where_is[src_bit] = dst;
      where_is[other_bit] = cur_pos;
    }
  }
  std::vector<std::pair<uint64_t, int>> layers;
  for (auto& s : swaps) layers.push_back({uint64_t(1) << s.first, s.second - s.first});
  return layers;
}
inline uint64_t apply_benes(const std::vector<std::pair<uint64_t, int>>& layers, uint64_t state) {
  for (auto& l : layers) {
    uint64_t delta = ((state >> l.second) ^ state) & l.first;
    state = state ^ delta ^ (delta << l.second);
  }
  return state;
}
// phase(g) — AbelianBasis.jl:222-224: product over factors in order
inline cplx gen_phase(const OBasis& b, const std::vector<int>& s) {
  cplx p = b.gens[0].c[s[0] - 1];
  for (size_t i = 1; i < b.gens.size(); ++i) p = p * b.gens[i].c[s[i] - 1];
  return p;
}
// odometer step on an integer state — check_min_int/shift_canonical_int inner loop
inline uint64_t odometer_int(const OBasis& b, std::vector<int>& s, uint64_t cur) {
  for (size_t i = 0; i < b.gens.size(); ++i) {
    cur = apply_benes(b.gens[i].layers, cur) ^ b.gens[i].inv_mask;
    if (++s[i] > b.gens[i].order) s[i] = 1; else break;
  }
  return cur;
}
// odometer step on a digit buffer — _apply_group_action! AbelianBasis.jl:292-299
inline void odometer_dgt(const OBasis& b, std::vector<int>& s, int64_t* dgt, int64_t* tmp) {
  int L = b.L;
  for (size_t i = 0; i < b.gens.size(); ++i) {
    const Gen& g = b.gens[i];
    for (int j = 0; j < L; ++j) tmp[j] = dgt[j];
    for (int j = 0; j < L; ++j) dgt[g.perm[j] - 1] = tmp[j];
    bool anyinv = false;
    for (int j = 0; j < L; ++j) anyinv |= g.inv[j] != 0;
    if (anyinv) for (int j = 0; j < L; ++j) if (g.inv[j]) dgt[j] = b.base - 1 - dgt[j];
    if (++s[i] > g.order) s[i] = 1; else break;
  }
}
// check_min_int — AbelianBasis.jl:399-418
std::pair<bool, int> check_min_int(const OBasis& b, uint64_t s0) {
  std::vector<int> s(b.gens.size(), 1);
  uint64_t cur = s0;
  int N = 1;
  int64_t ord = b.order();
  for (int64_t t = 2; t <= ord; ++t) {
    cur = odometer_int(b, s, cur);
    if (cur < s0) return {false, 0};
    if (cur == s0) {
      if (!(std::abs(gen_phase(b, s) - 1.0) < 1e-14)) return {false, 0};
      N += 1;
    }
  }
  return {true, N};
}
// check_min (digit path) — AbelianBasis.jl:312-328
std::pair<bool, int> check_min_dgt(const OBasis& b, int64_t* dgt) {
  std::vector<int> s(b.gens.size(), 1);
  std::vector<int64_t> tmp(b.L);
  int64_t I0 = index_dgt(dgt, b.L, b.base);
  int N = 1;
  int64_t ord = b.order();
  for (int64_t t = 2; t <= ord; ++t) {
    odometer_dgt(b, s, dgt, tmp.data());
    int64_t In = index_dgt(dgt, b.L, b.base);
    if (In < I0) return {false, 0};
    if (In == I0) {
      if (!(std::abs(gen_phase(b, s) - 1.0) < 1e-14)) return {false, 0};
      N += 1;
    }
  }
  return {true, N};
}

// ---------------------------------------------------------------------------
// Basis construction
// ---------------------------------------------------------------------------
// Generic ordered scan over 1-based indices [1, base^L]: each thread scans a
// contiguous block and the blocks are concatenated in order, like
// selectindexnorm_threaded (TranslationalBasis.jl:194-204) and dividerange
// (ProjectedBasis.jl:105-121).  `judge(dgt, i, &norm) -> bool`.
template <class Judge>
void ordered_scan(int L, int64_t base, int64_t lo, int64_t hi, bool threaded, Judge judge,
                  std::vector<int64_t>& I, std::vector<double>& R) {
  int nt = threaded ? omp_get_max_threads() : 1;
  int64_t n = hi - lo + 1;
  if (n <= 0) return;
  std::vector<std::vector<int64_t>> nI(nt);
  std::vector<std::vector<double>> nR(nt);
#pragma omp parallel num_threads(nt)
  {
    int t = omp_get_thread_num();
    int64_t each = n / nt, left = n % nt;
    int64_t start = lo + t * each + std::min<int64_t>(t, left);
    int64_t stop = start + each + (t < left ? 1 : 0) - 1;
    std::vector<int64_t> dgt(L);
    for (int64_t i = start; i <= stop; ++i) {
      change_dgt(dgt.data(), L, i, base);
      double nrm = 1.0;
      if (judge(dgt.data(), i, nrm)) { nI[t].push_back(i); nR[t].push_back(nrm); }
    }
  }
  for (int t = 0; t < nt; ++t) {
    I.insert(I.end(), nI[t].begin(), nI[t].end());
    R.insert(R.end(), nR[t].begin(), nR[t].end());
  }
}

// ordered Gosper scan over the 0-based states with `nset` set bits (base 2)
template <class Judge>
void gosper_scan(int L, int nset, bool threaded, Judge judge, std::vector<int64_t>& I,
                 std::vector<double>& R) {
  // enumerate candidates first (cheap), then judge in parallel preserving order
  std::vector<int64_t> cand;
  if (nset == 0) cand.push_back(1);
  else if (nset == L) cand.push_back((int64_t)(uint64_t(1) << L));
  else if (nset > 0 && nset < L) {
    uint64_t s = (uint64_t(1) << nset) - 1, mx = uint64_t(1) << L;
    while (s < mx) { cand.push_back((int64_t)s + 1); s = gosper_next(s); }
  }
  int nt = threaded ? omp_get_max_threads() : 1;
  int64_t n = (int64_t)cand.size();
  std::vector<std::vector<int64_t>> nI(nt);
  std::vector<std::vector<double>> nR(nt);
#pragma omp parallel num_threads(nt)
  {
    int t = omp_get_thread_num();
    int64_t each = n / nt, left = n % nt;
    int64_t start = t * each + std::min<int64_t>(t, left);
    int64_t stop = start + each + (t < left ? 1 : 0);
    std::vector<int64_t> dgt(L);
    for (int64_t k = start; k < stop; ++k) {
      int64_t i = cand[k];
      change_dgt(dgt.data(), L, i, 2);
      double nrm = 1.0;
      if (judge(dgt.data(), i, nrm)) { nI[t].push_back(i); nR[t].push_back(nrm); }
    }
  }
  for (int t = 0; t < nt; ++t) {
    I.insert(I.end(), nI[t].begin(), nI[t].end());
    R.insert(R.end(), nR[t].begin(), nR[t].end());
  }
}

inline bool charge_ok(const int64_t* dgt, int L, int64_t base, int N) {
  if (N < 0) return true;
  int64_t num = (int64_t)L * (base - 1) - N, s = 0;
  for (int i = 0; i < L; ++i) s += dgt[i];
  return s == num;
}

}  // namespace

// ===========================================================================
// C ABI for ctypes (oracle only)
// ===========================================================================
extern "C" {

typedef struct OBasis orc_basis;

const char* orc_last_error(void) { return g_err.c_str(); }

int orc_num_threads(void) { return omp_get_max_threads(); }
void orc_set_threads(int n) { if (n > 0) omp_set_num_threads(n); }

// TensorBasis(; L, base) — AbstractBasis.jl:234-238
orc_basis* orc_tensor(int L, int base) {
  auto* b = new OBasis; b->kind = K_TENSOR; b->L = L; b->base = base; return b;
}

// ProjectedBasis(; L, f, N, base, threaded, small_N) — ProjectedBasis.jl:244-260.
// N < 0 means `nothing`.  `gosper` selects the fixed-popcount enumeration for
// base 2 (same ordered output as the full scan: both list the states that pass
// the same filter in ascending order).
orc_basis* orc_projected(int L, int base, int N, orc_pred f, void* ud, int threaded, int gosper) {
  auto* b = new OBasis; b->kind = K_PROJECTED; b->L = L; b->base = base;
  auto judge = [&](const int64_t* dgt, int64_t, double& nrm) {
    nrm = 1.0;
    if (!charge_ok(dgt, L, base, N)) return false;
    if (f && !f(dgt, L, ud)) return false;
    return true;
  };
  if (gosper && base == 2 && N >= 0 && N <= L)
    gosper_scan(L, L - N, threaded && !f, judge, b->I, b->R);
  else
    ordered_scan(L, base, 1, ipow(base, L), threaded && !f, judge, b->I, b->R);
  b->R.clear();
  return b;
}

// TranslationalBasis(; L, f, k, N, a, base) — TranslationalBasis.jl:235-266,
// judge :94-114, phase_factor :277-285.
orc_basis* orc_translational(int L, int base, int k, int N, int a, orc_pred f, void* ud,
                             int threaded, int gosper) {
  if (a <= 0 || L % a != 0) { g_err = "Length of unit-cell incompatible with L"; return nullptr; }
  auto* b = new OBasis; b->kind = K_TRANS; b->L = L; b->base = base; b->A = a;
  int len = L / a; b->len = len;
  int K = ((-k) % len + len) % len;  // k = mod(-k, len)
  std::vector<double> norm(len);
  for (int i = 1; i <= len; ++i) norm[i - 1] = (double)len / std::sqrt((double)i);
  auto judge = [&](const int64_t* d0, int64_t i, double& nrm) {
    if (!charge_ok(d0, L, base, N)) return false;
    if (f && !f(d0, L, ud)) return false;
    std::vector<int64_t> dgt(d0, d0 + L), tmp(L);
    for (int n = 1; n <= len - 1; ++n) {
      circshift(dgt.data(), L, a, tmp.data());
      int64_t In = index_dgt(dgt.data(), L, base);
      if (In < i) return false;
      if (In == i) {
        if (((int64_t)n * K) % len != 0) return false;  // check_momentum :80
        nrm = norm[n - 1];
        return true;
      }
    }
    nrm = norm[len - 1];
    return true;
  };
  if (gosper && base == 2 && N >= 0 && N <= L)
    gosper_scan(L, L - N, threaded && !f, judge, b->I, b->R);
  else
    ordered_scan(L, base, 1, ipow(base, L), threaded && !f, judge, b->I, b->R);
  // phase_factor(k, len)
  b->C.resize(len);
  const double twopi = 2.0 * M_PI;
  for (int i = 0; i < len; ++i) {
    if (K == 0) b->C[i] = 1.0;
    else if (2 * K == len) b->C[i] = (i % 2 == 0) ? 1.0 : -1.0;
    else {
      // exp(-1im * 2π/len * k*i): angle = (((-2π)/len)*k)*i
      double th = ((-twopi / (double)len) * (double)K) * (double)i;
      if (i == 0) b->C[i] = cplx(1.0, th);
      else b->C[i] = cplx(std::cos(th), std::sin(th));
    }
  }
  return b;
}

// The TranslationalBasis of given tables (I 1-based ascending, R), with the
// phase table of TranslationalBasis.jl:264 / 277-285: for sectors too large to
// scan here, whose tables the tests check by sampling (orc_trans_judge).
orc_basis* orc_translational_tables(int L, int base, int k, int a, int64_t D, const int64_t* I,
                                    const double* R) {
  if (a <= 0 || L % a != 0) { g_err = "Length of unit-cell incompatible with L"; return nullptr; }
  auto* b = new OBasis; b->kind = K_TRANS; b->L = L; b->base = base; b->A = a;
  int len = L / a; b->len = len;
  int K = ((-k) % len + len) % len;
  b->I.assign(I, I + D);
  b->R.assign(R, R + D);
  b->C.resize(len);
  const double twopi = 2.0 * M_PI;
  for (int i = 0; i < len; ++i) {
    if (K == 0) b->C[i] = 1.0;
    else if (2 * K == len) b->C[i] = (i % 2 == 0) ? 1.0 : -1.0;
    else {
      double th = ((-twopi / (double)len) * (double)K) * (double)i;
      if (i == 0) b->C[i] = cplx(1.0, th);
      else b->C[i] = cplx(std::cos(th), std::sin(th));
    }
  }
  return b;
}

// The TranslationalBasis judge (TranslationalBasis.jl:94-114, norms :251-255)
// on explicit 1-based indices: accept[q] = 1 and R[q] = the norm when index
// idx[q] is an orbit representative of the sector (charge N, momentum k),
// else accept[q] = 0.  The same judge as orc_translational's scan.
void orc_trans_judge(int L, int base, int k, int N, int a, int64_t n, const int64_t* idx,
                     uint8_t* accept, double* R) {
  int len = L / a;
  int K = ((-k) % len + len) % len;
  std::vector<double> norm(len);
  for (int i = 1; i <= len; ++i) norm[i - 1] = (double)len / std::sqrt((double)i);
#pragma omp parallel
  {
    std::vector<int64_t> dgt(L), tmp(L);
#pragma omp for schedule(static)
    for (int64_t q = 0; q < n; ++q) {
      const int64_t i = idx[q];
      change_dgt(dgt.data(), L, i, base);
      accept[q] = 0;
      R[q] = 0.0;
      if (!charge_ok(dgt.data(), L, base, N)) continue;
      double nrm = norm[len - 1];
      bool ok = true;
      for (int m = 1; m <= len - 1; ++m) {
        circshift(dgt.data(), L, a, tmp.data());
        int64_t In = index_dgt(dgt.data(), L, base);
        if (In < i) { ok = false; break; }
        if (In == i) {
          if (((int64_t)m * K) % len != 0) ok = false;
          else nrm = norm[m - 1];
          break;
        }
      }
      if (ok) { accept[q] = 1; R[q] = nrm; }
    }
  }
}

// TranslationParityBasis(; L, f, k, p, N, a, base) — TranslationalParityBasis.jl:141-175,
// judge :68-112.
orc_basis* orc_transparity(int L, int base, int k, int p, int N, int a, orc_pred f, void* ud,
                           int threaded, int gosper) {
  if (a <= 0 || L % a != 0) { g_err = "Length of unit-cell incompatible with L"; return nullptr; }
  int len = L / a;
  int K;
  if (((k % len) + len) % len == 0) K = 1;
  else if ((((2 * k) % len) + len) % len == 0) K = -1;
  else { g_err = "Momentum " + std::to_string(k) + " incompatible with parity."; return nullptr; }
  if (!(p == 1 || p == -1)) { g_err = "Invalid parity"; return nullptr; }
  auto* b = new OBasis; b->kind = K_TRANSPAR; b->L = L; b->base = base; b->A = a; b->len = len;
  b->P = p; b->Kpar = K;
  std::vector<double> Cn(2 * len);
  for (int i = 1; i <= len; ++i) {
    double n2 = (double)(2 * len) / std::sqrt((double)i);
    Cn[len + i - 1] = n2;
    Cn[i - 1] = n2 / std::sqrt(2.0);
  }
  auto judge = [&](const int64_t* d0, int64_t i, double& nrm) {
    if (!charge_ok(d0, L, base, N)) return false;
    if (f && !f(d0, L, ud)) return false;
    std::vector<int64_t> dgt(d0, d0 + L), tmp(L);
    int Rr = len;
    bool Qp = false;
    int64_t In = rindex_dgt(dgt.data(), L, base);
    if (In < i) return false;
    if (In == i) { Qp = true; if (p != 1) return false; }
    for (int n = 1; n <= len - 1; ++n) {
      circshift(dgt.data(), L, a, tmp.data());
      int64_t In1 = index_dgt(dgt.data(), L, base);
      int64_t In2 = rindex_dgt(dgt.data(), L, base);
      if (In1 < i) return false;
      if (In2 < i) return false;
      if (In2 == i) {
        int Kn = (K == 1 || n % 2 == 0) ? 1 : -1;
        if (p * Kn != 1) return false;
        Qp = true;
      }
      if (In1 == i) {
        if (!(K == 1 || n % 2 == 0)) return false;
        Rr = n;
        break;
      }
    }
    nrm = Qp ? Cn[len + Rr - 1] : Cn[Rr - 1];
    return true;
  };
  if (gosper && base == 2 && N >= 0 && N <= L)
    gosper_scan(L, L - N, threaded && !f, judge, b->I, b->R);
  else
    ordered_scan(L, base, 1, ipow(base, L), threaded && !f, judge, b->I, b->R);
  b->C.resize(len);
  for (int i = 0; i < len; ++i) b->C[i] = (K == 1) ? 1.0 : ((i % 2 == 0) ? 1.0 : -1.0);
  return b;
}

// AbelianBasis via basis(...) — AbelianBasis.jl:516-555 (ctor), :771-847 (basis).
// Generators are passed already assembled (order, quantum number, 1-based perm,
// inversion flags), in the order `basis` pushes them: translation, parity,
// flip, then custom symmetries.  N < 0 means `nothing` (N here counts SET bits
// on the Gosper path, exactly as the reference's Gosper branch does).
orc_basis* orc_abelian(int L, int base, int N, int ngen, const int* orders, const int* ks,
                       const int* perms, const uint8_t* invs, orc_pred f, void* ud,
                       int threaded) {
  auto* b = new OBasis; b->kind = K_ABELIAN; b->L = L; b->base = base;
  const double twopi = 2.0 * M_PI;
  for (int gi = 0; gi < ngen; ++gi) {
    Gen g;
    g.order = orders[gi];
    int k = ks[gi];
    g.c.resize(g.order);
    for (int j = 0; j < g.order; ++j) {
      if (k == 0) g.c[j] = 1.0;
      else if (2 * k == g.order) g.c[j] = (j % 2 == 0) ? 1.0 : -1.0;
      else {
        // phase = 1im * 2π * k / order; exp(phase * j)
        double ph = (twopi * (double)k) / (double)g.order;
        double th = ph * (double)j;
        if (j == 0) g.c[j] = cplx(1.0, th);
        else g.c[j] = cplx(std::cos(th), std::sin(th));
      }
    }
    g.perm.assign(perms + (size_t)gi * L, perms + (size_t)(gi + 1) * L);
    g.inv.assign(invs + (size_t)gi * L, invs + (size_t)(gi + 1) * L);
    g.layers = compile_benes(g.perm, L);
    for (int i = 1; i <= L; ++i) if (g.inv[i - 1]) g.inv_mask |= uint64_t(1) << (L - i);
    b->gens.push_back(g);
  }
  int64_t Ng = b->order();
  std::vector<double> C(Ng, 0.0);
  for (int64_t i = 1; i <= Ng; ++i) if (Ng % i == 0) C[i - 1] = std::sqrt((double)(Ng * i));
  bool use_gosper = (base == 2 && N >= 0 && N <= L);
  if (use_gosper) {
    // Path 1: Gosper candidates (N set bits) + integer orbit search; f ignored.
    auto judge = [&](const int64_t*, int64_t i, double& nrm) {
      auto q = check_min_int(*b, (uint64_t)(i - 1));
      if (!q.first) return false;
      nrm = C[q.second - 1];
      return true;
    };
    gosper_scan(L, N, threaded != 0, judge, b->I, b->R);
  } else {
    int64_t num = (N >= 0) ? (int64_t)L * (base - 1) - N : -1;
    auto judge = [&](const int64_t* d0, int64_t, double& nrm) {
      if (num >= 0) { int64_t s = 0; for (int j = 0; j < L; ++j) s += d0[j]; if (s != num) return false; }
      if (f && !f(d0, L, ud)) return false;
      std::vector<int64_t> dgt(d0, d0 + L);
      auto q = check_min_dgt(*b, dgt.data());
      if (!q.first) return false;
      nrm = C[q.second - 1];
      return true;
    };
    ordered_scan(L, base, 1, ipow(base, L), threaded && !f, judge, b->I, b->R);
  }
  return b;
}

void orc_free(orc_basis* b) { delete b; }
int64_t orc_dim(const orc_basis* b) { return b->dim(); }
int orc_kind(const orc_basis* b) { return b->kind; }
int orc_len(const orc_basis* b) { return b->len; }
// copy tables out: I (1-based) and R (norms; left untouched for onsite bases)
void orc_export(const orc_basis* b, int64_t* I, double* R) {
  if (I) for (size_t i = 0; i < b->I.size(); ++i) I[i] = b->I[i];
  if (R) for (size_t i = 0; i < b->R.size(); ++i) R[i] = b->R[i];
}
// phase table C as interleaved complex (length len)
void orc_phase(const orc_basis* b, double* C) {
  for (size_t i = 0; i < b->C.size(); ++i) { C[2 * i] = b->C[i].real(); C[2 * i + 1] = b->C[i].imag(); }
}

}  // extern "C"

// ---------------------------------------------------------------------------
// index(b, dgt) for every basis kind
// ---------------------------------------------------------------------------
namespace {
// returns (coeff, pos) with pos 1-based; absent -> (0, 1)
std::pair<cplx, int64_t> basis_index(const OBasis& b, const int64_t* dgt) {
  int L = b.L;
  int64_t base = b.base;
  switch (b.kind) {
    case K_TENSOR:  // AbstractBasis.jl:246
      return {1.0, index_dgt(dgt, L, base)};
    case K_PROJECTED: {  // ProjectedBasis.jl:52-57
      int64_t i = index_dgt(dgt, L, base);
      int64_t ind = binary_search(b.I, i);
      if (ind > 0) return {1.0, ind};
      return {0.0, 1};
    }
    case K_TRANS: {  // TranslationalBasis.jl:310-341
      int64_t I0 = index_dgt(dgt, L, base);
      int64_t state = I0 - 1;
      int64_t Im = I0; int M = 0;
      int A = b.A;
      if (base == 2) {
        int64_t mask = (int64_t)((uint64_t(1) << L) - 1);
        for (int i = 1; i <= b.len - 1; ++i) {
          state = (int64_t)((((uint64_t)state >> A) | ((uint64_t)state << (L - A))) & (uint64_t)mask);
          int64_t In = state + 1;
          if (In == I0) break;
          if (In < Im) { Im = In; M = i; }
        }
      } else {
        int64_t pow_shift = ipow(base, L - A), base_shift = ipow(base, A);
        for (int i = 1; i <= b.len - 1; ++i) {
          state = int_translate(state, pow_shift, base_shift);
          int64_t In = state + 1;
          if (In == I0) break;
          if (In < Im) { Im = In; M = i; }
        }
      }
      int64_t i = binary_search(b.I, Im);
      if (i == 0) return {0.0, 1};
      return {b.C[M] * b.R[i - 1], i};
    }
    case K_TRANSPAR: {  // TranslationalParityBasis.jl:192-234
      int64_t Ia0 = index_dgt(dgt, L, base);
      int64_t state = Ia0 - 1;
      int A = b.A;
      int64_t Ib0 = int_reverse(state, L, base) + 1;
      int64_t Iam = Ia0, Ibm = Ib0;
      int Rr = 0, M = 0;
      int64_t pow_shift = ipow(base, L - A), base_shift = ipow(base, A);
      uint64_t mask = (uint64_t(1) << L) - 1;
      for (int i = 1; i <= b.len - 1; ++i) {
        if (base == 2) state = (int64_t)((((uint64_t)state >> A) | ((uint64_t)state << (L - A))) & mask);
        else state = int_translate(state, pow_shift, base_shift);
        int64_t Ia1 = state + 1;
        if (Ia1 == Ia0) break;
        else if (Ia1 < Iam) { Iam = Ia1; Rr = i; }
        int64_t Ib1 = int_reverse(state, L, base) + 1;
        if (Ib1 < Ibm) { Ibm = Ib1; M = i; }
      }
      int64_t i; double n;
      if (Ibm < Iam) { i = binary_search(b.I, Ibm); n = (double)b.P * b.C[M].real(); }
      else { i = binary_search(b.I, Iam); n = b.C[Rr].real(); }
      if (i == 0) return {0.0, 1};
      return {n * b.R[i - 1], i};
    }
    case K_ABELIAN: {  // AbelianBasis.jl:669-693
      std::vector<int> ms(b.gens.size(), 1), s(b.gens.size(), 1);
      int64_t Im;
      if (base == 2) {  // shift_canonical_int :428-445
        uint64_t state = 0;
        for (int i = 0; i < L; ++i) state = (state << 1) | (uint64_t)dgt[i];
        uint64_t best = state, cur = state;
        int64_t ord = b.order();
        for (int64_t t = 0; t < ord; ++t) {
          cur = odometer_int(b, s, cur);
          if (cur < best) { best = cur; ms = s; }
        }
        Im = (int64_t)best + 1;
      } else {  // shift_canonical! :346-362
        std::vector<int64_t> d(dgt, dgt + L), tmp(L);
        Im = index_dgt(d.data(), L, base);
        int64_t ord = b.order();
        for (int64_t t = 0; t < ord; ++t) {
          odometer_dgt(b, s, d.data(), tmp.data());
          int64_t In = index_dgt(d.data(), L, base);
          if (In < Im) { Im = In; ms = s; }
        }
      }
      int64_t ind = binary_search(b.I, Im);
      if (ind == 0) return {0.0, 1};
      return {gen_phase(b, ms) * b.R[ind - 1], ind};
    }
  }
  return {0.0, 1};
}

inline double basis_norm(const OBasis& b, int64_t j) {
  if (b.kind == K_TENSOR || b.kind == K_PROJECTED) return 1.0;
  return b.R[j - 1];
}
inline int64_t basis_content(const OBasis& b, int64_t j) {
  return b.kind == K_TENSOR ? j : b.I[j - 1];
}

struct OTerm {
  std::vector<int> sites;             // 1-based
  std::vector<int64_t> colptr;        // 1-based CSC
  std::vector<int64_t> rowval;        // 1-based
  std::vector<cplx> nzval;
};
struct OOperator {
  const OBasis* b;
  std::vector<OTerm> terms;
};

// colmn!(target, opt, j, dgt, coeff) — Operator.jl:458-465 with the per-term
// colmn! :426-439 and _accumulate! :399-407.  `target` is column-major D x nvec,
// coeff holds nvec values (row j of the input block).
void colmn(cplx* target, int64_t D, int64_t nvec, const OOperator& op, int64_t j, int64_t* dgt,
           const cplx* coeff_in, cplx* coeff) {
  const OBasis& b = *op.b;
  change_dgt(dgt, b.L, basis_content(b, j), b.base);
  double r = basis_norm(b, j);
  for (int64_t k = 0; k < nvec; ++k) coeff[k] = (r == 1.0) ? coeff_in[k] : coeff_in[k] / r;
  for (const OTerm& t : op.terms) {
    int ns = (int)t.sites.size();
    int64_t jl = index_sites(dgt, t.sites.data(), ns, b.base);
    bool change = false;
    for (int64_t q = t.colptr[jl - 1]; q < t.colptr[jl]; ++q) {
      int64_t row = t.rowval[q - 1];
      cplx val = t.nzval[q - 1];
      change_sites(dgt, t.sites.data(), ns, row, b.base);
      auto ci = basis_index(b, dgt);
      if (nvec == 1) {
        target[ci.second - 1] += coeff[0] * ci.first * val;
      } else {
        cplx cv = ci.first * val;
        for (int64_t k = 0; k < nvec; ++k) target[(ci.second - 1) + k * D] += cv * coeff[k];
      }
      change = true;
    }
    if (change) change_sites(dgt, t.sites.data(), ns, jl, b.base);
  }
}
}  // namespace

extern "C" {
typedef struct OOperator orc_operator;

// index(b, dgt) for testing: coefficient (re, im) and 1-based position
void orc_index(const orc_basis* b, const int64_t* dgt, double* cre, double* cim, int64_t* pos) {
  auto r = basis_index(*b, dgt);
  *cre = r.first.real(); *cim = r.first.imag(); *pos = r.second;
}

// operator(mats, inds, B) after the caller has merged repeated site lists
// (Operator.jl:56-78).  Terms are concatenated: nsites[t], sites (1-based),
// colptr (1-based, size dim+1 each), rowval (1-based), nzval complex interleaved.
orc_operator* orc_operator_create(const orc_basis* b, int nterms, const int* nsites,
                                  const int* sites, const int64_t* nnz_per_term,
                                  const int64_t* colptr, const int64_t* rowval,
                                  const double* nzval) {
  auto* op = new OOperator; op->b = b;
  size_t so = 0, co = 0, no = 0;
  for (int t = 0; t < nterms; ++t) {
    OTerm term;
    int ns = nsites[t];
    term.sites.assign(sites + so, sites + so + ns); so += ns;
    int64_t dim = ipow(b->base, ns);
    term.colptr.assign(colptr + co, colptr + co + dim + 1); co += dim + 1;
    int64_t nz = nnz_per_term[t];
    term.rowval.assign(rowval + no, rowval + no + nz);
    term.nzval.resize(nz);
    for (int64_t q = 0; q < nz; ++q) term.nzval[q] = cplx(nzval[2 * (no + q)], nzval[2 * (no + q) + 1]);
    no += nz;
    op->terms.push_back(std::move(term));
  }
  return op;
}
void orc_operator_free(orc_operator* op) { delete op; }

// mul!(target, opt, m) / opt * m (single thread, accumulating) — Operator.jl:309-328
void orc_mul_serial(const orc_operator* op, const double* x, double* y, int64_t nvec) {
  const OBasis& b = *op->b;
  int64_t D = b.dim();
  std::vector<int64_t> dgt(b.L);
  std::vector<cplx> cin(nvec), cw(nvec);
  const cplx* X = reinterpret_cast<const cplx*>(x);
  cplx* Y = reinterpret_cast<cplx*>(y);
  for (int64_t j = 1; j <= D; ++j) {
    for (int64_t k = 0; k < nvec; ++k) cin[k] = X[(j - 1) + k * D];
    colmn(Y, D, nvec, *op, j, dgt.data(), cin.data(), cw.data());
  }
}

// mul(opt, v) / mul(opt, m) — Operator.jl:340-370: dividerange over input rows,
// one private full-length output per thread, summed at the end.  y is
// overwritten (mul allocates its result).
void orc_mul(const orc_operator* op, const double* x, double* y, int64_t nvec, int nthreads) {
  const OBasis& b = *op->b;
  int64_t D = b.dim();
  int nt = nthreads > 0 ? nthreads : omp_get_max_threads();
  const cplx* X = reinterpret_cast<const cplx*>(x);
  cplx* Y = reinterpret_cast<cplx*>(y);
  std::vector<std::vector<cplx>> Ms(nt);
#pragma omp parallel num_threads(nt)
  {
    int t = omp_get_thread_num();
    Ms[t].assign((size_t)D * nvec, cplx(0.0, 0.0));
    int64_t each = D / nt, left = D % nt;
    int64_t start = 1 + t * each + std::min<int64_t>(t, left);
    int64_t stop = start + each + (t < left ? 1 : 0) - 1;
    std::vector<int64_t> dgt(b.L);
    std::vector<cplx> cin(nvec), cw(nvec);
    for (int64_t j = start; j <= stop; ++j) {
      for (int64_t k = 0; k < nvec; ++k) cin[k] = X[(j - 1) + k * D];
      colmn(Ms[t].data(), D, nvec, *op, j, dgt.data(), cin.data(), cw.data());
    }
  }
  int64_t tot = D * nvec;
#pragma omp parallel for num_threads(nt) schedule(static)
  for (int64_t i = 0; i < tot; ++i) {
    cplx s = Ms[0][i];
    for (int t = 1; t < nt; ++t) s += Ms[t][i];
    Y[i] = s;
  }
}

// mul(opt, v) restricted to the input columns j0..j1 (1-based, inclusive):
// the same thread-private scatter as orc_mul, for bounded timing samples.
// y (D x nvec) is overwritten with the partial product.
void orc_mul_cols(const orc_operator* op, const double* x, double* y, int64_t nvec, int64_t j0,
                  int64_t j1, int nthreads) {
  const OBasis& b = *op->b;
  int64_t D = b.dim();
  int nt = nthreads > 0 ? nthreads : omp_get_max_threads();
  const cplx* X = reinterpret_cast<const cplx*>(x);
  cplx* Y = reinterpret_cast<cplx*>(y);
  std::vector<std::vector<cplx>> Ms(nt);
  int64_t n = j1 - j0 + 1;
#pragma omp parallel num_threads(nt)
  {
    int t = omp_get_thread_num();
    Ms[t].assign((size_t)D * nvec, cplx(0.0, 0.0));
    int64_t each = n / nt, left = n % nt;
    int64_t start = j0 + t * each + std::min<int64_t>(t, left);
    int64_t stop = start + each + (t < left ? 1 : 0) - 1;
    std::vector<int64_t> dgt(b.L);
    std::vector<cplx> cin(nvec), cw(nvec);
    for (int64_t j = start; j <= stop; ++j) {
      for (int64_t k = 0; k < nvec; ++k) cin[k] = X[(j - 1) + k * D];
      colmn(Ms[t].data(), D, nvec, *op, j, dgt.data(), cin.data(), cw.data());
    }
  }
  int64_t tot = D * nvec;
#pragma omp parallel for num_threads(nt) schedule(static)
  for (int64_t i = 0; i < tot; ++i) {
    cplx s = Ms[0][i];
    for (int t = 1; t < nt; ++t) s += Ms[t][i];
    Y[i] = s;
  }
}

// Rows of H*x through columns: y[q] = sum_t conj(H[t, j]) x[t] for j = rows[q]
// (1-based), the entries H[:, j] being exactly those colmn! scatters for
// column j (Operator.jl:426-465: H[pos, j] = coefficient(index) * M[r, c] /
// R[j]).  For a Hermitian operator this is row j of H*x; the tests use it to
// check sampled rows of products whose full oracle mul would take too long.
// x and y complex interleaved.
void orc_rows_hermitian(const orc_operator* op, int64_t n, const int64_t* rows, const double* x,
                        double* y) {
  const OBasis& b = *op->b;
  const cplx* X = reinterpret_cast<const cplx*>(x);
  cplx* Y = reinterpret_cast<cplx*>(y);
#pragma omp parallel
  {
    std::vector<int64_t> dgt(b.L);
#pragma omp for schedule(dynamic, 16)
    for (int64_t q = 0; q < n; ++q) {
      const int64_t j = rows[q];
      change_dgt(dgt.data(), b.L, basis_content(b, j), b.base);
      const double r = basis_norm(b, j);
      cplx acc(0.0, 0.0);
      for (const OTerm& t : op->terms) {
        int ns = (int)t.sites.size();
        int64_t jl = index_sites(dgt.data(), t.sites.data(), ns, b.base);
        bool change = false;
        for (int64_t k = t.colptr[jl - 1]; k < t.colptr[jl]; ++k) {
          change_sites(dgt.data(), t.sites.data(), ns, t.rowval[k - 1], b.base);
          auto ci = basis_index(b, dgt.data());
          if (ci.first != 0.0) acc += std::conj(ci.first * t.nzval[k - 1] / r) * X[ci.second - 1];
          change = true;
        }
        if (change) change_sites(dgt.data(), t.sites.data(), ns, jl, b.base);
      }
      Y[q] = acc;
    }
  }
}

// The nonzeros colmn! scatters, as coordinate triplets (duplicates not
// summed): entry (pos, j, H[pos, j]) with H[pos, j] = coefficient(index) *
// M[r, c] / R[j] for every column j (Operator.jl:426-465), pos and j 1-based.
// With rows == nullptr only the count is returned.
int64_t orc_coo(const orc_operator* op, int64_t* rows, int64_t* cols, double* vals) {
  const OBasis& b = *op->b;
  const int64_t D = b.dim();
  std::vector<int64_t> dgt(b.L);
  int64_t n = 0;
  for (int64_t j = 1; j <= D; ++j) {
    change_dgt(dgt.data(), b.L, basis_content(b, j), b.base);
    const double r = basis_norm(b, j);
    for (const OTerm& t : op->terms) {
      int ns = (int)t.sites.size();
      int64_t jl = index_sites(dgt.data(), t.sites.data(), ns, b.base);
      bool change = false;
      for (int64_t k = t.colptr[jl - 1]; k < t.colptr[jl]; ++k) {
        change_sites(dgt.data(), t.sites.data(), ns, t.rowval[k - 1], b.base);
        auto ci = basis_index(b, dgt.data());
        if (ci.first != 0.0) {
          if (rows) {
            const cplx h = ci.first * t.nzval[k - 1] / r;
            rows[n] = ci.second;
            cols[n] = j;
            vals[2 * n] = h.real();
            vals[2 * n + 1] = h.imag();
          }
          ++n;
        }
        change = true;
      }
      if (change) change_sites(dgt.data(), t.sites.data(), ns, jl, b.base);
    }
  }
  return n;
}

// Array(opt) — Operator.jl:171-196: dense column-major D x D complex matrix
void orc_dense(const orc_operator* op, double* M) {
  const OBasis& b = *op->b;
  int64_t D = b.dim();
  cplx* out = reinterpret_cast<cplx*>(M);
  std::memset(M, 0, sizeof(double) * 2 * D * D);
#pragma omp parallel
  {
    std::vector<int64_t> dgt(b.L);
    cplx one(1.0, 0.0), cw;
#pragma omp for schedule(dynamic, 64)
    for (int64_t j = 1; j <= D; ++j) colmn(out + (j - 1) * D, D, 1, *op, j, dgt.data(), &one, &cw);
  }
}

// Gosper helpers exposed for the known-answer tests (AbelianBasis.jl:456-485)
uint64_t orc_gosper_next(uint64_t s) { return gosper_next(s); }
// apply_benes on a compiled permutation (AbelianBasis.jl:28-87)
uint64_t orc_apply_perm_benes(const int* perm, int L, uint64_t state) {
  std::vector<int> p(perm, perm + L);
  return apply_benes(compile_benes(p, L), state);
}
}  // extern "C"
