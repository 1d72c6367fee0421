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
#include <type_traits>

#include "edk_spmm.cuh"

namespace edk {

// y(:, k) (+)= H x(:, k); blockIdx.y = k.
template <int BK, class S, class VT, bool GATHER>
__global__ void __launch_bounds__(256) k_apply(BasisDev b, OpDev op, const VT* __restrict__ x,
                                               VT* __restrict__ y, int64_t ldx, int64_t ldy,
                                               int accumulate) {
  __shared__ uint32_t s_binom[32 * 33];
  if constexpr (BK == BK_PROJ_RANK) {
    fill_binom32(s_binom);
    __syncthreads();
  }
  const VT* xk = x + (int64_t)blockIdx.y * ldx;
  VT* yk = y + (int64_t)blockIdx.y * ldy;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < b.D;
       i += (int64_t)gridDim.x * blockDim.x)
    gen_row<BK, S, VT, GATHER>(b, op, i, xk, yk, accumulate, s_binom);
}

// Resident blocks per SM asked of the compiler: the rank-search kernels are
// latency bound and fit 32 registers (8 blocks of 256 threads fill every warp
// slot) for real and single-precision complex vectors, or single precision
// when the sector has a phase or a parity; the others keep the compiler's
// choice.
template <int BK, class VT>
constexpr int ff_min_blocks() {
  constexpr bool single = std::is_same<VT, float>::value || std::is_same<VT, float2>::value;
  return (BK == BK_TRANS0_RANK && !std::is_same<VT, double2>::value) ||
                 ((BK == BK_TRANS_RANK || BK == BK_TRANSPAR_RANK) && single)
             ? 8 : 1;
}

template <int BK, class VT, int TPS>
__global__ void __launch_bounds__(256, ff_min_blocks<BK, VT>())
    k_apply_ff(BasisDev b, OpDev op, FFParams ff,
                                                  const VT* __restrict__ x, VT* __restrict__ y,
                                                  int64_t ldx, int64_t ldy, int accumulate,
                                                  int64_t tile0) {
  ff_tile<BK, VT, TPS>(b, op, ff, (tile0 + blockIdx.x) * (256 / TPS),
                       x + (int64_t)blockIdx.y * ldx, y + (int64_t)blockIdx.y * ldy, accumulate);
}

namespace {

int apply_grid(int64_t D) {
  int64_t g = (D + 255) / 256;
  if (g < 1) g = 1;
  if (g > 148 * 64) g = 148 * 64;
  return (int)g;
}

template <class VT, int TPS>
edk_status launch_apply_ff(const BasisDev& b, const OpDev& op, const FFParams& ff, const void* x,
                           void* y, int64_t nvec, int64_t ldx, int64_t ldy, int accumulate,
                           cudaStream_t st, int64_t row0 = 0, int64_t row1 = -1) {
  const VT* X = static_cast<const VT*>(x);
  VT* Y = static_cast<VT*>(y);
  constexpr int RT = 256 / TPS;
  if (row1 < 0) row1 = b.D;
  const int64_t tile0 = row0 / RT, tile1 = (row1 + RT - 1) / RT;
  if (tile1 <= tile0) return EDK_OK;
  for (int64_t k0 = 0; k0 < nvec; k0 += 65535) {
    int64_t nk = std::min<int64_t>(nvec - k0, 65535);
    dim3 grid((unsigned)(tile1 - tile0), (unsigned)nk);
    const VT* Xk = X + k0 * ldx;
    VT* Yk = Y + k0 * ldy;
#define EDK_FF(BK)                                                                         \
  case BK:                                                                                 \
    k_apply_ff<BK, VT, TPS><<<grid, 256, 0, st>>>(b, op, ff, Xk, Yk, ldx, ldy, accumulate, \
                                                  tile0);                                     \
    break;
    const int kind = b.search != 2 ? b.bk
                     : (b.bk == BK_TRANS0 ? (int)BK_TRANS0_RANK
                        : (b.bk == BK_TRANS ? (int)BK_TRANS_RANK
                           : (b.bk == BK_TRANSPAR ? (int)BK_TRANSPAR_RANK : b.bk)));
    switch (kind) {
      EDK_FF(BK_TENSOR)
      EDK_FF(BK_PROJ_RANK)
      EDK_FF(BK_PROJ_HASH)
      EDK_FF(BK_TRANS0)
      EDK_FF(BK_TRANS0_RANK)
      EDK_FF(BK_TRANS_RANK)
      EDK_FF(BK_TRANSPAR_RANK)
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

namespace {

// column-major (ld) <-> row-major (p) blocks through 32 x 32 shared-memory
// tiles, coalesced on both sides; the reverse direction can accumulate
template <class VT>
__global__ void k_cols_to_rows_t(const VT* __restrict__ src, int64_t ld, int64_t D, int p,
                                 VT* __restrict__ dst) {
  __shared__ VT tile[32][33];
  const int64_t i0 = (int64_t)blockIdx.x * 32;
  const int c0 = blockIdx.y * 32;
  for (int k = threadIdx.y; k < 32; k += 8) {
    const int64_t i = i0 + threadIdx.x;
    const int c = c0 + k;
    if (i < D && c < p) tile[k][threadIdx.x] = src[(int64_t)c * ld + i];
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += 8) {
    const int64_t i = i0 + k;
    const int c = c0 + threadIdx.x;
    if (i < D && c < p) dst[i * p + c] = tile[threadIdx.x][k];
  }
}

template <class VT>
__global__ void k_rows_to_cols_t(const VT* __restrict__ src, int64_t D, int p,
                                 VT* __restrict__ dst, int64_t ld, int accumulate) {
  using A = typename VTraits<VT>::A;
  __shared__ VT tile[32][33];
  const int64_t i0 = (int64_t)blockIdx.x * 32;
  const int c0 = blockIdx.y * 32;
  for (int k = threadIdx.y; k < 32; k += 8) {
    const int64_t i = i0 + k;
    const int c = c0 + threadIdx.x;
    if (i < D && c < p) tile[k][threadIdx.x] = src[i * p + c];
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += 8) {
    const int64_t i = i0 + threadIdx.x;
    const int c = c0 + k;
    if (i < D && c < p) {
      VT* d = dst + (int64_t)c * ld + i;
      if (accumulate) {
        const Cx<A> a = ldout(d), v = ldout(&tile[threadIdx.x][k]);
        stv(d, Cx<A>{a.r + v.r, a.i + v.i});
      } else {
        *d = tile[threadIdx.x][k];
      }
    }
  }
}

template <class VT>
edk_status apply_block_t(edk_operator* op, const void* x, void* y, int64_t nvec, int64_t ldx,
                         int64_t ldy, int accumulate, cudaStream_t st, int bk, int64_t slots) {
  const int64_t D = op->b->D;
  const int pmax = 64;
  const int pc0 = (int)std::min<int64_t>(nvec, pmax);
  const size_t need = (size_t)D * pc0 * sizeof(VT);
  if (op->bx.bytes < need) EDK_RETURN_IF(op->bx.alloc(need));
  if (op->by.bytes < need) EDK_RETURN_IF(op->by.alloc(need));
  VT* bx = op->bx.as<VT>();
  VT* by = op->by.as<VT>();
  const VT* X = static_cast<const VT*>(x);
  VT* Y = static_cast<VT*>(y);
  for (int64_t k0 = 0; k0 < nvec; k0 += pmax) {
    const int pc = (int)std::min<int64_t>(nvec - k0, pmax);
    const dim3 tb(32, 8), tg((unsigned)((D + 31) / 32), (unsigned)((pc + 31) / 32));
    k_cols_to_rows_t<VT><<<tg, tb, 0, st>>>(X + k0 * ldx, ldx, D, pc, bx);
    EDK_TRY_CUDA(cudaGetLastError());
    EDK_RETURN_IF(launch_spmm<VT>(op->bop.as<SpmmOp>(), 1, bk, slots, D, pc, bx, by, 0, st));
    k_rows_to_cols_t<VT><<<tg, tb, 0, st>>>(by, D, pc, Y + k0 * ldy, ldy, accumulate);
    EDK_TRY_CUDA(cudaGetLastError());
  }
  return EDK_OK;
}

// Several right-hand sides on the row-gather paths: one SpMM over row-major
// copies of at most 64 columns at a time, so every hit is located once for
// all of them (false: not applicable, the caller uses the column kernels).
bool block_apply_ok(const edk_operator* op, int64_t nvec) {
  return nvec >= 4 && op->gather && (op->sell_ok || (op->ff_ok && op->use_ff && op->b->dev.L <= 32));
}

edk_status apply_block(edk_operator* op, int dtype, const void* x, void* y, int64_t nvec,
                       int64_t ldx, int64_t ldy, int accumulate, cudaStream_t st) {
  SpmmOp h;
  int bk;
  int64_t slots;
  spmm_describe(op, h, bk, slots);
  std::vector<unsigned char> bytes(sizeof(SpmmOp));
  std::memcpy(bytes.data(), &h, sizeof(SpmmOp));
  if (op->bop_host != bytes || !op->bop.p) {
    if (!op->bop.p) EDK_RETURN_IF(op->bop.alloc(sizeof(SpmmOp)));
    op->bop_host = bytes;
    EDK_TRY_CUDA(cudaMemcpyAsync(op->bop.p, op->bop_host.data(), sizeof(SpmmOp),
                                 cudaMemcpyHostToDevice, st));
  }
  switch (dtype) {
    case EDK_F64: return apply_block_t<double>(op, x, y, nvec, ldx, ldy, accumulate, st, bk, slots);
    case EDK_C128: return apply_block_t<double2>(op, x, y, nvec, ldx, ldy, accumulate, st, bk, slots);
    case EDK_F32: return apply_block_t<float>(op, x, y, nvec, ldx, ldy, accumulate, st, bk, slots);
    case EDK_C64: return apply_block_t<float2>(op, x, y, nvec, ldx, ldy, accumulate, st, bk, slots);
  }
  set_error("apply: unknown dtype");
  return EDK_INVALID_ARG;
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
  // automatic choice: the SpMM for a block of columns unless the operator is
  // materialised or runs on a row plan (both stream one column faster than
  // the SpMM locates hits once for all of them)
  if (block_apply_ok(op, nvec) &&
      (op->use_block > 0 || (op->use_block < 0 && !op->sell_ok && !plan_applies(op))))
    return apply_block(op, dtype, x, y, nvec, ldx, ldy, accumulate, st);
  if (op->sell_ok && !sc) return apply_sell(op, dtype, x, y, nvec, ldx, ldy, accumulate, st);
  if (op->ff_ok && !sc && op->use_ff) {
    if (plan_applies(op)) return apply_plan(op, dtype, x, y, nvec, ldx, ldy, accumulate, st, 0, -1);
    const FFParams& ff = *reinterpret_cast<const FFParams*>(op->ff_params.data());
#define EDK_FF_TPS(VT)                                                                          \
  switch (op->tps) {                                                                            \
    case 2: return launch_apply_ff<VT, 2>(b, op->dev, ff, x, y, nvec, ldx, ldy, accumulate, st); \
    case 4: return launch_apply_ff<VT, 4>(b, op->dev, ff, x, y, nvec, ldx, ldy, accumulate, st); \
    default: return launch_apply_ff<VT, 1>(b, op->dev, ff, x, y, nvec, ldx, ldy, accumulate, st); \
  }
    switch (dtype) {
      case EDK_F64: EDK_FF_TPS(double)
      case EDK_C128: EDK_FF_TPS(double2)
      case EDK_F32: EDK_FF_TPS(float)
      case EDK_C64: EDK_FF_TPS(float2)
    }
#undef EDK_FF_TPS
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
  for (cudaEvent_t e : cevents) cudaEventDestroy(e);
  if (cstream) cudaStreamDestroy(cstream);
  if (stream) cudaStreamDestroy(stream);
}

namespace edk {

bool rows_apply_ok(const edk_operator* op) {
  if (!op->gather) return false;
  return op->sell_ok || (op->ff_ok && op->use_ff);
}

edk_status apply_rows(edk_operator* op, int dtype, const void* x, void* y, int64_t row0,
                      int64_t row1, int accumulate, cudaStream_t st) {
  const BasisDev& b = op->b->dev;
  EDK_RETURN_IF(check_basis_dev(b));
  if (op->sell_ok) return apply_sell_rows(op, dtype, x, y, row0, row1, accumulate, st);
  if (plan_applies(op)) return apply_plan(op, dtype, x, y, 1, b.D, b.D, accumulate, st, row0, row1);
  const FFParams& ff = *reinterpret_cast<const FFParams*>(op->ff_params.data());
  const int64_t D = b.D;
#define EDK_FF_ROWS(VT)                                                                      \
  switch (op->tps) {                                                                         \
    case 2: return launch_apply_ff<VT, 2>(b, op->dev, ff, x, y, 1, D, D, accumulate, st,     \
                                          row0, row1);                                       \
    case 4: return launch_apply_ff<VT, 4>(b, op->dev, ff, x, y, 1, D, D, accumulate, st,     \
                                          row0, row1);                                       \
    default: return launch_apply_ff<VT, 1>(b, op->dev, ff, x, y, 1, D, D, accumulate, st,    \
                                           row0, row1);                                      \
  }
  switch (dtype) {
    case EDK_F64: EDK_FF_ROWS(double)
    case EDK_C128: EDK_FF_ROWS(double2)
    case EDK_F32: EDK_FF_ROWS(float)
    case EDK_C64: EDK_FF_ROWS(float2)
  }
#undef EDK_FF_ROWS
  set_error("apply: unknown dtype");
  return EDK_INVALID_ARG;
}

}  // namespace edk

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
  if (const char* e = std::getenv("EDK_DISABLE_PLAN")) op->use_plan = !(e[0] == '1');
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
        ff.same[f] = ff.v1[f].x == ff.v2[f].x && ff.v1[f].y == ff.v2[f].y;
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

// after a synchronised product: a bounded wait of the staged materialised
// kernel that ran out (never expected) is reported instead of a silent result
static edk_status staged_status(edk_operator* op) {
  if (!(op->sell_ok && op->sell_tma && op->sell_tma_ok && op->s_err.p)) return EDK_OK;
  int err = 0;
  EDK_TRY_CUDA(cudaMemcpy(&err, op->s_err.p, sizeof(int), cudaMemcpyDeviceToHost));
  if (err) {
    // the device did not complete a bulk copy: never use the staged kernel on
    // this operator again (later products take the plain materialised kernel)
    op->sell_tma_ok = false;
    op->sell_tma = false;
    set_error("apply: the staged materialised product timed out waiting for its copies");
    return EDK_TIMEOUT;
  }
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
    return staged_status(op);
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
  constexpr int64_t kChunkRows = 262144;  // a multiple of every tile height
  if (nvec == 1 && D >= 2 * kChunkRows && rows_apply_ok(op)) {
    // pipelined: row chunks computed in order on the operator's stream, each
    // chunk of y copied back on the copy stream while the next one computes
    // (psi gathers reach any row, so the input copy cannot be split this way)
    const int nch = (int)((D + kChunkRows - 1) / kChunkRows);
    if (!op->cstream) EDK_TRY_CUDA(cudaStreamCreateWithFlags(&op->cstream, cudaStreamNonBlocking));
    while ((int)op->cevents.size() < nch) {
      cudaEvent_t e;
      EDK_TRY_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
      op->cevents.push_back(e);
    }
    for (int c = 0; c < nch; ++c) {
      const int64_t r0 = (int64_t)c * kChunkRows, r1 = std::min<int64_t>(D, r0 + kChunkRows);
      EDK_RETURN_IF(apply_rows(op, dtype, dx.p, dy.p, r0, r1, accumulate, st));
      EDK_TRY_CUDA(cudaEventRecord(op->cevents[c], st));
      EDK_TRY_CUDA(cudaStreamWaitEvent(op->cstream, op->cevents[c], 0));
      EDK_TRY_CUDA(cudaMemcpyAsync((char*)y + r0 * es, (char*)dy.p + r0 * es, (r1 - r0) * es,
                                   cudaMemcpyDeviceToHost, op->cstream));
    }
    EDK_TRY_CUDA(cudaStreamSynchronize(op->cstream));
    EDK_TRY_CUDA(cudaStreamSynchronize(st));
    return staged_status(op);
  }
  EDK_RETURN_IF(apply_device(op, dtype, dx.p, dy.p, nvec, D, D, accumulate, st));
  EDK_TRY_CUDA(cudaMemcpy2DAsync(y, ldy * es, dy.p, D * es, D * es, nvec, cudaMemcpyDeviceToHost, st));
  EDK_TRY_CUDA(cudaStreamSynchronize(st));
  return staged_status(op);
}
