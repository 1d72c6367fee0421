// edk_plan.cu — row plans of the flip-flop fast path on rank-searched sectors
// (translation and translation + parity sectors with their rank table, and
// complete fixed-charge sectors), and the kernel that applies H through them.
//
// A plan is built once per operator, on the device, the first time the
// operator is applied with such a search: for every 256-row window the rows
// are ordered by their number of off-diagonal hits, and each slot keeps the
// row's 32-bit state, its colex rank, `row | norm class << 27` and the rank of
// its wrap-around exchange (plus the summed diagonal when the operator has
// diagonal-only generic terms, e.g. random fields).  The product then runs
// one thread per slot with the tables it reads per hit (binomials, norms,
// phases) in shared memory; edk_rankrows.cuh holds the per-row arithmetic.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <type_traits>

#include "edk_rankrows.cuh"

namespace edk {

namespace {

// Order the 256 rows of window blockIdx.x by hit count (ties by row, so the
// plan is the same on every build) and write their slots.
template <int BK>
__global__ void __launch_bounds__(256) k_plan_build(BasisDev b, OpDev op, FFParams ff,
                                                    int want_diag,
                                                    const uint32_t* __restrict__ binom,
                                                    uint4* __restrict__ slot_o,
                                                    double* __restrict__ dg_o,
                                                    int* __restrict__ bad) {
  __shared__ int s_key[kPlanWindow];
  __shared__ uint32_t s_binom[32 * 33];
  for (int q = threadIdx.x; q < 32 * 33; q += blockDim.x) s_binom[q] = __ldg(binom + q);
  __syncthreads();
  const int t = threadIdx.x;
  const int64_t r0 = (int64_t)blockIdx.x * kPlanWindow, i = r0 + t;
  const bool valid = i < b.D;
  const uint32_t mask = (uint32_t)b.maskL;
  uint32_t s = 0, rk = 0, rw = ~0u, rkw = ~0u;
  int key = 1 << 20;  // past the last row: sorted to the end
  double dr = 0.0, di = 0.0;
  if (valid) {
    s = (uint32_t)__ldg(b.I + i);
    key = 0;
    for (int f = 0; f < ff.nfam; ++f)
      key += __popc((s ^ rotl_L(s, ff.d[f], b.L, mask)) & ff.valid[f]);
    uint32_t cls = 0;
    if constexpr (BK == BK_PROJ_RANK) {
      rk = (uint32_t)i;
    } else {
      rk = __ldg(b.rowrank + i);
      const uint32_t v = __ldg(b.rankmap + rk);
      if (v == ~0u || (int64_t)(v >> b.rank_shift) != i) atomicOr(bad, 1);
      cls = v & 31u;
    }
    rw = (uint32_t)i | (cls << 27);
    // the wrap-around bond (bits 0 and L-1) of a nearest-neighbour family:
    // its target rank walks the set bits in between, so it is kept per row
    bool wrap = false;
    for (int f = 0; f < ff.nfam; ++f) wrap |= ff.d[f] == 1 && (ff.valid[f] & 1u);
    if (wrap && ((s ^ (s >> (b.L - 1))) & 1u)) rkw = rank_after_swap(s, rk, 0, b.L - 1, s_binom);
    if (want_diag) {
      for (int f = 0; f < ff.nfam; ++f)
        ff_diag(ff, f, s, rotl_L(s, ff.d[f], b.L, mask), ff.valid[f], dr, di);
      term_diag(op, s, dr, di);
      if (di != 0.0) atomicOr(bad, 2);
    }
  }
  s_key[t] = key;
  __syncthreads();
  int pos = 0;
  for (int u = 0; u < kPlanWindow; ++u) {
    const int ku = s_key[u];
    pos += (ku < key) || (ku == key && u < t);
  }
  const int64_t slot = r0 + pos;
  slot_o[slot] = make_uint4(rw, s, rk, rkw);
  if (want_diag) dg_o[slot] = dr;
}

// NN = 1: the operator is one nearest-neighbour family of equal exchange
// values (its loop only); NN = 2: any other operator (the general loop only)
template <int BK, class VT, int NN>
__global__ void __launch_bounds__(256, plan_min_blocks<BK, VT>())
    k_apply_plan(BasisDev b, OpDev op, FFParams ff, const VT* __restrict__ x,
                 VT* __restrict__ y, int64_t ldx, int64_t ldy, int accumulate, int64_t slot0,
                 int64_t slot1) {
  __shared__ FFTab<BK> sm;
  ff_tab_fill<BK>(sm, b, op.plan.binom);
  __syncthreads();
  const VT* xk = x + (int64_t)blockIdx.y * ldx;
  VT* yk = y + (int64_t)blockIdx.y * ldy;
  for (int64_t s = slot0 + (int64_t)blockIdx.x * kPlanWindow + threadIdx.x; s < slot1;
       s += (int64_t)gridDim.x * kPlanWindow)
    plan_row<BK, VT, NN>(b, op, ff, sm, s, xk, yk, accumulate);
}

int sm_count() {
  static int n[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
  if (!n[dev] && cudaDeviceGetAttribute(&n[dev], cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    n[dev] = 148;
  return n[dev];
}

template <int BK, class VT, int NN>
edk_status launch_plan_nn(const BasisDev& b, const OpDev& op, const FFParams& ff, const VT* X,
                          VT* Y, int64_t nvec, int64_t ldx, int64_t ldy, int accumulate,
                          cudaStream_t st, int64_t slot0, int64_t slot1) {
  static int per_sm = 0;  // resident blocks per SM of this instantiation
  if (!per_sm) {
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_apply_plan<BK, VT, NN>,
                                                      kPlanWindow, 0) != cudaSuccess || per_sm < 1)
      per_sm = 1;
  }
  const int64_t nwin = (slot1 - slot0) / kPlanWindow;
  const unsigned gx = (unsigned)std::min<int64_t>(nwin, (int64_t)sm_count() * per_sm);
  for (int64_t k0 = 0; k0 < nvec; k0 += 65535) {
    const int64_t nk = std::min<int64_t>(nvec - k0, 65535);
    k_apply_plan<BK, VT, NN><<<dim3(gx, (unsigned)nk), kPlanWindow, 0, st>>>(
        b, op, ff, X + k0 * ldx, Y + k0 * ldy, ldx, ldy, accumulate, slot0, slot1);
    EDK_TRY_CUDA(cudaGetLastError());
  }
  return EDK_OK;
}

template <int BK, class VT>
edk_status launch_plan_kind(const BasisDev& b, const OpDev& op, const FFParams& ff, const VT* X,
                            VT* Y, int64_t nvec, int64_t ldx, int64_t ldy, int accumulate,
                            cudaStream_t st, int64_t slot0, int64_t slot1) {
  if (plan_nn(ff))
    return launch_plan_nn<BK, VT, 1>(b, op, ff, X, Y, nvec, ldx, ldy, accumulate, st, slot0, slot1);
  return launch_plan_nn<BK, VT, 2>(b, op, ff, X, Y, nvec, ldx, ldy, accumulate, st, slot0, slot1);
}

// lookup kind of the plan kernels for the basis as it is searched now, or -1
int plan_kind(const BasisDev& b) {
  if (b.bk == BK_PROJ_RANK) return BK_PROJ_RANK;
  if (b.search != 2) return -1;
  switch (b.bk) {
    case BK_TRANS0: return BK_TRANS0_RANK;
    case BK_TRANS: return BK_TRANS_RANK;
    case BK_TRANSPAR: return BK_TRANSPAR_RANK;
  }
  return -1;
}

template <int BK>
edk_status build_plan_kind(edk_operator* op, const FFParams& ff, int want_diag) {
  const BasisDev& b = op->b->dev;
  const int64_t nwin = (b.D + kPlanWindow - 1) / kPlanWindow;
  const int64_t ns = nwin * kPlanWindow;
  cudaStream_t st = op->stream;
  EDK_RETURN_IF(op->p_slot.alloc(ns * sizeof(uint4)));
  if (want_diag) EDK_RETURN_IF(op->p_dg.alloc(ns * 8));
  EDK_RETURN_IF(op->p_bad.alloc(sizeof(int)));
  std::vector<uint32_t> binom(32 * 33, 0);
  for (int p = 0; p < 32; ++p) {
    binom[p * 33] = 1;
    for (int k = 1; k <= p; ++k)
      binom[p * 33 + k] = binom[(p - 1) * 33 + k - 1] + binom[(p - 1) * 33 + k];
  }
  EDK_RETURN_IF(op->p_binom.alloc(binom.size() * 4));
  EDK_TRY_CUDA(cudaMemcpyAsync(op->p_binom.p, binom.data(), binom.size() * 4,
                               cudaMemcpyHostToDevice, st));
  EDK_TRY_CUDA(cudaMemsetAsync(op->p_bad.p, 0, sizeof(int), st));
  k_plan_build<BK><<<(unsigned)nwin, kPlanWindow, 0, st>>>(
      b, op->dev, ff, want_diag, op->p_binom.as<uint32_t>(), op->p_slot.as<uint4>(),
      want_diag ? op->p_dg.as<double>() : nullptr, op->p_bad.as<int>());
  EDK_TRY_CUDA(cudaGetLastError());
  int bad = 0;
  EDK_TRY_CUDA(cudaMemcpyAsync(&bad, op->p_bad.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  EDK_TRY_CUDA(cudaStreamSynchronize(st));
  if (bad & 1) {
    set_error("row plan: a representative's rank-table entry does not point back at its row");
    return EDK_CUDA_ERROR;
  }
  if (bad & 2) return EDK_UNSUPPORTED;  // complex diagonal: keep the tile kernel
  return EDK_OK;
}

void plan_release(edk_operator* op) {
  op->p_slot.release();
  op->p_dg.release();
  op->p_binom.release();
  op->dev.plan = RowPlanDev{};
}

}  // namespace

// The plan applies to this operator as its basis is searched now.
bool plan_applies(const edk_operator* op) {
  const BasisDev& b = op->b->dev;
  return op->use_plan && op->ff_ok && op->use_ff && op->gather && op->tps == 1 && b.L <= 32 &&
         b.D > 0 && b.D <= (int64_t)kPlanRowMask && plan_kind(b) >= 0 &&
         (b.bk == BK_PROJ_RANK || b.packed) && op->plan_state >= 0;
}

// Build the plan the first time it is needed (plan_state: 0 not built yet,
// 1 built, -1 not available for this operator).  Allocates and synchronises:
// call it outside any stream capture.
edk_status plan_ensure(edk_operator* op) {
  if (op->plan_state != 0) return EDK_OK;
  const BasisDev& b = op->b->dev;
  const FFParams& ff = *reinterpret_cast<const FFParams*>(op->ff_params.data());
  const int want_diag = op->ngeneric > 0 ? 1 : 0;
  edk_status rc = EDK_OK;
  switch (plan_kind(b)) {
    case BK_PROJ_RANK: rc = build_plan_kind<BK_PROJ_RANK>(op, ff, want_diag); break;
    case BK_TRANS0_RANK: rc = build_plan_kind<BK_TRANS0_RANK>(op, ff, want_diag); break;
    case BK_TRANS_RANK: rc = build_plan_kind<BK_TRANS_RANK>(op, ff, want_diag); break;
    case BK_TRANSPAR_RANK: rc = build_plan_kind<BK_TRANSPAR_RANK>(op, ff, want_diag); break;
    default: return EDK_OK;
  }
  if (rc == EDK_UNSUPPORTED) {
    plan_release(op);
    op->plan_state = -1;
    return EDK_OK;
  }
  if (rc != EDK_OK) {
    plan_release(op);
    return rc;
  }
  RowPlanDev& pl = op->dev.plan;
  pl.slot = op->p_slot.as<uint4>();
  pl.dg = want_diag ? op->p_dg.as<double>() : nullptr;
  pl.binom = op->p_binom.as<uint32_t>();
  pl.nslots = ((b.D + kPlanWindow - 1) / kPlanWindow) * kPlanWindow;
  op->plan_state = 1;
  return EDK_OK;
}

// Rows [row0, row1) of y = H x through the plan (row0 a multiple of 256,
// row1 a multiple of 256 or the dimension): the slots of the same windows.
edk_status apply_plan(edk_operator* op, int dtype, const void* x, void* y, int64_t nvec,
                      int64_t ldx, int64_t ldy, int accumulate, cudaStream_t st, int64_t row0,
                      int64_t row1) {
  EDK_RETURN_IF(plan_ensure(op));
  const BasisDev& b = op->b->dev;
  const FFParams& ff = *reinterpret_cast<const FFParams*>(op->ff_params.data());
  if (op->plan_state != 1) {
    set_error("row plan: not available for this operator");
    return EDK_UNSUPPORTED;
  }
  if (row1 < 0) row1 = b.D;
  const int64_t slot0 = (row0 / kPlanWindow) * kPlanWindow;
  const int64_t slot1 = std::min<int64_t>(((row1 + kPlanWindow - 1) / kPlanWindow) * kPlanWindow,
                                          op->dev.plan.nslots);
  if (slot1 <= slot0 || nvec <= 0) return EDK_OK;
  auto go = [&](auto vp) -> edk_status {
    using VT = std::remove_pointer_t<decltype(vp)>;
    const VT* X = static_cast<const VT*>(x);
    VT* Y = static_cast<VT*>(y);
    switch (plan_kind(b)) {
      case BK_PROJ_RANK:
        return launch_plan_kind<BK_PROJ_RANK, VT>(b, op->dev, ff, X, Y, nvec, ldx, ldy, accumulate,
                                                  st, slot0, slot1);
      case BK_TRANS0_RANK:
        return launch_plan_kind<BK_TRANS0_RANK, VT>(b, op->dev, ff, X, Y, nvec, ldx, ldy,
                                                    accumulate, st, slot0, slot1);
      case BK_TRANS_RANK:
        return launch_plan_kind<BK_TRANS_RANK, VT>(b, op->dev, ff, X, Y, nvec, ldx, ldy,
                                                   accumulate, st, slot0, slot1);
      case BK_TRANSPAR_RANK:
        return launch_plan_kind<BK_TRANSPAR_RANK, VT>(b, op->dev, ff, X, Y, nvec, ldx, ldy,
                                                      accumulate, st, slot0, slot1);
    }
    set_error("row plan: unknown lookup kind");
    return EDK_INVALID_ARG;
  };
  switch (dtype) {
    case EDK_F64: return go((double*)nullptr);
    case EDK_C128: return go((double2*)nullptr);
    case EDK_F32: return go((float*)nullptr);
    case EDK_C64: return go((float2*)nullptr);
  }
  set_error("apply: unknown dtype");
  return EDK_INVALID_ARG;
}

}  // namespace edk
