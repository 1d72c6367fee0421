// edk_tune.cu — autotuner of the operator application.
//
// The best way to apply H depends on the basis and the operator: the
// flip-flop fast kernel or the generic row kernel, how many threads share one
// state (row) in the fast kernel, which index search finds a target
// representative (hash table or binary search over the sorted array), and
// whether materialising the matrix once (the device counterpart of EDKit's
// sparse!(opt), src/Operator.jl:221-285) pays.  edk_operator_autotune times
// every admissible combination on the operator's own basis with the caller's
// vector count and keeps the fastest; every combination gives the same
// product (the tests check this), so the choice changes speed only.
#include <algorithm>
#include <vector>

#include "edk_internal.cuh"

using namespace edk;

namespace {

size_t elem_size(int dtype) {
  switch (dtype) {
    case EDK_F64: return 8;
    case EDK_C128: return 16;
    case EDK_F32: return 4;
    case EDK_C64: return 8;
  }
  return 0;
}

// median time of `reps` back-to-back applications on the operator's stream
// bytes of the rank table of a phase-free translation sector: 4 * C(L, K)
size_t rank_table_bytes(edk_basis* b) {
  uint64_t s0 = 0;
  if (b->D == 0 || cudaMemcpy(&s0, b->I.p, sizeof(uint64_t), cudaMemcpyDeviceToHost) != cudaSuccess)
    return 0;
  const int L = b->L, K = __builtin_popcountll(s0);
  uint64_t n = 1;
  for (int k = 1; k <= K; ++k) n = n * (uint64_t)(L - K + k) / (uint64_t)k;
  return (size_t)n * 4;
}

edk_status time_apply(edk_operator* op, int dtype, const void* x, void* y, int64_t nvec,
                      int reps, double& ms) {
  const int64_t D = op->b->D;
  cudaStream_t st = op->stream;
  for (int w = 0; w < 2; ++w) EDK_RETURN_IF(apply_device(op, dtype, x, y, nvec, D, D, 0, st));
  std::vector<cudaEvent_t> ev(2 * reps);
  for (auto& e : ev) EDK_TRY_CUDA(cudaEventCreate(&e));
  edk_status rc = EDK_OK;
  for (int r = 0; r < reps && rc == EDK_OK; ++r) {
    cudaEventRecord(ev[2 * r], st);
    rc = apply_device(op, dtype, x, y, nvec, D, D, 0, st);
    cudaEventRecord(ev[2 * r + 1], st);
  }
  cudaError_t ce = cudaStreamSynchronize(st);
  std::vector<float> t(reps, 0.f);
  for (int r = 0; r < reps && rc == EDK_OK && ce == cudaSuccess; ++r)
    cudaEventElapsedTime(&t[r], ev[2 * r], ev[2 * r + 1]);
  for (auto& e : ev) cudaEventDestroy(e);
  EDK_RETURN_IF(rc);
  EDK_TRY_CUDA(ce);
  std::sort(t.begin(), t.end());
  ms = t[reps / 2];
  return EDK_OK;
}

}  // namespace

extern "C" edk_status edk_operator_configure(edk_operator* op, int32_t kernel, int32_t tps,
                                             int32_t block) {
  EDK_CHECK_ARG(op != nullptr, "edk_operator_configure: NULL operator");
  EDK_CHECK_ARG(kernel >= EDK_KERNEL_FAST && kernel <= EDK_KERNEL_MATERIALIZED_STAGED,
                "edk_operator_configure: unknown kernel");
  EDK_CHECK_ARG(tps == 1 || tps == 2 || tps == 4,
                "edk_operator_configure: threads per state must be 1, 2 or 4");
  std::lock_guard<std::mutex> lk(op->mu);
  if (kernel == EDK_KERNEL_MATERIALIZED || kernel == EDK_KERNEL_MATERIALIZED_STAGED) {
    if (!op->sell_ok || (kernel == EDK_KERNEL_MATERIALIZED_STAGED && !op->sell_tma_ok)) {
      set_error("edk_operator_configure: that materialised kernel needs a materialised operator "
                "(edk_operator_materialize) whose windows fit the shared-memory stages");
      return EDK_UNSUPPORTED;
    }
    op->sell_tma = kernel == EDK_KERNEL_MATERIALIZED_STAGED;
    op->use_block = block < 0 ? -1 : (block != 0);
    return EDK_OK;
  }
  if (kernel == EDK_KERNEL_FAST && !(op->ff_ok && op->gather)) {
    set_error("edk_operator_configure: the fast kernel does not apply to this operator");
    return EDK_UNSUPPORTED;
  }
  op->use_ff = kernel == EDK_KERNEL_FAST;
  op->tps = tps;
  op->use_block = block < 0 ? -1 : (block != 0);
  return EDK_OK;
}

extern "C" edk_status edk_operator_autotune(edk_operator* op, int32_t dtype, int64_t nvec,
                                            int32_t flags, edk_tune_result* res) {
  EDK_CHECK_ARG(op != nullptr, "edk_operator_autotune: NULL operator");
  EDK_CHECK_ARG(dtype >= EDK_F64 && dtype <= EDK_C64, "edk_operator_autotune: unknown dtype");
  EDK_CHECK_ARG(nvec >= 1, "edk_operator_autotune: nvec must be >= 1");
  if (op->is_complex && (dtype == EDK_F64 || dtype == EDK_F32)) {
    set_error("edk_operator_autotune: the operator has complex matrix elements; use a complex dtype");
    return EDK_INVALID_ARG;
  }
  edk_basis* b = op->b;
  const int64_t D = b->D;
  edk_tune_result out{};
  if (D == 0) {
    out.kernel = op->use_ff && op->ff_ok ? EDK_KERNEL_FAST : EDK_KERNEL_GENERIC;
    out.tps = op->tps;
    edk_basis_get_search(b, &out.search);
    if (res) *res = out;
    return EDK_OK;
  }
  const size_t es = elem_size(dtype);
  DevBuf x, y;
  EDK_RETURN_IF(x.alloc((size_t)nvec * D * es));
  EDK_RETURN_IF(y.alloc((size_t)nvec * D * es));
  // 0x3F in every byte is a finite value of every dtype (about 4.8e-4 / 0.75)
  EDK_TRY_CUDA(cudaMemsetAsync(x.p, 0x3F, (size_t)nvec * D * es, op->stream));

  const bool has_search = b->dev.bk != BK_TENSOR && b->dev.bk != BK_PROJ_RANK;
  std::vector<int> searches{EDK_SEARCH_HASH};
  if (has_search && edk_basis_set_search(b, EDK_SEARCH_SORTED) == EDK_OK)
    searches.push_back(EDK_SEARCH_SORTED);
  // the rank table (4 bytes per state of the charge sector) when it applies
  // and takes at most a quarter of the free memory
  if (has_search && op->ff_ok && op->gather && b->L <= 32 &&
      (b->dev.bk == BK_TRANS0 || (b->dev.bk == BK_TRANS && b->D < (1ll << 22)) ||
       (b->dev.bk == BK_TRANSPAR && b->D < (1ll << 26)))) {
    size_t freeb = 0, totalb = 0;
    if (cudaMemGetInfo(&freeb, &totalb) == cudaSuccess &&
        (b->rankmap.p || rank_table_bytes(b) <= freeb / 4) &&
        edk_basis_set_search(b, EDK_SEARCH_RANK) == EDK_OK)
      searches.push_back(EDK_SEARCH_RANK);
  }
  struct Cand { int kernel, search, tps, block; };
  std::vector<Cand> cands;
  const bool fast = op->ff_ok && op->gather;
  // several right-hand sides: the bond-family and materialised kernels also
  // run as one SpMM over the block (block = 1)
  const bool multi = nvec >= 4 && op->gather;
  for (int s : searches) {
    if (fast)
      for (int t : {1, 2, 4}) cands.push_back({EDK_KERNEL_FAST, s, t, 0});
    if (s == EDK_SEARCH_RANK) continue;  // only the bond-family row kernel reads the rank table
    if (fast && multi && op->b->dev.L <= 32) cands.push_back({EDK_KERNEL_FAST, s, 1, 1});
    cands.push_back({EDK_KERNEL_GENERIC, s, 1, 0});
  }
  const bool was_mat = op->sell_ok;
  if ((flags & EDK_TUNE_MATERIALIZE) || was_mat) {
    cands.push_back({EDK_KERNEL_MATERIALIZED, 0, 1, 0});
    if (multi) cands.push_back({EDK_KERNEL_MATERIALIZED, 0, 1, 1});
    else cands.push_back({EDK_KERNEL_MATERIALIZED_STAGED, 0, 1, 0});
  }

  const int reps = 7;
  double best = 1e300, best_free = 1e300;
  Cand pick = cands.front(), pick_free = cands.front();
  edk_status rc = EDK_OK;
  for (const Cand& c : cands) {
    double ms = -1.0;
    const bool matk = c.kernel == EDK_KERNEL_MATERIALIZED || c.kernel == EDK_KERNEL_MATERIALIZED_STAGED;
    if (matk) {
      if (edk_operator_materialize(op, 1, nullptr) != EDK_OK) continue;  // not materialisable
      if (c.kernel == EDK_KERNEL_MATERIALIZED_STAGED && !op->sell_tma_ok) continue;
      op->sell_tma = c.kernel == EDK_KERNEL_MATERIALIZED_STAGED;
    } else {
      if (op->sell_ok) edk_operator_materialize(op, 0, nullptr);
      edk_basis_set_search(b, c.search);
      op->use_ff = c.kernel == EDK_KERNEL_FAST;
      op->tps = c.tps;
    }
    op->use_block = c.block;
    {
      std::lock_guard<std::mutex> lk(op->mu);
      rc = time_apply(op, dtype, x.p, y.p, nvec, reps, ms);
    }
    if (rc != EDK_OK) break;
    if (out.ncand < EDK_TUNE_MAX) {
      out.cand_kernel[out.ncand] = c.kernel;
      out.cand_search[out.ncand] = c.search;
      out.cand_tps[out.ncand] = c.tps;
      out.cand_block[out.ncand] = c.block;
      out.cand_ms[out.ncand] = ms;
      ++out.ncand;
    }
    if (ms < best) { best = ms; pick = c; }
    if (!matk && ms < best_free) { best_free = ms; pick_free = c; }
  }
  if (rc != EDK_OK) return rc;
  // install the fastest matrix-free choice (it also serves whenever the
  // materialised matrix is cleared), then the matrix if that wins
  const bool pick_mat =
      pick.kernel == EDK_KERNEL_MATERIALIZED || pick.kernel == EDK_KERNEL_MATERIALIZED_STAGED;
  if (op->sell_ok && !pick_mat) edk_operator_materialize(op, 0, nullptr);
  if (has_search) edk_basis_set_search(b, pick_free.search);
  op->use_ff = pick_free.kernel == EDK_KERNEL_FAST;
  op->tps = pick_free.tps;
  op->use_block = multi ? (pick_mat ? pick : pick_free).block : -1;
  if (pick_mat) {
    EDK_RETURN_IF(edk_operator_materialize(op, 1, nullptr));
    op->sell_tma = pick.kernel == EDK_KERNEL_MATERIALIZED_STAGED;
  }
  out.kernel = pick.kernel;
  edk_basis_get_search(b, &out.search);
  out.tps = pick_free.tps;
  out.block = pick.block;
  out.ms = best;
  if (res) *res = out;
  return EDK_OK;
}
