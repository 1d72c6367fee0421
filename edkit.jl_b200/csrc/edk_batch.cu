// edk_batch.cu — Lanczos over many independent operators (momentum sectors
// of one chain, disorder instances).
#include <vector>

#include "edk_internal.cuh"

using namespace edk;

extern "C" edk_status edk_batch_lanczos_e0(int32_t nops, edk_operator* const* ops,
                                           const edk_lanczos_opts* opts, const void* v0s,
                                           int32_t v0_dtype, double* evals,
                                           edk_lanczos_diag* diag) {
  EDK_CHECK_ARG(nops >= 0 && ops && opts && v0s && evals, "edk_batch_lanczos_e0: NULL argument");
  EDK_CHECK_ARG(v0_dtype == EDK_F64 || v0_dtype == EDK_C128,
                "edk_batch_lanczos_e0: v0s must be F64 or C128");
  size_t es = v0_dtype == EDK_F64 ? 8 : 16;
  size_t off = 0;
  edk_lanczos_diag tot{};
  for (int q = 0; q < nops; ++q) {
    EDK_CHECK_ARG(ops[q] != nullptr, "edk_batch_lanczos_e0: NULL operator");
    edk_lanczos_diag d{};
    const char* v = static_cast<const char*>(v0s) + off;
    EDK_RETURN_IF(edk_lanczos_e0(ops[q], opts, v, v0_dtype, EDK_HOST, evals + (size_t)q * opts->nev,
                                 nullptr, nullptr, &d));
    off += (size_t)ops[q]->b->D * es;
    tot.steps = std::max(tot.steps, d.steps);
    tot.steps_low = std::max(tot.steps_low, d.steps_low);
    tot.matvecs += d.matvecs;
    tot.breakdown |= d.breakdown;
    tot.seconds += d.seconds;
    tot.seconds_matvec += d.seconds_matvec;
    tot.seconds_reorth += d.seconds_reorth;
    tot.residual = std::max(tot.residual, d.residual);
  }
  if (diag) *diag = tot;
  return EDK_OK;
}
