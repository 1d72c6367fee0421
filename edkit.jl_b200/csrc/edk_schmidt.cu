// edk_schmidt.cu — eigenvector post-processing on the device: the Schmidt
// matrix of a sector vector, its singular values and entanglement entropies,
// and the DoubleBasis map and symmetrizer between two bases of one chain.
//
// Reference:
//   schmidtmatrix / addto!          src/Schmidt.jl:16-71
//   schmidt per basis type          src/Schmidt.jl:186-336,
//                                   src/Basis/AbelianBasis.jl:704-719
//   ent_spec / entropy / ent_S      src/Schmidt.jl:84-165
//   orbit_order / basis_embedding   src/LinearMap.jl:25, 57-70
//   DoubleBasis action, symmetrizer src/LinearMap.jl:140-185
//
// Schmidt matrix.  One thread per representative expands it over its orbit
// in the reference's order (translations right by the unit cell with the
// phase C[j], then the reflected / flipped copy times P, or the generator
// odometer with the product of generator phases) and adds v[i] / R[i] times
// the weight at (row, column) = (A digits, B digits) of each orbit member.
// Orbits of different representatives are disjoint, so every entry is owned
// by one thread and updated without atomics, in the reference's summation
// order.  Singular values come from the Gram matrix (cuBLAS SYRK / HERK on
// the smaller side) and a dense symmetric eigensolver (cuSOLVER SYEVD /
// HEEVD), the GEMM-shaped route; eigenvalues of the Gram matrix below
// n * eps * lambda_max (its rounding floor) are reported as zero.
//
// DoubleBasis: one thread per full-space state looks the state up in the
// source basis and, when present, in the target basis, and accumulates
// conj(c1 / ord1) * (c2 / ord2) * v[pos2] into out[pos1] (atomics: a target
// row collects every member of its orbit).
#include <cublas_v2.h>
#include <cusolverDn.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "edk_lookup.cuh"

namespace edk {
namespace {

// Site split of a state into the (row, column) of the Schmidt matrix: for
// byte q of the state and its value u, a[q][u] holds the bits that byte
// contributes to the A index and b[q][u] those of the B index.  Site i
// (1-based) is bit L - i of the state; the A index is big-endian in Ainds
// order, the B index big-endian over the remaining sites in ascending order
// (schmidtmatrix with TensorBasis subsystems, Schmidt.jl:39-57).
struct SplitTab {
  uint32_t a[4][256];
  uint32_t b[4][256];
};

enum OrbitKind : int { ORB_ONSITE = 0, ORB_TRANS = 1, ORB_TRANSPAR = 2, ORB_GROUP = 3 };

int grid_of(int64_t n, int block = 256, int cap = 148 * 16) {
  int64_t g = (n + block - 1) / block;
  if (g < 1) g = 1;
  return (int)std::min<int64_t>(g, cap);
}

__device__ __forceinline__ void split_state(const uint32_t* sa, const uint32_t* sb, uint32_t t,
                                            uint32_t& ia, uint32_t& ib) {
  const uint32_t u0 = t & 255u, u1 = (t >> 8) & 255u, u2 = (t >> 16) & 255u, u3 = t >> 24;
  ia = sa[u0] | sa[256 + u1] | sa[512 + u2] | sa[768 + u3];
  ib = sb[u0] | sb[256 + u1] | sb[512 + u2] | sb[768 + u3];
}

// M[ia + ib * dA] += w * val  (the thread owns the entry; no atomics)
template <bool CM>
__device__ __forceinline__ void addto(void* M, const uint32_t* sa, const uint32_t* sb,
                                      uint64_t dA, uint32_t t, double wr, double wi, double vr,
                                      double vi) {
  uint32_t ia, ib;
  split_state(sa, sb, t, ia, ib);
  const uint64_t idx = (uint64_t)ia + (uint64_t)ib * dA;
  if constexpr (CM) {
    double2* m = reinterpret_cast<double2*>(M) + idx;
    double2 c = *m;
    c.x += wr * vr - wi * vi;
    c.y += wr * vi + wi * vr;
    *m = c;
  } else {
    double* m = reinterpret_cast<double*>(M) + idx;
    *m += wr * vr;
  }
}

template <int ORB, bool CV, bool CM>
__global__ void k_schmidt(BasisDev b, const void* __restrict__ v, const SplitTab* __restrict__ tab,
                          uint64_t dA, void* M) {
  __shared__ uint32_t sa[1024], sb[1024];
  for (int q = threadIdx.x; q < 1024; q += blockDim.x) {
    sa[q] = tab->a[q >> 8][q & 255];
    sb[q] = tab->b[q >> 8][q & 255];
  }
  __syncthreads();
  const uint32_t mask = (uint32_t)b.maskL;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < b.D;
       i += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t s = b.I ? (uint32_t)__ldg(reinterpret_cast<const unsigned long long*>(b.I) + i)
                           : (uint32_t)i;
    double vr, vi = 0.0;
    if constexpr (CV) {
      const double2 x = __ldg(reinterpret_cast<const double2*>(v) + i);
      vr = x.x; vi = x.y;
    } else {
      vr = __ldg(reinterpret_cast<const double*>(v) + i);
    }
    if constexpr (ORB == ORB_ONSITE) {  // Schmidt.jl:186-194
      addto<CM>(M, sa, sb, dA, s, 1.0, 0.0, vr, vi);
      continue;
    } else {
      const double r = __ldg(b.R + i);  // val = v[i] / R[i]
      vr /= r;
      vi /= r;
      if constexpr (ORB == ORB_TRANS || ORB == ORB_TRANSPAR) {
        // Schmidt.jl:202-216 and parity_schmidt :249-270: circshift!(dgt, A)
        // moves digits right (rotation right by A); weight phase^j = C[j]
        uint32_t t = s;
        for (int j = 0; j < b.len; ++j) {
          const double2 c = __ldg(b.phase + j);
          addto<CM>(M, sa, sb, dA, t, c.x, c.y, vr, vi);
          t = rotr_L(t, b.A, b.L, mask);
        }
        if constexpr (ORB == ORB_TRANSPAR) {
          t = rev_L(s, b.L);
          const double P = (double)b.P;
          for (int j = 0; j < b.len; ++j) {
            const double2 c = __ldg(b.phase + j);
            addto<CM>(M, sa, sb, dA, t, P * c.x, P * c.y, vr, vi);
            t = rotr_L(t, b.A, b.L, mask);
          }
        }
      } else {  // AbelianBasis.jl:704-719: odometer over the generators (:282-289)
        int cnt[kMaxGen];
        int64_t order = 1;
        for (int g = 0; g < b.ngen; ++g) {
          cnt[g] = 0;
          order *= b.gens[g].order;
        }
        uint32_t cur = s;
        addto<CM>(M, sa, sb, dA, cur, 1.0, 0.0, vr, vi);
        for (int64_t e = 1; e < order; ++e) {
          for (int g = 0; g < b.ngen; ++g) {
            cur = apply_gen(b.gens[g], cur, b.L, mask);
            if (++cnt[g] >= b.gens[g].order) cnt[g] = 0;
            else break;
          }
          // phase(g) = prod over generators of c_g[s_g] (AbelianBasis.jl:224-226)
          double2 c = __ldg(b.phase + b.gens[0].phase_off + cnt[0]);
          double pr = c.x, pi = c.y;
          for (int g = 1; g < b.ngen; ++g) {
            c = __ldg(b.phase + b.gens[g].phase_off + cnt[g]);
            const double nr = pr * c.x - pi * c.y, ni = pr * c.y + pi * c.x;
            pr = nr;
            pi = ni;
          }
          addto<CM>(M, sa, sb, dA, cur, pr, pi, vr, vi);
        }
      }
    }
  }
}

// index(b, s) with the lookup kind chosen at run time (two bases of different
// kinds in one kernel)
__device__ __forceinline__ bool lookup_any(const BasisDev& b, uint32_t s, const uint32_t* binom,
                                           Hit& h) {
  switch (b.bk) {
    case BK_TENSOR: return lookup<BK_TENSOR, uint32_t>(b, s, binom, h);
    case BK_PROJ_RANK: return lookup<BK_PROJ_RANK, uint32_t>(b, s, binom, h);
    case BK_PROJ_HASH: return lookup<BK_PROJ_HASH, uint32_t>(b, s, binom, h);
    case BK_TRANS0: return lookup<BK_TRANS0, uint32_t>(b, s, binom, h);
    case BK_TRANS: return lookup<BK_TRANS, uint32_t>(b, s, binom, h);
    case BK_TRANSPAR: return lookup<BK_TRANSPAR, uint32_t>(b, s, binom, h);
    default: return lookup<BK_ABELIAN, uint32_t>(b, s, binom, h);
  }
}

// MATRIX = false: out[pos1] += conj(c1/o1) (c2/o2) v[pos2]   (LinearMap.jl:152-163)
// MATRIX = true:  out[pos1 + pos2 * D1] += conj(c1/o1) (c2/o2)  (symmetrizer)
template <bool MATRIX, bool CV>
__global__ void k_double_map(BasisDev b1, BasisDev b2, double o1, double o2,
                             const void* __restrict__ v, double2* out, uint64_t nfull) {
  __shared__ uint32_t s_binom[32 * 33];
  for (int q = threadIdx.x; q < 32 * 33; q += blockDim.x) {
    const int pp = q / 33, kk = q % 33;
    uint64_t c = 1;
    if (kk > pp) c = 0;
    else
      for (int r = 1; r <= kk; ++r) c = c * (uint64_t)(pp - kk + r) / (uint64_t)r;
    s_binom[q] = (uint32_t)c;
  }
  __syncthreads();
  for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < nfull;
       j += (uint64_t)gridDim.x * blockDim.x) {
    Hit h2, h1;
    if (!lookup_any(b2, (uint32_t)j, s_binom, h2)) continue;
    if (!lookup_any(b1, (uint32_t)j, s_binom, h1)) continue;
    const double c1r = (h1.pre * h1.rpos) / o1, c1i = (h1.pim * h1.rpos) / o1;
    const double c2r = (h2.pre * h2.rpos) / o2, c2i = (h2.pim * h2.rpos) / o2;
    // conj(c1) * c2
    double wr = c1r * c2r + c1i * c2i, wi = c1r * c2i - c1i * c2r;
    double2* dst;
    if constexpr (MATRIX) {
      dst = out + (uint64_t)h1.pos + (uint64_t)h2.pos * (uint64_t)b1.D;
    } else {
      double xr, xi = 0.0;
      if constexpr (CV) {
        const double2 x = __ldg(reinterpret_cast<const double2*>(v) + h2.pos);
        xr = x.x; xi = x.y;
      } else {
        xr = __ldg(reinterpret_cast<const double*>(v) + h2.pos);
      }
      const double nr = wr * xr - wi * xi, ni = wr * xi + wi * xr;
      wr = nr;
      wi = ni;
      dst = out + h1.pos;
    }
    atomicAdd(&dst->x, wr);
    atomicAdd(&dst->y, wi);
  }
}

int orbit_kind(const edk_basis* b) {
  switch (b->kind) {
    case EDK_TENSOR:
    case EDK_PROJECTED: return ORB_ONSITE;
    case EDK_TRANSLATIONAL: return ORB_TRANS;
    case EDK_TRANSPARITY: return ORB_TRANSPAR;
    default: return ORB_GROUP;
  }
}

// order(B) as orbit_order uses it (LinearMap.jl:25): 1 for onsite bases,
// L for TranslationalBasis (TranslationalBasis.jl:349), 2L for
// TranslationParityBasis / TranslationFlipBasis (TranslationalParityBasis.jl:241,
// TranslationalFlipBasis.jl:222), the product of the generator orders for the
// symmetry-group bases (AbelianBasis.jl:507; 2, 2, 4 for Parity / Flip /
// ParityFlip, ParityBasis.jl:128, FlipBasis.jl:122, ParityFlipBasis.jl:152).
double orbit_order(const edk_basis* b) {
  switch (b->kind) {
    case EDK_TENSOR:
    case EDK_PROJECTED: return 1.0;
    case EDK_TRANSLATIONAL: return (double)b->L;
    case EDK_TRANSPARITY: return 2.0 * b->L;
    default: {
      if (b->pairnorm) return 2.0 * b->L;
      double o = 1.0;
      for (int q : b->gen_order) o *= (double)q;
      return o;
    }
  }
}

edk_status make_split(const edk_basis* b, int32_t nA, const int32_t* Ainds, SplitTab& t,
                      uint64_t& dA, uint64_t& dB) {
  const int L = b->L;
  EDK_CHECK_ARG(b->desc.base == 2, "schmidt: the device path supports base 2");
  EDK_CHECK_ARG(L >= 1 && L <= 32, "schmidt: the device path supports L <= 32");
  EDK_CHECK_ARG(nA >= 0 && nA <= L, "schmidt: Ainds has more sites than the chain");
  EDK_CHECK_ARG(nA == 0 || Ainds != nullptr, "schmidt: Ainds is NULL");
  std::vector<int> posA(L + 1, -1), posB(L + 1, -1);
  for (int q = 0; q < nA; ++q) {
    const int site = Ainds[q];
    EDK_CHECK_ARG(site >= 1 && site <= L, "schmidt: site index out of range");
    EDK_CHECK_ARG(posA[site] < 0, "schmidt: repeated site in Ainds");
    posA[site] = q;
  }
  int nB = 0;
  for (int site = 1; site <= L; ++site)
    if (posA[site] < 0) posB[site] = nB++;
  std::memset(&t, 0, sizeof(t));
  for (int q = 0; q < 4; ++q)
    for (int u = 0; u < 256; ++u)
      for (int bit = 0; bit < 8; ++bit) {
        if (!((u >> bit) & 1)) continue;
        const int sbit = 8 * q + bit;
        if (sbit >= L) continue;
        const int site = L - sbit;
        if (posA[site] >= 0) t.a[q][u] |= 1u << (nA - 1 - posA[site]);
        else t.b[q][u] |= 1u << (nB - 1 - posB[site]);
      }
  dA = 1ull << nA;
  dB = 1ull << nB;
  return EDK_OK;
}

bool basis_complex(const edk_basis* b) { return b->phase_complex; }

// Schmidt matrix of the device vector v_d into the zeroed device matrix M_d.
edk_status schmidt_device(edk_basis* b, int vdt, const void* v_d, const SplitTab& tab,
                          uint64_t dA, int mdt, void* M_d, cudaStream_t st) {
  EDK_RETURN_IF(check_basis_dev(b->dev));
  if (b->D == 0) return EDK_OK;
  DevBuf dtab;
  EDK_RETURN_IF(dtab.alloc(sizeof(SplitTab)));
  EDK_TRY_CUDA(cudaMemcpyAsync(dtab.p, &tab, sizeof(SplitTab), cudaMemcpyHostToDevice, st));
  const int orb = orbit_kind(b);
  EDK_CHECK_ARG(orb == ORB_ONSITE || b->dev.R != nullptr, "internal: basis norms missing");
  const bool cv = vdt == EDK_C128, cm = mdt == EDK_C128;
  const int g = grid_of(b->D);
  const SplitTab* tp = dtab.as<SplitTab>();
#define EDK_SCH(ORB)                                                                          \
  case ORB:                                                                                   \
    if (cv) k_schmidt<ORB, true, true><<<g, 256, 0, st>>>(b->dev, v_d, tp, dA, M_d);          \
    else if (cm) k_schmidt<ORB, false, true><<<g, 256, 0, st>>>(b->dev, v_d, tp, dA, M_d);    \
    else k_schmidt<ORB, false, false><<<g, 256, 0, st>>>(b->dev, v_d, tp, dA, M_d);           \
    break;
  switch (orb) {
    EDK_SCH(ORB_ONSITE)
    EDK_SCH(ORB_TRANS)
    EDK_SCH(ORB_TRANSPAR)
    EDK_SCH(ORB_GROUP)
  }
#undef EDK_SCH
  EDK_TRY_CUDA(cudaGetLastError());
  // the split table must outlive the kernel
  EDK_TRY_CUDA(cudaStreamSynchronize(st));
  return EDK_OK;
}

edk_status check_v_dtype(int vdt) {
  EDK_CHECK_ARG(vdt == EDK_F64 || vdt == EDK_C128, "schmidt: v must be F64 or C128");
  return EDK_OK;
}

const char* solver_msg(cusolverStatus_t s) {
  switch (s) {
    case CUSOLVER_STATUS_NOT_INITIALIZED: return "not initialized";
    case CUSOLVER_STATUS_ALLOC_FAILED: return "allocation failed";
    case CUSOLVER_STATUS_INVALID_VALUE: return "invalid value";
    case CUSOLVER_STATUS_EXECUTION_FAILED: return "execution failed";
    case CUSOLVER_STATUS_INTERNAL_ERROR: return "internal error";
    default: return "error";
  }
}

#define EDK_TRY_SOLVER(call)                                                         \
  do {                                                                               \
    cusolverStatus_t s_ = (call);                                                    \
    if (s_ != CUSOLVER_STATUS_SUCCESS) {                                             \
      set_error(std::string(#call) + " failed: cuSOLVER " + solver_msg(s_));         \
      return EDK_CUDA_ERROR;                                                         \
    }                                                                                \
  } while (0)
#define EDK_TRY_CUBLAS(call)                                                         \
  do {                                                                               \
    cublasStatus_t s_ = (call);                                                      \
    if (s_ != CUBLAS_STATUS_SUCCESS) {                                               \
      set_error(std::string(#call) + " failed: cuBLAS status " + std::to_string((int)s_)); \
      return EDK_CUDA_ERROR;                                                         \
    }                                                                                \
  } while (0)

struct Handles {
  cublasHandle_t blas = nullptr;
  cusolverDnHandle_t solver = nullptr;
  ~Handles() {
    if (blas) cublasDestroy(blas);
    if (solver) cusolverDnDestroy(solver);
  }
};

// Squared singular values of the dA x dB column-major device matrix M_d,
// descending, into s2 (min(dA, dB) values).
edk_status gram_spectrum(const void* M_d, bool cm, uint64_t dA, uint64_t dB, cudaStream_t st,
                         std::vector<double>& s2) {
  const uint64_t n64 = std::min(dA, dB), k64 = std::max(dA, dB);
  EDK_CHECK_ARG(n64 <= 32768, "ent_spec: the smaller side of the Schmidt matrix exceeds 32768");
  EDK_CHECK_ARG(k64 < (1ull << 31), "ent_spec: the larger side of the Schmidt matrix exceeds 2^31");
  const int n = (int)n64, k = (int)k64, lda = (int)dA;
  const bool rows = dA <= dB;  // G = M M^H (dA x dA) or M^H M (dB x dB)
  Handles h;
  EDK_TRY_CUBLAS(cublasCreate(&h.blas));
  EDK_TRY_CUBLAS(cublasSetStream(h.blas, st));
  EDK_TRY_SOLVER(cusolverDnCreate(&h.solver));
  EDK_TRY_SOLVER(cusolverDnSetStream(h.solver, st));
  const size_t es = cm ? 16 : 8;
  DevBuf G, W, info, work;
  EDK_RETURN_IF(G.alloc((size_t)n * n * es));
  EDK_RETURN_IF(W.alloc((size_t)n * 8));
  EDK_RETURN_IF(info.alloc(sizeof(int)));
  const double one = 1.0, zero = 0.0;
  int lwork = 0;
  if (cm) {
    EDK_TRY_CUBLAS(cublasZherk(h.blas, CUBLAS_FILL_MODE_LOWER, rows ? CUBLAS_OP_N : CUBLAS_OP_C,
                               n, k, &one, reinterpret_cast<const cuDoubleComplex*>(M_d), lda,
                               &zero, G.as<cuDoubleComplex>(), n));
    EDK_TRY_SOLVER(cusolverDnZheevd_bufferSize(h.solver, CUSOLVER_EIG_MODE_NOVECTOR,
                                               CUBLAS_FILL_MODE_LOWER, n, G.as<cuDoubleComplex>(),
                                               n, W.as<double>(), &lwork));
    EDK_RETURN_IF(work.alloc((size_t)std::max(lwork, 1) * 16));
    EDK_TRY_SOLVER(cusolverDnZheevd(h.solver, CUSOLVER_EIG_MODE_NOVECTOR, CUBLAS_FILL_MODE_LOWER,
                                    n, G.as<cuDoubleComplex>(), n, W.as<double>(),
                                    work.as<cuDoubleComplex>(), lwork, info.as<int>()));
  } else {
    EDK_TRY_CUBLAS(cublasDsyrk(h.blas, CUBLAS_FILL_MODE_LOWER, rows ? CUBLAS_OP_N : CUBLAS_OP_T,
                               n, k, &one, reinterpret_cast<const double*>(M_d), lda, &zero,
                               G.as<double>(), n));
    EDK_TRY_SOLVER(cusolverDnDsyevd_bufferSize(h.solver, CUSOLVER_EIG_MODE_NOVECTOR,
                                               CUBLAS_FILL_MODE_LOWER, n, G.as<double>(), n,
                                               W.as<double>(), &lwork));
    EDK_RETURN_IF(work.alloc((size_t)std::max(lwork, 1) * 8));
    EDK_TRY_SOLVER(cusolverDnDsyevd(h.solver, CUSOLVER_EIG_MODE_NOVECTOR, CUBLAS_FILL_MODE_LOWER,
                                    n, G.as<double>(), n, W.as<double>(), work.as<double>(),
                                    lwork, info.as<int>()));
  }
  std::vector<double> w(n);
  int hinfo = 0;
  EDK_TRY_CUDA(cudaMemcpyAsync(w.data(), W.p, (size_t)n * 8, cudaMemcpyDeviceToHost, st));
  EDK_TRY_CUDA(cudaMemcpyAsync(&hinfo, info.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  EDK_TRY_CUDA(cudaStreamSynchronize(st));
  if (hinfo != 0) {
    set_error("ent_spec: the eigensolver did not converge (info " + std::to_string(hinfo) + ")");
    return EDK_NOT_CONVERGED;
  }
  // ascending -> descending; the rounding floor of the Gram matrix is zero
  const double lmax = std::max(w.empty() ? 0.0 : w.back(), 0.0);
  const double floor_ = (double)n * 2.220446049250313e-16 * lmax;
  s2.resize(n);
  for (int q = 0; q < n; ++q) {
    const double x = w[n - 1 - q];
    s2[q] = x > floor_ ? x : 0.0;
  }
  return EDK_OK;
}

// entropy(s; alpha, cutoff) on squared Schmidt values, descending
// (Schmidt.jl:101-139)
double entropy_of(const std::vector<double>& s, double alpha, double cutoff) {
  if (alpha == 1.0) {
    double ent = 0.0;
    for (double si : s) {
      if (!(si > cutoff)) break;
      ent -= si * std::log(si);
    }
    return ent;
  }
  if (alpha == 0.0) {
    int64_t n = 0;
    for (double si : s) {
      if (!(si > cutoff)) break;
      ++n;
    }
    return (double)n;
  }
  double sum = 0.0;
  for (double si : s) sum += std::pow(si, alpha);
  return std::log(sum) / (1.0 - alpha);
}

// Schmidt matrix in device memory for the spectrum routines (complex when v
// or the basis phases are complex).
edk_status schmidt_for_spectrum(edk_basis* b, int vdt, const void* v, int32_t nA,
                                const int32_t* Ainds, int32_t ptr_kind, std::vector<double>& s2) {
  EDK_RETURN_IF(check_v_dtype(vdt));
  EDK_CHECK_ARG(v != nullptr || b->D == 0, "ent_spec: v is NULL");
  SplitTab tab;
  uint64_t dA = 0, dB = 0;
  EDK_RETURN_IF(make_split(b, nA, Ainds, tab, dA, dB));
  const bool cm = vdt == EDK_C128 || basis_complex(b);
  cudaStream_t st = b->stream;
  const size_t vb = (size_t)b->D * (vdt == EDK_C128 ? 16 : 8);
  DevBuf dv, dM;
  const void* v_d = v;
  if (ptr_kind == EDK_HOST && b->D > 0) {
    EDK_RETURN_IF(dv.alloc(vb));
    EDK_TRY_CUDA(cudaMemcpyAsync(dv.p, v, vb, cudaMemcpyHostToDevice, st));
    v_d = dv.p;
  }
  const size_t mb = (size_t)(dA * dB) * (cm ? 16 : 8);
  EDK_RETURN_IF(dM.alloc(mb));
  EDK_TRY_CUDA(cudaMemsetAsync(dM.p, 0, mb, st));
  EDK_RETURN_IF(schmidt_device(b, vdt, v_d, tab, dA, cm ? EDK_C128 : EDK_F64, dM.p, st));
  return gram_spectrum(dM.p, cm, dA, dB, st, s2);
}

struct BasisPairLock {
  std::unique_lock<std::mutex> a, b;
  BasisPairLock(edk_basis* x, edk_basis* y) {
    if (x == y) {
      a = std::unique_lock<std::mutex>(x->mu);
    } else if (x < y) {
      a = std::unique_lock<std::mutex>(x->mu);
      b = std::unique_lock<std::mutex>(y->mu);
    } else {
      a = std::unique_lock<std::mutex>(y->mu);
      b = std::unique_lock<std::mutex>(x->mu);
    }
  }
};

edk_status check_pair(const edk_basis* b1, const edk_basis* b2) {
  EDK_CHECK_ARG(b1 && b2, "DoubleBasis: NULL basis");
  if (b1->L != b2->L) {
    set_error("DoubleBasis requires bases with the same length.");
    return EDK_INVALID_ARG;
  }
  if (b1->desc.base != b2->desc.base) {
    set_error("DoubleBasis requires bases with the same local base.");
    return EDK_INVALID_ARG;
  }
  EDK_CHECK_ARG(b1->desc.base == 2, "DoubleBasis: the device path supports base 2");
  EDK_CHECK_ARG(b1->L <= 32, "DoubleBasis: the device path supports L <= 32");
  EDK_CHECK_ARG(b1->device == b2->device, "DoubleBasis: bases live on different devices");
  EDK_RETURN_IF(check_basis_dev(b1->dev));
  EDK_RETURN_IF(check_basis_dev(b2->dev));
  return EDK_OK;
}

}  // namespace
}  // namespace edk

using namespace edk;

extern "C" edk_status edk_schmidt(const edk_basis* bc, int32_t vdtype, const void* v, int32_t nA,
                                  const int32_t* Ainds, void* M, int32_t mdtype,
                                  int32_t ptr_kind) {
  EDK_CHECK_ARG(bc != nullptr && M != nullptr, "edk_schmidt: NULL argument");
  edk_basis* b = const_cast<edk_basis*>(bc);
  std::lock_guard<std::mutex> lk(b->mu);
  EDK_RETURN_IF(check_v_dtype(vdtype));
  EDK_CHECK_ARG(mdtype == EDK_F64 || mdtype == EDK_C128, "edk_schmidt: M must be F64 or C128");
  EDK_CHECK_ARG(mdtype == EDK_C128 || (vdtype == EDK_F64 && !basis_complex(b)),
                "edk_schmidt: a complex vector or complex basis phases need a C128 matrix");
  EDK_CHECK_ARG(v != nullptr || b->D == 0, "edk_schmidt: v is NULL");
  SplitTab tab;
  uint64_t dA = 0, dB = 0;
  EDK_RETURN_IF(make_split(b, nA, Ainds, tab, dA, dB));
  cudaStream_t st = b->stream;
  const size_t mb = (size_t)(dA * dB) * (mdtype == EDK_C128 ? 16 : 8);
  const size_t vb = (size_t)b->D * (vdtype == EDK_C128 ? 16 : 8);
  if (ptr_kind == EDK_HOST) {
    DevBuf dv, dM;
    if (b->D > 0) {
      EDK_RETURN_IF(dv.alloc(vb));
      EDK_TRY_CUDA(cudaMemcpyAsync(dv.p, v, vb, cudaMemcpyHostToDevice, st));
    }
    EDK_RETURN_IF(dM.alloc(mb));
    EDK_TRY_CUDA(cudaMemsetAsync(dM.p, 0, mb, st));
    EDK_RETURN_IF(schmidt_device(b, vdtype, dv.p, tab, dA, mdtype, dM.p, st));
    EDK_TRY_CUDA(cudaMemcpyAsync(M, dM.p, mb, cudaMemcpyDeviceToHost, st));
    EDK_TRY_CUDA(cudaStreamSynchronize(st));
    return EDK_OK;
  }
  EDK_TRY_CUDA(cudaMemsetAsync(M, 0, mb, st));
  return schmidt_device(b, vdtype, v, tab, dA, mdtype, M, st);
}

extern "C" edk_status edk_ent_spec(const edk_basis* bc, int32_t vdtype, const void* v, int32_t nA,
                                   const int32_t* Ainds, double* s, int64_t* ns,
                                   int32_t ptr_kind) {
  EDK_CHECK_ARG(bc != nullptr && ns != nullptr, "edk_ent_spec: NULL argument");
  edk_basis* b = const_cast<edk_basis*>(bc);
  std::lock_guard<std::mutex> lk(b->mu);
  std::vector<double> s2;
  EDK_RETURN_IF(schmidt_for_spectrum(b, vdtype, v, nA, Ainds, ptr_kind, s2));
  *ns = (int64_t)s2.size();
  if (s)
    for (size_t q = 0; q < s2.size(); ++q) s[q] = std::sqrt(s2[q]);
  return EDK_OK;
}

extern "C" edk_status edk_ent_S(const edk_basis* bc, int32_t vdtype, const void* v, int32_t nA,
                                const int32_t* Ainds, double alpha, double cutoff, double* S,
                                int32_t ptr_kind) {
  EDK_CHECK_ARG(bc != nullptr && S != nullptr, "edk_ent_S: NULL argument");
  EDK_CHECK_ARG(alpha >= 0.0, "edk_ent_S: alpha < 0");
  edk_basis* b = const_cast<edk_basis*>(bc);
  std::lock_guard<std::mutex> lk(b->mu);
  std::vector<double> s2;
  EDK_RETURN_IF(schmidt_for_spectrum(b, vdtype, v, nA, Ainds, ptr_kind, s2));
  *S = entropy_of(s2, alpha, cutoff);  // ent_S squares ent_spec (Schmidt.jl:150-153)
  return EDK_OK;
}

extern "C" edk_status edk_double_basis_apply(const edk_basis* b1c, const edk_basis* b2c,
                                             int32_t vdtype, const void* v, double* out,
                                             int32_t ptr_kind) {
  EDK_RETURN_IF(check_pair(b1c, b2c));
  EDK_RETURN_IF(check_v_dtype(vdtype));
  EDK_CHECK_ARG(out != nullptr || b1c->D == 0, "edk_double_basis_apply: out is NULL");
  EDK_CHECK_ARG(v != nullptr || b2c->D == 0, "edk_double_basis_apply: v is NULL");
  edk_basis* b1 = const_cast<edk_basis*>(b1c);
  edk_basis* b2 = const_cast<edk_basis*>(b2c);
  BasisPairLock lk(b1, b2);
  cudaStream_t st = b1->stream;
  EDK_TRY_CUDA(cudaStreamSynchronize(b2->stream));
  const size_t vb = (size_t)b2->D * (vdtype == EDK_C128 ? 16 : 8), ob = (size_t)b1->D * 16;
  DevBuf dv, dout;
  const void* v_d = v;
  double2* o_d = reinterpret_cast<double2*>(out);
  if (ptr_kind == EDK_HOST) {
    if (b2->D > 0) {
      EDK_RETURN_IF(dv.alloc(vb));
      EDK_TRY_CUDA(cudaMemcpyAsync(dv.p, v, vb, cudaMemcpyHostToDevice, st));
    }
    v_d = dv.p;
    EDK_RETURN_IF(dout.alloc(ob));
    o_d = dout.as<double2>();
  }
  if (ob) EDK_TRY_CUDA(cudaMemsetAsync(o_d, 0, ob, st));
  const uint64_t nfull = 1ull << b1->L;
  if (b1->D > 0 && b2->D > 0) {
    const int g = grid_of((int64_t)nfull, 256, 148 * 32);
    if (vdtype == EDK_C128)
      k_double_map<false, true><<<g, 256, 0, st>>>(b1->dev, b2->dev, orbit_order(b1),
                                                   orbit_order(b2), v_d, o_d, nfull);
    else
      k_double_map<false, false><<<g, 256, 0, st>>>(b1->dev, b2->dev, orbit_order(b1),
                                                    orbit_order(b2), v_d, o_d, nfull);
    EDK_TRY_CUDA(cudaGetLastError());
  }
  if (ptr_kind == EDK_HOST && ob)
    EDK_TRY_CUDA(cudaMemcpyAsync(out, o_d, ob, cudaMemcpyDeviceToHost, st));
  EDK_TRY_CUDA(cudaStreamSynchronize(st));
  return EDK_OK;
}

extern "C" edk_status edk_symmetrizer(const edk_basis* b1c, const edk_basis* b2c, double* M,
                                      int32_t ptr_kind) {
  EDK_RETURN_IF(check_pair(b1c, b2c));
  edk_basis* b1 = const_cast<edk_basis*>(b1c);
  edk_basis* b2 = const_cast<edk_basis*>(b2c);
  const size_t mb = (size_t)b1->D * (size_t)b2->D * 16;
  EDK_CHECK_ARG(M != nullptr || mb == 0, "edk_symmetrizer: M is NULL");
  BasisPairLock lk(b1, b2);
  cudaStream_t st = b1->stream;
  EDK_TRY_CUDA(cudaStreamSynchronize(b2->stream));
  DevBuf dM;
  double2* m_d = reinterpret_cast<double2*>(M);
  if (ptr_kind == EDK_HOST && mb) {
    EDK_RETURN_IF(dM.alloc(mb));
    m_d = dM.as<double2>();
  }
  if (mb) {
    EDK_TRY_CUDA(cudaMemsetAsync(m_d, 0, mb, st));
    const uint64_t nfull = 1ull << b1->L;
    const int g = grid_of((int64_t)nfull, 256, 148 * 32);
    k_double_map<true, false><<<g, 256, 0, st>>>(b1->dev, b2->dev, orbit_order(b1),
                                                 orbit_order(b2), nullptr, m_d, nfull);
    EDK_TRY_CUDA(cudaGetLastError());
    if (ptr_kind == EDK_HOST) EDK_TRY_CUDA(cudaMemcpyAsync(M, m_d, mb, cudaMemcpyDeviceToHost, st));
  }
  EDK_TRY_CUDA(cudaStreamSynchronize(st));
  return EDK_OK;
}
