// edk_block.cu — block Lanczos over a batch of operators (momentum sectors of
// one chain), each with a block of p right-hand-side vectors.
//
// EDKit's Krylov loop (_lanczos_build!, src/algorithms/TimeEvolution.jl:250-306)
// advances one vector.  The block form advances p vectors per operator:
//
//   W = H V_j;  W -= V_j A_j + V_{j-1} C  (one classical block Gram-Schmidt
//   pass against the two previous blocks); W = V_{j+1} B_{j+1} by
//   Cholesky-QR, twice.
//
// and the lowest eigenvalues come from the Hermitian block-tridiagonal
// T = tridiag(B_j, A_j, B_j^H) of order p*steps.  No global
// re-orthogonalisation is done (the Krylov blocks of 26 sectors x 100 steps
// x 64 vectors would not fit in HBM), so converged eigenvalues recur in T as
// numerically identical copies; the eigenvalues of T are extracted by a
// single-vector Lanczos with full re-orthogonalisation on T itself, which sees
// each such cluster once (distinct eigenvalues).
//
// Layout: one "slot" holds the blocks of every operator, operator q at
// q * Dpad * p, row-major D x p (row i, vector c at i * p + c), rows past D_q
// zero.  Read as column-major p x Dpad matrices (ld = p) these are what the
// strided-batched cuBLAS ZGEMMs consume: the K = D reductions are split in
// chunks of Kc rows (one batch entry each) and the partial p x p products
// summed by a kernel.  H V is this file's own SpMM: one warp per row, the
// row's off-diagonal hits found by different lanes, then every hit applied to
// the p vectors with the lanes spread over the vectors (coalesced p x 16-byte
// row gathers).
#include <cublas_v2.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstring>
#include <thread>
#include <vector>

#include "edk_spmm.cuh"

namespace edk {

namespace {

using cplx = std::complex<double>;

double wall_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

// row-major D x p <-> column-major D x p (ld = D), for operators on the
// generic column kernels
__global__ void k_rows_to_cols(const double2* __restrict__ src, double2* __restrict__ dst,
                               int64_t D, int p) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < D * p;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = e / p;
    const int c = (int)(e - i * p);
    dst[(int64_t)c * D + i] = src[e];
  }
}
__global__ void k_cols_to_rows(const double2* __restrict__ src, double2* __restrict__ dst,
                               int64_t D, int p) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < D * p;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = e / p;
    const int c = (int)(e - i * p);
    dst[e] = src[(int64_t)c * D + i];
  }
}

// ---------------------------------------------------------------------------
// small dense kernels
// ---------------------------------------------------------------------------
// out[q] = sum over S chunks of part[q * S + s] (p x p each)
__global__ void k_sum_chunks(const double2* __restrict__ part, double2* __restrict__ out,
                             int nops, int S, int pp) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < (int64_t)nops * pp;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int q = (int)(e / pp);
    const int k = (int)(e - (int64_t)q * pp);
    double sr = 0.0, si = 0.0;
    const double2* src = part + (int64_t)q * S * pp + k;
    for (int s = 0; s < S; ++s) {
      const double2 v = src[(int64_t)s * pp];
      sr += v.x;
      si += v.y;
    }
    out[e] = make_double2(sr, si);
  }
}

// splitmix64 finaliser: a counter-based stream of 64-bit words
__device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z += 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

// seeded start blocks: real and imaginary parts N(0, 1) (Box-Muller on two
// 53-bit uniforms drawn from the counter (seed, operator, row, vector))
__global__ void k_seed_blocks(const SpmmOp* __restrict__ ops, int nops, int64_t Dpad, int p,
                              uint64_t seed, double2* __restrict__ X) {
  const int64_t total = (int64_t)nops * Dpad * p;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t g = e / p;
    const int c = (int)(e - g * p);
    const int q = (int)(g / Dpad);
    const int64_t i = g - (int64_t)q * Dpad;
    if (i >= ops[q].D) { X[e] = make_double2(0.0, 0.0); continue; }
    const uint64_t key = mix64(seed ^ mix64(((uint64_t)q << 40) ^ ((uint64_t)i << 8) ^ (uint64_t)c));
    const uint64_t k2 = mix64(key);
    const double u1 = ((double)(key >> 11) + 1.0) * (1.0 / 9007199254740992.0);  // (0, 1]
    const double u2 = (double)(k2 >> 11) * (1.0 / 9007199254740992.0);          // [0, 1)
    const double r = sqrt(-2.0 * log(u1));
    double sn, cs;
    sincospi(2.0 * u2, &sn, &cs);
    X[e] = make_double2(r * cs, r * sn);
  }
}

// One block per operator: Cholesky of the Gram matrix G = conj(Gt) (Gt is
// the column-major p x p product S_W S_W^H), G = R^H R with R upper
// triangular; writes R^{-1} (column-major) for the next GEMM and, when
// `round` is 2, B = R * Rprev.  A pivot below tiny * max diag marks a
// rank-deficient block: the operator's Krylov space is exhausted, flag[q] is
// set and R = I so the slot stays finite.
__global__ void __launch_bounds__(256) k_chol(const double2* __restrict__ Gt, int p,
                                              double2* __restrict__ Rinv, double2* __restrict__ Rm,
                                              const double2* __restrict__ Rprev,
                                              double2* __restrict__ Bout, int* __restrict__ flag,
                                              int round) {
  extern __shared__ double2 sm[];
  double2* G = sm;           // p x p, row-major G[a * p + c]
  double2* R = sm + p * p;   // p x p upper, row-major
  double2* Ri = R + p * p;   // inverse, row-major
  __shared__ int bad;
  __shared__ double gmax;
  const int q = blockIdx.x;
  const int pp = p * p;
  const double2* gt = Gt + (int64_t)q * pp;
  for (int e = threadIdx.x; e < pp; e += blockDim.x) {
    const int a = e / p, c = e % p;
    const double2 v = gt[a + c * p];  // Gt(a, c)
    G[e] = make_double2(v.x, -v.y);   // G(a, c) = conj(Gt(a, c))
    R[e] = make_double2(0.0, 0.0);
    Ri[e] = make_double2(0.0, 0.0);
  }
  if (threadIdx.x == 0) {
    bad = 0;
    double m = 0.0;
    for (int a = 0; a < p; ++a) m = fmax(m, G[a * p + a].x);
    gmax = m;
  }
  __syncthreads();
  for (int k = 0; k < p; ++k) {
    const double dkk = G[k * p + k].x;
    if (!(dkk > 1e-26 * gmax) || !(gmax > 0.0)) {
      if (threadIdx.x == 0) bad = 1;
    }
    __syncthreads();
    if (bad) break;
    const double rkk = sqrt(dkk);
    for (int c = k + threadIdx.x; c < p; c += blockDim.x) {
      const double2 g = G[k * p + c];
      R[k * p + c] = c == k ? make_double2(rkk, 0.0) : make_double2(g.x / rkk, g.y / rkk);
    }
    __syncthreads();
    // trailing update: G(a, c) -= conj(R(k, a)) R(k, c), a, c > k
    const int n = p - k - 1;
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
      const int a = k + 1 + e / n, c = k + 1 + e % n;
      const double2 ra = R[k * p + a], rc = R[k * p + c];
      G[a * p + c].x -= ra.x * rc.x + ra.y * rc.y;
      G[a * p + c].y -= ra.x * rc.y - ra.y * rc.x;
    }
    __syncthreads();
  }
  if (bad) {
    for (int e = threadIdx.x; e < pp; e += blockDim.x) {
      const int a = e / p, c = e % p;
      R[e] = make_double2(a == c ? 1.0 : 0.0, 0.0);
      Ri[e] = R[e];
    }
    if (threadIdx.x == 0) flag[q] = 1;
    __syncthreads();
  } else {
    // R^{-1} column by column: R Ri(:, c) = e_c, back substitution
    for (int c = threadIdx.x; c < p; c += blockDim.x) {
      for (int a = c; a >= 0; --a) {
        double sr = (a == c) ? 1.0 : 0.0, si = 0.0;
        for (int t = a + 1; t <= c; ++t) {
          const double2 r = R[a * p + t], x = Ri[t * p + c];
          sr -= r.x * x.x - r.y * x.y;
          si -= r.x * x.y + r.y * x.x;
        }
        const double2 raa = R[a * p + a];  // real
        Ri[a * p + c] = make_double2(sr / raa.x, si / raa.x);
      }
    }
    __syncthreads();
  }
  double2* ri = Rinv + (int64_t)q * pp;
  double2* rm = Rm + (int64_t)q * pp;
  for (int e = threadIdx.x; e < pp; e += blockDim.x) {
    const int a = e / p, c = e % p;
    ri[a + c * p] = Ri[e];
    rm[a + c * p] = R[e];
  }
  if (round == 2) {
    // B = R * Rprev (both upper, column-major in global)
    const double2* rp = Rprev + (int64_t)q * pp;
    double2* bo = Bout + (int64_t)q * pp;
    for (int e = threadIdx.x; e < pp; e += blockDim.x) {
      const int a = e / p, c = e % p;
      double sr = 0.0, si = 0.0;
      for (int t = a; t <= c; ++t) {
        const double2 x = R[a * p + t], y = rp[t + c * p];
        sr += x.x * y.x - x.y * y.y;
        si += x.x * y.y + x.y * y.x;
      }
      bo[a + c * p] = make_double2(sr, si);
    }
  }
}

int grid_for(int64_t n, int cap = 148 * 16) {
  int64_t g = (n + 255) / 256;
  return (int)std::max<int64_t>(1, std::min<int64_t>(g, cap));
}

const char* cublas_msg(cublasStatus_t s) {
  switch (s) {
    case CUBLAS_STATUS_NOT_INITIALIZED: return "not initialized";
    case CUBLAS_STATUS_ALLOC_FAILED: return "allocation failed";
    case CUBLAS_STATUS_INVALID_VALUE: return "invalid value";
    case CUBLAS_STATUS_EXECUTION_FAILED: return "execution failed";
    default: return "error";
  }
}

#define EDK_TRY_BLAS(call)                                                          \
  do {                                                                              \
    cublasStatus_t s_ = (call);                                                     \
    if (s_ != CUBLAS_STATUS_SUCCESS) {                                              \
      set_error(std::string(#call) + " failed: cuBLAS " + cublas_msg(s_));          \
      return EDK_CUDA_ERROR;                                                        \
    }                                                                               \
  } while (0)

struct BlasHandle {
  cublasHandle_t h = nullptr;
  ~BlasHandle() { if (h) cublasDestroy(h); }
};

// ---------------------------------------------------------------------------
// eigenvalues of the block-tridiagonal T (host)
// ---------------------------------------------------------------------------
// T of `m` blocks: A[j] (p x p, T(j, j)), B[j] for j >= 1 (T(j, j-1)); both
// column-major complex (interleaved re, im).  Lowest `nev` distinct
// eigenvalues by Lanczos with full (twice classical Gram-Schmidt)
// re-orthogonalisation on T.  Plain real arithmetic throughout (no
// std::complex operators in the loops).
void band_candidates(const std::vector<const double*>& A, const std::vector<const double*>& B,
                     int p, int m, int nev, std::vector<double>& out) {
  const int n = p * m;
  // y = T x (x, y interleaved complex of length n)
  auto matvec = [&](const double* x, double* y) {
    for (int j = 0; j < m; ++j) {
      double* yj = y + 2 * (size_t)j * p;
      const double* xj = x + 2 * (size_t)j * p;
      for (int a = 0; a < 2 * p; ++a) yj[a] = 0.0;
      for (int c = 0; c < p; ++c) {
        const double xr = xj[2 * c], xi = xj[2 * c + 1];
        const double* col = A[j] + 2 * (size_t)c * p;
        for (int a = 0; a < p; ++a) {
          yj[2 * a] += col[2 * a] * xr - col[2 * a + 1] * xi;
          yj[2 * a + 1] += col[2 * a] * xi + col[2 * a + 1] * xr;
        }
      }
      if (j >= 1) {  // + B_j x_{j-1}
        const double* xp = x + 2 * (size_t)(j - 1) * p;
        for (int c = 0; c < p; ++c) {
          const double xr = xp[2 * c], xi = xp[2 * c + 1];
          const double* col = B[j] + 2 * (size_t)c * p;
          for (int a = 0; a < p; ++a) {
            yj[2 * a] += col[2 * a] * xr - col[2 * a + 1] * xi;
            yj[2 * a + 1] += col[2 * a] * xi + col[2 * a + 1] * xr;
          }
        }
      }
      if (j + 1 < m) {  // + B_{j+1}^H x_{j+1}
        const double* xn = x + 2 * (size_t)(j + 1) * p;
        for (int a = 0; a < p; ++a) {
          const double* col = B[j + 1] + 2 * (size_t)a * p;  // B(:, a)
          double sr = 0.0, si = 0.0;
          for (int c = 0; c < p; ++c) {  // conj(B(c, a)) * x_c
            sr += col[2 * c] * xn[2 * c] + col[2 * c + 1] * xn[2 * c + 1];
            si += col[2 * c] * xn[2 * c + 1] - col[2 * c + 1] * xn[2 * c];
          }
          yj[2 * a] += sr;
          yj[2 * a + 1] += si;
        }
      }
    }
  };
  const int mmax = std::min(n, 1200);
  std::vector<double> V(2 * (size_t)n * (mmax + 1)), w(2 * (size_t)n);
  std::vector<double> al, be;
  uint64_t st = 0x12345678abcdefull;
  auto rnd = [&]() {
    st ^= st << 13; st ^= st >> 7; st ^= st << 17;
    return ((st >> 11) * (1.0 / 9007199254740992.0)) - 0.5;
  };
  double nr = 0.0;
  for (int i = 0; i < 2 * n; ++i) { V[i] = rnd(); nr += V[i] * V[i]; }
  nr = std::sqrt(nr);
  for (int i = 0; i < 2 * n; ++i) V[i] /= nr;
  std::vector<double> prev, ev;
  out.assign(nev, NAN);
  for (int j = 0; j < mmax; ++j) {
    const double* vj = V.data() + 2 * (size_t)j * n;
    matvec(vj, w.data());
    double a = 0.0;
    for (int i = 0; i < n; ++i) a += vj[2 * i] * w[2 * i] + vj[2 * i + 1] * w[2 * i + 1];
    al.push_back(a);
    for (int pass = 0; pass < 2; ++pass) {
      for (int k = 0; k <= j; ++k) {
        const double* vk = V.data() + 2 * (size_t)k * n;
        double sr = 0.0, si = 0.0;  // vk^H w
        for (int i = 0; i < n; ++i) {
          sr += vk[2 * i] * w[2 * i] + vk[2 * i + 1] * w[2 * i + 1];
          si += vk[2 * i] * w[2 * i + 1] - vk[2 * i + 1] * w[2 * i];
        }
        for (int i = 0; i < n; ++i) {
          w[2 * i] -= sr * vk[2 * i] - si * vk[2 * i + 1];
          w[2 * i + 1] -= sr * vk[2 * i + 1] + si * vk[2 * i];
        }
      }
    }
    double b = 0.0;
    for (int i = 0; i < 2 * n; ++i) b += w[i] * w[i];
    b = std::sqrt(b);
    const bool last = (j + 1 == mmax) || b < 1e-12 * std::max(1.0, std::fabs(a));
    if (last || (j + 1) % 10 == 0) {
      const int mm = j + 1;
      ev.resize(mm);
      tridiag_eigvals(mm, al.data(), be.data(), ev.data());
      // distinct values: clusters closer than 1e-12 relative merge
      std::vector<double> d;
      for (double x : ev)
        if (d.empty() || x - d.back() > 1e-12 * std::max(1.0, std::fabs(x))) d.push_back(x);
      bool conv = last;
      if (!conv && (int)d.size() >= nev && (int)prev.size() >= nev) {
        conv = true;
        for (int k = 0; k < nev; ++k)
          if (std::fabs(d[k] - prev[k]) > 1e-13 * std::max(1.0, std::fabs(d[0]))) conv = false;
      }
      prev = d;
      if (conv) break;
    }
    be.push_back(b);
    double* vn = V.data() + 2 * (size_t)(j + 1) * n;
    for (int i = 0; i < 2 * n; ++i) vn[i] = w[i] / b;
  }
  out.assign(prev.begin(), prev.begin() + std::min<size_t>(prev.size(), (size_t)nev));
}

// Number of eigenvalues below sigma of the block-tridiagonal matrix made of
// blocks j0..m-1 (Sylvester inertia of its block LDL^H factorisation:
// M_j = A_j - sigma - B_j M_{j-1}^{-1} B_j^H, each M_j by unpivoted LDL^H).
int sturm_count(const std::vector<const double*>& A, const std::vector<const double*>& B,
                int p, int m, int j0, double sigma) {
  std::vector<double> M(2 * (size_t)p * p), L(2 * (size_t)p * p), dg(p), X(2 * (size_t)p * p);
  double scale = 1.0;
  for (int j = j0; j < m; ++j)
    for (int a = 0; a < p; ++a) scale = std::max(scale, std::fabs(A[j][2 * ((size_t)a * p + a)]));
  const double tiny = 1e-300 + 1e-15 * scale;
  int neg = 0;
  bool have_x = false;
  for (int j = j0; j < m; ++j) {
    // M = A_j - sigma I (column-major complex)
    for (size_t e = 0; e < 2 * (size_t)p * p; ++e) M[e] = A[j][e];
    for (int a = 0; a < p; ++a) M[2 * ((size_t)a * p + a)] -= sigma;
    if (have_x) {  // M -= B_j X,  X = M_{j-1}^{-1} B_j^H
      const double* Bj = B[j];
      for (int c = 0; c < p; ++c)
        for (int t = 0; t < p; ++t) {
          const double xr = X[2 * ((size_t)c * p + t)], xi = X[2 * ((size_t)c * p + t) + 1];
          const double* bt = Bj + 2 * (size_t)t * p;  // column t of B_j
          double* mc = M.data() + 2 * (size_t)c * p;
          for (int a = 0; a < p; ++a) {
            mc[2 * a] -= bt[2 * a] * xr - bt[2 * a + 1] * xi;
            mc[2 * a + 1] -= bt[2 * a] * xi + bt[2 * a + 1] * xr;
          }
        }
    }
    // unpivoted LDL^H: M = L diag(dg) L^H, L unit lower (column-major)
    for (int k = 0; k < p; ++k) {
      double dk = M[2 * ((size_t)k * p + k)];
      for (int t = 0; t < k; ++t) {
        const double lr = L[2 * ((size_t)t * p + k)], li = L[2 * ((size_t)t * p + k) + 1];
        dk -= (lr * lr + li * li) * dg[t];
      }
      if (std::fabs(dk) < tiny) dk = dk < 0 ? -tiny : tiny;
      dg[k] = dk;
      if (dk < 0) ++neg;
      L[2 * ((size_t)k * p + k)] = 1.0;
      L[2 * ((size_t)k * p + k) + 1] = 0.0;
      for (int i = k + 1; i < p; ++i) {
        double sr = M[2 * ((size_t)k * p + i)], si = M[2 * ((size_t)k * p + i) + 1];  // M(i, k)
        for (int t = 0; t < k; ++t) {  // - L(i,t) conj(L(k,t)) d_t
          const double ar = L[2 * ((size_t)t * p + i)], ai = L[2 * ((size_t)t * p + i) + 1];
          const double br = L[2 * ((size_t)t * p + k)], bi = L[2 * ((size_t)t * p + k) + 1];
          sr -= (ar * br + ai * bi) * dg[t];
          si -= (ai * br - ar * bi) * dg[t];
        }
        L[2 * ((size_t)k * p + i)] = sr / dk;
        L[2 * ((size_t)k * p + i) + 1] = si / dk;
      }
    }
    if (j + 1 < m) {
      // X = M^{-1} B_{j+1}^H, column c of B^H = conj(row c of B)
      const double* Bn = B[j + 1];
      for (int c = 0; c < p; ++c) {
        double* x = X.data() + 2 * (size_t)c * p;
        for (int a = 0; a < p; ++a) {  // rhs(a) = conj(B(c, a))
          x[2 * a] = Bn[2 * ((size_t)a * p + c)];
          x[2 * a + 1] = -Bn[2 * ((size_t)a * p + c) + 1];
        }
        for (int a = 0; a < p; ++a)  // L y = rhs
          for (int t = 0; t < a; ++t) {
            const double lr = L[2 * ((size_t)t * p + a)], li = L[2 * ((size_t)t * p + a) + 1];
            x[2 * a] -= lr * x[2 * t] - li * x[2 * t + 1];
            x[2 * a + 1] -= lr * x[2 * t + 1] + li * x[2 * t];
          }
        for (int a = 0; a < p; ++a) { x[2 * a] /= dg[a]; x[2 * a + 1] /= dg[a]; }
        for (int a = p - 1; a >= 0; --a)  // L^H z = y
          for (int t = a + 1; t < p; ++t) {
            const double lr = L[2 * ((size_t)a * p + t)], li = -L[2 * ((size_t)a * p + t) + 1];
            x[2 * a] -= lr * x[2 * t] - li * x[2 * t + 1];
            x[2 * a + 1] -= lr * x[2 * t + 1] + li * x[2 * t];
          }
      }
      have_x = true;
    }
  }
  return neg;
}

// Lowest `nev` distinct eigenvalues of the operator from T: candidates from
// the Lanczos on T, each kept only when it is a genuine eigenvalue in the
// Cullum-Willoughby sense generalised to blocks — the number of copies T has
// in a small window around it exceeds the number T-hat (T without its first
// block row and column) has there.  Copies that arise from the loss of
// orthogonality (converged values repeated, or still converging towards
// them) are eigenvalues of T-hat as well.
void band_lowest(const std::vector<const double*>& A, const std::vector<const double*>& B,
                 int p, int m, int nev, std::vector<double>& out) {
  std::vector<double> cand;
  band_candidates(A, B, p, m, nev + 4, cand);
  out.assign(nev, NAN);
  int got = 0;
  // candidates closer than the window merge into one cluster, counted once
  for (size_t c = 0; c < cand.size() && got < nev;) {
    const double lo = cand[c];
    const double dl = 1e-10 * std::max(1.0, std::fabs(lo));
    double hi = lo;
    size_t e = c + 1;
    while (e < cand.size() && cand[e] - hi <= dl) hi = cand[e++];
    const int nt = sturm_count(A, B, p, m, 0, hi + dl) - sturm_count(A, B, p, m, 0, lo - dl);
    const int nh =
        m > 1 ? sturm_count(A, B, p, m, 1, hi + dl) - sturm_count(A, B, p, m, 1, lo - dl) : 0;
    if (nt - nh >= 1) out[got++] = lo;
    c = e;
  }
}

}  // namespace

// ---------------------------------------------------------------------------
// the engine
// ---------------------------------------------------------------------------
static edk_status block_lanczos(int nops, edk_operator* const* ops,
                                const edk_block_lanczos_opts& o, const double* x0,
                                double* evals, edk_block_lanczos_diag* diag) {
  const double t_start = wall_s();
  const int p = o.block;
  const int pp = p * p;
  cudaStream_t st = ops[0]->stream;
  int64_t Dmax = 0;
  for (int q = 0; q < nops; ++q) Dmax = std::max<int64_t>(Dmax, ops[q]->b->D);
  const int64_t Kc = std::min<int64_t>(2048, ((Dmax + 31) / 32) * 32);
  const int64_t S = (Dmax + Kc - 1) / Kc;
  const int64_t Dpad = S * Kc;
  const size_t slot = (size_t)nops * Dpad * p;

  // operator table
  std::vector<SpmmOp> hops(nops);
  bool any_generic = false;
  int64_t smax = 0;
  int bk_ff = -1;
  for (int q = 0; q < nops; ++q) {
    EDK_RETURN_IF(check_basis_dev(ops[q]->b->dev));
    int bk;
    int64_t slots;
    const int kind = spmm_describe(ops[q], hops[q], bk, slots);
    if (kind == 1) smax = std::max<int64_t>(smax, slots);
    if (kind == 2) any_generic = true;
    if (kind == 0) {
      if (bk_ff >= 0 && bk_ff != bk) {
        set_error("edk_block_lanczos: operators on different kinds of basis in one batch");
        return EDK_UNSUPPORTED;
      }
      bk_ff = bk;
    }
  }

  DevBuf d_ops, ring0, ring1, ring2, part, Q1, Q2, G, Rinv, R1, R2, Bm, flags, colx, coly;
  EDK_RETURN_IF(d_ops.alloc(sizeof(SpmmOp) * nops));
  EDK_RETURN_IF(ring0.alloc(slot * sizeof(double2)));
  EDK_RETURN_IF(ring1.alloc(slot * sizeof(double2)));
  EDK_RETURN_IF(ring2.alloc(slot * sizeof(double2)));
  EDK_RETURN_IF(part.alloc((size_t)nops * S * pp * sizeof(double2)));
  for (DevBuf* bf : {&Q1, &Q2, &G, &Rinv, &R1, &R2, &Bm})
    EDK_RETURN_IF(bf->alloc((size_t)nops * pp * sizeof(double2)));
  EDK_RETURN_IF(flags.alloc(nops * sizeof(int)));
  if (any_generic) {
    EDK_RETURN_IF(colx.alloc((size_t)Dmax * p * sizeof(double2)));
    EDK_RETURN_IF(coly.alloc((size_t)Dmax * p * sizeof(double2)));
  }
  EDK_TRY_CUDA(cudaMemcpyAsync(d_ops.p, hops.data(), sizeof(SpmmOp) * nops,
                               cudaMemcpyHostToDevice, st));
  EDK_TRY_CUDA(cudaMemsetAsync(flags.p, 0, nops * sizeof(int), st));
  for (DevBuf* bf : {&ring0, &ring1, &ring2})
    EDK_TRY_CUDA(cudaMemsetAsync(bf->p, 0, slot * sizeof(double2), st));
  double2* U = ring0.as<double2>();
  double2* V = ring1.as<double2>();
  double2* W = ring2.as<double2>();

  BlasHandle bh;
  EDK_TRY_BLAS(cublasCreate(&bh.h));
  EDK_TRY_BLAS(cublasSetStream(bh.h, st));
  EDK_TRY_BLAS(cublasSetPointerMode(bh.h, CUBLAS_POINTER_MODE_HOST));
  const cuDoubleComplex one = make_cuDoubleComplex(1.0, 0.0);
  const cuDoubleComplex mone = make_cuDoubleComplex(-1.0, 0.0);
  const cuDoubleComplex zero = make_cuDoubleComplex(0.0, 0.0);
  auto C = [](double2* x) { return reinterpret_cast<cuDoubleComplex*>(x); };

  // out = sum over rows of X Y^H per operator (p x p, column-major): the
  // split-K strided batch plus the chunk sum
  auto gram = [&](const double2* Xs, const double2* Ys, double2* out) -> edk_status {
    EDK_TRY_BLAS(cublasZgemmStridedBatched(
        bh.h, CUBLAS_OP_N, CUBLAS_OP_C, p, p, (int)Kc, &one,
        reinterpret_cast<const cuDoubleComplex*>(Xs), p, Kc * p,
        reinterpret_cast<const cuDoubleComplex*>(Ys), p, Kc * p, &zero, C(part.as<double2>()), p,
        pp, (int)(nops * S)));
    k_sum_chunks<<<grid_for((int64_t)nops * pp), 256, 0, st>>>(part.as<double2>(), out, nops,
                                                                (int)S, pp);
    EDK_TRY_CUDA(cudaGetLastError());
    return EDK_OK;
  };
  // Ws -= Qm Xs per operator (Qm p x p)
  auto update = [&](const double2* Qm, const double2* Xs, double2* Ws) -> edk_status {
    EDK_TRY_BLAS(cublasZgemmStridedBatched(
        bh.h, CUBLAS_OP_N, CUBLAS_OP_N, p, (int)Dpad, p, &mone,
        reinterpret_cast<const cuDoubleComplex*>(Qm), p, pp,
        reinterpret_cast<const cuDoubleComplex*>(Xs), p, Dpad * p, &one, C(Ws), p, Dpad * p,
        nops));
    return EDK_OK;
  };
  // Out = Rinv^T In per operator
  auto rmul = [&](const double2* In, double2* Out) -> edk_status {
    EDK_TRY_BLAS(cublasZgemmStridedBatched(
        bh.h, CUBLAS_OP_T, CUBLAS_OP_N, p, (int)Dpad, p, &one,
        reinterpret_cast<const cuDoubleComplex*>(Rinv.as<double2>()), p, pp,
        reinterpret_cast<const cuDoubleComplex*>(In), p, Dpad * p, &zero, C(Out), p, Dpad * p,
        nops));
    return EDK_OK;
  };
  const size_t chol_smem = 3 * (size_t)pp * sizeof(double2);
  EDK_TRY_CUDA(cudaFuncSetAttribute(k_chol, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)chol_smem));
  // Cholesky-QR twice: X (in slot W) = Q B; Q lands back in W, `spare` is
  // overwritten; B in Bm
  auto cholqr = [&](double2* Wx, double2* spare) -> edk_status {
    EDK_RETURN_IF(gram(Wx, Wx, G.as<double2>()));
    k_chol<<<nops, 256, chol_smem, st>>>(G.as<double2>(), p, Rinv.as<double2>(),
                                         R1.as<double2>(), nullptr, nullptr, flags.as<int>(), 1);
    EDK_TRY_CUDA(cudaGetLastError());
    EDK_RETURN_IF(rmul(Wx, spare));
    EDK_RETURN_IF(gram(spare, spare, G.as<double2>()));
    k_chol<<<nops, 256, chol_smem, st>>>(G.as<double2>(), p, Rinv.as<double2>(),
                                         R2.as<double2>(), R1.as<double2>(), Bm.as<double2>(),
                                         flags.as<int>(), 2);
    EDK_TRY_CUDA(cudaGetLastError());
    EDK_RETURN_IF(rmul(spare, Wx));
    return EDK_OK;
  };

  float t_spmm = 0.f, t_orth = 0.f;
  cudaEvent_t e0, e1, e2;
  EDK_TRY_CUDA(cudaEventCreate(&e0));
  EDK_TRY_CUDA(cudaEventCreate(&e1));
  EDK_TRY_CUDA(cudaEventCreate(&e2));
  struct EvGuard {
    cudaEvent_t a, b, c;
    ~EvGuard() { cudaEventDestroy(a); cudaEventDestroy(b); cudaEventDestroy(c); }
  } evg{e0, e1, e2};

  auto spmm = [&](const double2* X, double2* Y) -> edk_status {
    EDK_RETURN_IF(launch_spmm<double2>(d_ops.as<SpmmOp>(), nops, bk_ff, smax, Dpad, p, X, Y, 0,
                                       st));
    if (any_generic) {
      for (int q = 0; q < nops; ++q) {
        if (hops[q].kind != 2) continue;
        const int64_t D = hops[q].D;
        const double2* xq = X + (size_t)q * Dpad * p;
        double2* yq = Y + (size_t)q * Dpad * p;
        k_rows_to_cols<<<grid_for(D * p), 256, 0, st>>>(xq, colx.as<double2>(), D, p);
        EDK_TRY_CUDA(cudaGetLastError());
        EDK_RETURN_IF(apply_device(ops[q], EDK_C128, colx.p, coly.p, p, D, D, 0, st));
        k_cols_to_rows<<<grid_for(D * p), 256, 0, st>>>(coly.as<double2>(), yq, D, p);
        EDK_TRY_CUDA(cudaGetLastError());
      }
    }
    return EDK_OK;
  };

  // start blocks into W, orthonormalised into V
  if (x0) {
    // host column-major D_q x p per operator, concatenated
    std::vector<double2> rows;
    size_t off = 0;
    for (int q = 0; q < nops; ++q) {
      const int64_t D = hops[q].D;
      rows.assign((size_t)D * p, make_double2(0.0, 0.0));
      for (int c = 0; c < p; ++c)
        for (int64_t i = 0; i < D; ++i) {
          const double* s = x0 + 2 * (off + (size_t)c * D + i);
          rows[(size_t)i * p + c] = make_double2(s[0], s[1]);
        }
      off += (size_t)D * p;
      EDK_TRY_CUDA(cudaMemcpyAsync(W + (size_t)q * Dpad * p, rows.data(),
                                   rows.size() * sizeof(double2), cudaMemcpyHostToDevice, st));
      EDK_TRY_CUDA(cudaStreamSynchronize(st));
    }
  } else {
    k_seed_blocks<<<grid_for((int64_t)nops * Dpad * p), 256, 0, st>>>(d_ops.as<SpmmOp>(), nops,
                                                                      Dpad, p, o.seed, W);
    EDK_TRY_CUDA(cudaGetLastError());
  }
  EDK_RETURN_IF(cholqr(W, U));
  std::swap(V, W);  // V = V_1; U (zero rows not needed: j = 1 skips it)

  // per step host copies: A and B
  const int m = o.max_steps;
  std::vector<cplx> hA((size_t)m * nops * pp),
      hB((size_t)(m + 1) * nops * pp);
  std::vector<int> hflag(nops, 0), broke_at(nops, -1);
  std::vector<double> cur((size_t)nops * o.nev, NAN), prev((size_t)nops * o.nev, NAN);
  double t_eig = 0.0;
  int steps = 0;
  bool converged = false;

  // eigenvalues of every operator's block tridiagonal T: the blocks are put
  // together on the host (threads over the operators), the eigenvalue step
  // itself runs on the device (band_lowest_device)
  std::vector<std::vector<cplx>> Aall(nops);
  auto extract = [&](int nsteps) -> edk_status {
    const double te = wall_s();
    const int nth = (int)std::max(1u, std::min<unsigned>(std::thread::hardware_concurrency(), 64));
    std::vector<std::thread> pool;
    std::vector<int> mqs(nops);
    std::vector<std::vector<const double*>> Ap(nops), Bp(nops);
    auto work = [&](int t) {
      for (int q = t; q < nops; q += nth) {
        const int mq = broke_at[q] >= 0 ? broke_at[q] : nsteps;
        mqs[q] = mq;
        Aall[q].assign((size_t)mq * pp, cplx(0.0, 0.0));
        Ap[q].assign(mq, nullptr);
        Bp[q].assign(mq, nullptr);
        for (int j = 0; j < mq; ++j) {
          cplx* Aj = Aall[q].data() + (size_t)j * pp;
          const cplx* a1 = hA.data() + ((size_t)j * nops + q) * pp;
          // device holds (V^H W)^T column-major = A row-major; make A
          // column-major and Hermitian
          for (int r = 0; r < p; ++r)
            for (int c = 0; c < p; ++c) Aj[r + (size_t)c * p] = a1[c + (size_t)r * p];
          for (int r = 0; r < p; ++r)
            for (int c = r; c < p; ++c) {
              const cplx h = 0.5 * (Aj[r + (size_t)c * p] + std::conj(Aj[c + (size_t)r * p]));
              Aj[r + (size_t)c * p] = h;
              Aj[c + (size_t)r * p] = std::conj(h);
            }
          Ap[q][j] = reinterpret_cast<const double*>(Aj);
          if (j >= 1) Bp[q][j] = reinterpret_cast<const double*>(hB.data() + ((size_t)j * nops + q) * pp);
        }
      }
    };
    for (int t = 0; t < nth; ++t) pool.emplace_back(work, t);
    for (auto& th : pool) th.join();
    std::vector<std::vector<double>> res;
    EDK_RETURN_IF(band_lowest_device(p, o.nev, mqs, Ap, Bp, st, res));
    for (int q = 0; q < nops; ++q)
      for (int k = 0; k < o.nev; ++k) cur[(size_t)q * o.nev + k] = res[q][k];
    t_eig += wall_s() - te;
    return EDK_OK;
  };

  for (int j = 0; j < m; ++j) {
    EDK_TRY_CUDA(cudaEventRecord(e0, st));
    EDK_RETURN_IF(spmm(V, W));
    EDK_TRY_CUDA(cudaEventRecord(e1, st));
    // one classical block Gram-Schmidt pass against V_j and V_{j-1}; the
    // Cholesky-QR below runs twice
    EDK_RETURN_IF(gram(W, V, Q1.as<double2>()));
    if (j > 0) EDK_RETURN_IF(gram(W, U, Q2.as<double2>()));
    EDK_RETURN_IF(update(Q1.as<double2>(), V, W));
    if (j > 0) EDK_RETURN_IF(update(Q2.as<double2>(), U, W));
    EDK_RETURN_IF(cholqr(W, U));  // U (= V_{j-1}) is free now
    EDK_TRY_CUDA(cudaEventRecord(e2, st));
    EDK_TRY_CUDA(cudaMemcpyAsync(hA.data() + (size_t)j * nops * pp, Q1.p,
                                 (size_t)nops * pp * sizeof(double2), cudaMemcpyDeviceToHost, st));
    EDK_TRY_CUDA(cudaMemcpyAsync(hB.data() + (size_t)(j + 1) * nops * pp, Bm.p,
                                 (size_t)nops * pp * sizeof(double2), cudaMemcpyDeviceToHost, st));
    EDK_TRY_CUDA(cudaMemcpyAsync(hflag.data(), flags.p, nops * sizeof(int),
                                 cudaMemcpyDeviceToHost, st));
    EDK_TRY_CUDA(cudaStreamSynchronize(st));
    float a = 0.f, c = 0.f;
    cudaEventElapsedTime(&a, e0, e1);
    cudaEventElapsedTime(&c, e1, e2);
    t_spmm += a;
    t_orth += c;
    // rotate: V_{j-1} <- V_j, V_j <- V_{j+1} (in W), spare <- old U
    double2* oldU = U;
    U = V;
    V = W;
    W = oldU;
    steps = j + 1;
    bool all_broken = true;
    for (int q = 0; q < nops; ++q) {
      // a flag raised in this step's QR: block j+1 is not part of the space
      if (hflag[q] && broke_at[q] < 0) broke_at[q] = j + 1;
      all_broken = all_broken && broke_at[q] >= 0;
    }
    const bool check = (o.check_every > 0 && (j + 1) % o.check_every == 0) || j + 1 == m ||
                       all_broken;
    if (check) {
      EDK_RETURN_IF(extract(j + 1));
      if (o.tol > 0.0 && j + 1 < m) {
        bool conv = true;
        for (int q = 0; q < nops && conv; ++q)
          for (int k = 0; k < o.nev; ++k) {
            const double a0 = cur[(size_t)q * o.nev + k], b0 = prev[(size_t)q * o.nev + k];
            if (!(std::fabs(a0 - b0) <= o.tol * std::max(1.0, std::fabs(cur[(size_t)q * o.nev]))))
              conv = false;
          }
        prev = cur;
        if (conv) { converged = true; break; }
      }
      if (all_broken) break;
    }
  }
  if (steps > 0 && std::isnan(cur[0])) EDK_RETURN_IF(extract(steps));
  std::memcpy(evals, cur.data(), cur.size() * sizeof(double));
  if (diag) {
    std::memset(diag, 0, sizeof(*diag));
    diag->steps = steps;
    diag->matvecs = (int64_t)steps * p * nops;
    int nb = 0;
    for (int q = 0; q < nops; ++q) nb += broke_at[q] >= 0;
    diag->breakdowns = nb;
    diag->converged = converged ? 1 : 0;
    diag->seconds = wall_s() - t_start;
    diag->seconds_spmm = t_spmm * 1e-3;
    diag->seconds_orth = t_orth * 1e-3;
    diag->seconds_eig = t_eig;
  }
  return EDK_OK;
}

}  // namespace edk

using namespace edk;

extern "C" edk_status edk_block_tridiag_lowest(int32_t p, int32_t m, const double* A,
                                              const double* B, int32_t nev, double* out) {
  EDK_CHECK_ARG(p >= 1 && m >= 1 && nev >= 1 && A && out && (m == 1 || B),
                "edk_block_tridiag_lowest: bad argument");
  const size_t pp = (size_t)p * p;
  std::vector<const double*> Ap(m), Bp(m, nullptr);
  for (int j = 0; j < m; ++j) {
    Ap[j] = A + 2 * pp * j;
    if (j >= 1) Bp[j] = B + 2 * pp * (j - 1);
  }
  std::vector<double> res;
  band_lowest(Ap, Bp, p, m, nev, res);
  for (int k = 0; k < nev; ++k) out[k] = k < (int)res.size() ? res[k] : NAN;
  return EDK_OK;
}

extern "C" void edk_block_lanczos_default_opts(edk_block_lanczos_opts* o) {
  if (!o) return;
  o->block = 64;
  o->max_steps = 100;
  o->nev = 4;
  o->tol = 0.0;
  o->check_every = 10;
  o->seed = 1234;
}

extern "C" edk_status edk_block_lanczos(int32_t nops, edk_operator* const* ops,
                                        const edk_block_lanczos_opts* opts, const double* x0,
                                        double* evals, edk_block_lanczos_diag* diag) {
  EDK_CHECK_ARG(nops >= 1 && ops != nullptr && opts != nullptr && evals != nullptr,
                "edk_block_lanczos: NULL argument or no operators");
  const edk_block_lanczos_opts& o = *opts;
  EDK_CHECK_ARG(o.block >= 8 && o.block <= 64 && o.block % 8 == 0,
                "edk_block_lanczos: block must be a multiple of 8 between 8 and 64");
  EDK_CHECK_ARG(o.max_steps >= 1 && o.nev >= 1, "edk_block_lanczos: max_steps and nev >= 1");
  int dev = -1;
  for (int q = 0; q < nops; ++q) {
    EDK_CHECK_ARG(ops[q] != nullptr, "edk_block_lanczos: NULL operator");
    EDK_CHECK_ARG(ops[q]->gather, "edk_block_lanczos: operators must be Hermitian and "
                                  "symmetric under the basis (row-gather form)");
    EDK_CHECK_ARG(ops[q]->b->D > 0, "edk_block_lanczos: empty basis");
    if (dev < 0) dev = ops[q]->b->device;
    EDK_CHECK_ARG(ops[q]->b->device == dev, "edk_block_lanczos: operators on different devices");
    EDK_CHECK_ARG((int64_t)o.block * o.max_steps < ops[q]->b->D,
                  "edk_block_lanczos: block * max_steps must stay below every dimension");
  }
  std::vector<std::unique_lock<std::mutex>> locks;
  for (int q = 0; q < nops; ++q) {
    bool seen = false;
    for (int r = 0; r < q; ++r) seen = seen || ops[r] == ops[q];
    if (!seen) locks.emplace_back(ops[q]->mu);
  }
  EDK_TRY_CUDA(cudaSetDevice(dev));
  return block_lanczos(nops, ops, o, x0, evals, diag);
}
