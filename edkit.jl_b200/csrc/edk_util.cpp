// edk_util.cpp — host helpers: error state, version, and the symmetric
// tridiagonal eigensolver used by the Lanczos and Krylov drivers
// (the role of eigen(SymTridiagonal(α, β)) in src/algorithms/TimeEvolution.jl:311-323).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "edk_internal.cuh"
#include "edk_srchash.h"

namespace edk {

static thread_local std::string g_error;

void set_error(const std::string& msg) { g_error = msg; }
const std::string& get_error() { return g_error; }

double elapsed_ms(cudaEvent_t a, cudaEvent_t b) {
  float ms = 0.f;
  cudaEventElapsedTime(&ms, a, b);
  return (double)ms;
}

// Implicit symmetric QL iteration with Wilkinson shifts on the tridiagonal
// matrix (diagonal a[0..m-1], off-diagonal b[0..m-2]).  Eigenvalues are
// returned ascending in w; when Q is non-null it receives the orthonormal
// eigenvectors as columns (column-major m x m, Q[r + c*m]), ordered like w.
// Returns 0 on success, -1 if an eigenvalue did not converge in 60 sweeps.
static int tql(int m, const double* a, const double* b, double* w, double* Q) {
  if (m <= 0) return 0;
  std::vector<double> d(a, a + m), e(m, 0.0);
  for (int i = 0; i + 1 < m; ++i) e[i] = b[i];
  if (Q) {
    std::fill(Q, Q + (size_t)m * m, 0.0);
    for (int i = 0; i < m; ++i) Q[i + (size_t)i * m] = 1.0;
  }
  const double eps = std::numeric_limits<double>::epsilon();
  for (int l = 0; l < m; ++l) {
    int iter = 0;
    while (true) {
      // find a negligible off-diagonal element e[k], k >= l
      int k = l;
      for (; k < m - 1; ++k) {
        double dd = std::fabs(d[k]) + std::fabs(d[k + 1]);
        if (std::fabs(e[k]) <= eps * dd) break;
      }
      if (k == l) break;
      if (++iter > 60) return -1;
      // Wilkinson shift from the leading 2x2 block at l
      double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
      double r = std::hypot(g, 1.0);
      g = d[k] - d[l] + e[l] / (g + (g >= 0 ? r : -r));
      double s = 1.0, c = 1.0, p = 0.0;
      int i = k - 1;
      bool deflated = false;
      for (; i >= l; --i) {
        double f = s * e[i], h = c * e[i];
        r = std::hypot(f, g);
        e[i + 1] = r;
        if (r == 0.0) {  // split: recover and restart the sweep
          d[i + 1] -= p;
          e[k] = 0.0;
          deflated = true;
          break;
        }
        s = f / r;
        c = g / r;
        g = d[i + 1] - p;
        r = (d[i] - g) * s + 2.0 * c * h;
        p = s * r;
        d[i + 1] = g + p;
        g = c * r - h;
        if (Q) {
          for (int q = 0; q < m; ++q) {
            double* col1 = Q + (size_t)(i + 1) * m;
            double* col0 = Q + (size_t)i * m;
            double t = col1[q];
            col1[q] = s * col0[q] + c * t;
            col0[q] = c * col0[q] - s * t;
          }
        }
      }
      if (deflated && i >= l) continue;
      d[l] -= p;
      e[l] = g;
      e[k] = 0.0;
    }
  }
  // sort ascending (selection sort keeps vectors in step)
  std::vector<int> idx(m);
  for (int i = 0; i < m; ++i) idx[i] = i;
  std::sort(idx.begin(), idx.end(), [&](int x, int y) { return d[x] < d[y]; });
  for (int i = 0; i < m; ++i) w[i] = d[idx[i]];
  if (Q) {
    std::vector<double> T((size_t)m * m);
    for (int c = 0; c < m; ++c)
      for (int r = 0; r < m; ++r) T[r + (size_t)c * m] = Q[r + (size_t)idx[c] * m];
    std::copy(T.begin(), T.end(), Q);
  }
  return 0;
}

int tridiag_eigvals(int m, const double* a, const double* b, double* w) {
  return tql(m, a, b, w, nullptr);
}
int tridiag_eigen(int m, const double* a, const double* b, double* w, double* Q) {
  return tql(m, a, b, w, Q);
}

}  // namespace edk

extern "C" const char* edk_last_error(void) { return edk::get_error().c_str(); }
extern "C" const char* edk_version(void) { return "edk-b200 0.1.0 (sm_100a) src " EDK_SRC_HASH; }

// exported for tests of the host eigensolver
extern "C" int edk_tridiag_eigen(int m, const double* a, const double* b, double* w, double* Q) {
  return edk::tridiag_eigen(m, a, b, w, Q);
}
