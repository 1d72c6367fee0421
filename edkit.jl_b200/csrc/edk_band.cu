// edk_band.cu — the eigenvalue step of the block Lanczos on the device: the
// lowest distinct eigenvalues of each operator's block-tridiagonal T (p x p
// Hermitian blocks A_j on the diagonal, B_j below it), found the way the host
// form in edk_block.cu finds them (band_lowest): candidates from a Lanczos on
// T with full re-orthogonalisation (classical Gram-Schmidt twice), each kept
// only when T has more eigenvalues in a small window around it than T-hat (T
// without its first block row and column) — the Cullum-Willoughby test
// generalised to blocks, with exact counts from block Sturm (inertia)
// sequences.  All operators' T run together: a Lanczos step is seven
// launches over every operator, and every Sturm count is one thread block.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "edk_internal.cuh"

namespace edk {

namespace {

constexpr int kBandSteps = 1200;  // Lanczos steps on T at most (the host form's limit)

__device__ __forceinline__ double bwsum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Shapes shared by the kernels: T_q has mq[q] blocks (at most mmax), rows
// n_q = p * mq[q] (at most nmax); A and B hold mmax blocks per operator
// (B_0 unused); V holds `vcols` columns of nmax rows per operator.
struct BandDims {
  int p, mmax, vcols;
  int64_t nmax;
};

// w = T v_k for block row jb of operator q (thread a: row a of the block)
__global__ void k_band_mv(BandDims d, const double2* __restrict__ A, const double2* __restrict__ B,
                          const int* __restrict__ mq, const double2* __restrict__ V, int k,
                          double2* __restrict__ w, const int* __restrict__ stop) {
  extern __shared__ double2 sx[];  // x_{jb-1}, x_jb, x_{jb+1}
  const int q = blockIdx.y, jb = blockIdx.x, p = d.p;
  if (stop[q] || jb >= mq[q]) return;
  const int m = mq[q];
  const double2* x = V + ((size_t)q * d.vcols + k) * d.nmax;
  const int a = threadIdx.x;
  for (int t = 0; t < 3; ++t) {
    const int jj = jb - 1 + t;
    sx[t * p + a] = (jj >= 0 && jj < m) ? x[(size_t)jj * p + a] : make_double2(0.0, 0.0);
  }
  __syncthreads();
  const size_t pp = (size_t)p * p;
  const double2* Aj = A + ((size_t)q * d.mmax + jb) * pp;
  double yr = 0.0, yi = 0.0;
  for (int c = 0; c < p; ++c) {  // A_j x_j
    const double2 v = Aj[a + (size_t)c * p], xc = sx[p + c];
    yr += v.x * xc.x - v.y * xc.y;
    yi += v.x * xc.y + v.y * xc.x;
  }
  if (jb >= 1) {  // + B_j x_{j-1}
    const double2* Bj = B + ((size_t)q * d.mmax + jb) * pp;
    for (int c = 0; c < p; ++c) {
      const double2 v = Bj[a + (size_t)c * p], xc = sx[c];
      yr += v.x * xc.x - v.y * xc.y;
      yi += v.x * xc.y + v.y * xc.x;
    }
  }
  if (jb + 1 < m) {  // + B_{j+1}^H x_{j+1}: conj(B(c, a)) x_c
    const double2* Bn = B + ((size_t)q * d.mmax + jb + 1) * pp;
    for (int c = 0; c < p; ++c) {
      const double2 v = Bn[c + (size_t)a * p], xc = sx[2 * p + c];
      yr += v.x * xc.x + v.y * xc.y;
      yi += v.x * xc.y - v.y * xc.x;
    }
  }
  w[(size_t)q * d.nmax + (size_t)jb * p + a] = make_double2(yr, yi);
}

// s[q][c] = V_q[:, c]^H w_q for c <= k: one warp per (column, operator)
__global__ void __launch_bounds__(256) k_band_dots(BandDims d, const int* __restrict__ nq,
                                                   const double2* __restrict__ V, int k,
                                                   const double2* __restrict__ w,
                                                   double2* __restrict__ s,
                                                   const int* __restrict__ stop) {
  const int q = blockIdx.y;
  const int c = blockIdx.x * 8 + (threadIdx.x >> 5);
  if (stop[q] || c > k) return;
  const int lane = threadIdx.x & 31;
  const int64_t n = nq[q];
  const double2* v = V + ((size_t)q * d.vcols + c) * d.nmax;
  const double2* x = w + (size_t)q * d.nmax;
  double sr[4] = {0.0, 0.0, 0.0, 0.0}, si[4] = {0.0, 0.0, 0.0, 0.0};
  int64_t i = lane;
  for (; i + 96 < n; i += 128) {
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const double2 a = v[i + 32 * u], b = x[i + 32 * u];
      sr[u] += a.x * b.x + a.y * b.y;
      si[u] += a.x * b.y - a.y * b.x;
    }
  }
  for (; i < n; i += 32) {
    const double2 a = v[i], b = x[i];
    sr[0] += a.x * b.x + a.y * b.y;
    si[0] += a.x * b.y - a.y * b.x;
  }
  const double r = bwsum((sr[0] + sr[1]) + (sr[2] + sr[3]));
  const double im = bwsum((si[0] + si[1]) + (si[2] + si[3]));
  if (lane == 0) s[(size_t)q * d.vcols + c] = make_double2(r, im);
}

// w_q -= V_q[:, 0:k+1] s_q (one thread per row)
__global__ void __launch_bounds__(256) k_band_update(BandDims d, const int* __restrict__ nq,
                                                     const double2* __restrict__ V, int k,
                                                     const double2* __restrict__ s,
                                                     double2* __restrict__ w,
                                                     const int* __restrict__ stop) {
  extern __shared__ double2 ss[];  // k + 1 coefficients
  const int q = blockIdx.y;
  if (stop[q]) return;
  for (int c = threadIdx.x; c <= k; c += blockDim.x) ss[c] = s[(size_t)q * d.vcols + c];
  __syncthreads();
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nq[q]) return;
  const double2* v = V + (size_t)q * d.vcols * d.nmax + i;
  double ar = 0.0, ai = 0.0;
  for (int c = 0; c <= k; ++c) {
    const double2 x = v[(size_t)c * d.nmax], t = ss[c];
    ar += x.x * t.x - x.y * t.y;
    ai += x.x * t.y + x.y * t.x;
  }
  double2* wi = w + (size_t)q * d.nmax + i;
  *wi = make_double2(wi->x - ar, wi->y - ai);
}

// alpha_k (the first sweep's s_k), beta_k = |w|, 1/beta; a negligible beta
// (the host form's rule b < 1e-12 max(1, |a|)) stops the operator with k + 1
// steps, recorded in stop[q]
__global__ void __launch_bounds__(256) k_band_norm(BandDims d, const int* __restrict__ nq, int k,
                                                   const double2* __restrict__ w,
                                                   const double2* __restrict__ s1,
                                                   double* __restrict__ alpha,
                                                   double* __restrict__ beta,
                                                   double* __restrict__ invb,
                                                   int* __restrict__ stop) {
  __shared__ double sh[8];
  const int q = blockIdx.x;
  if (stop[q]) return;
  const int64_t n = nq[q];
  const double2* x = w + (size_t)q * d.nmax;
  double t = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) t += x[i].x * x[i].x + x[i].y * x[i].y;
  t = bwsum(t);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = t;
  __syncthreads();
  if (threadIdx.x != 0) return;
  double n2 = 0.0;
  for (int u = 0; u < 8; ++u) n2 += sh[u];
  const double a = s1[(size_t)q * d.vcols + k].x, b = sqrt(n2);
  alpha[(size_t)q * d.vcols + k] = a;
  beta[(size_t)q * d.vcols + k] = b;
  if (b < 1e-12 * fmax(1.0, fabs(a))) {
    stop[q] = k + 1;
    invb[q] = 0.0;
  } else {
    invb[q] = 1.0 / b;
  }
}

// v_{k+1} = w / beta
__global__ void __launch_bounds__(256) k_band_scale(BandDims d, const int* __restrict__ nq,
                                                    int k, const double2* __restrict__ w,
                                                    const double* __restrict__ invb,
                                                    double2* __restrict__ V,
                                                    const int* __restrict__ stop) {
  const int q = blockIdx.y;
  if (stop[q] || k + 1 >= d.vcols) return;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nq[q]) return;
  const double sc = invb[q];
  const double2 x = w[(size_t)q * d.nmax + i];
  V[((size_t)q * d.vcols + k + 1) * d.nmax + i] = make_double2(x.x * sc, x.y * sc);
}

// One Sturm count: the number of eigenvalues below sigma of the
// block-tridiagonal matrix of operator q's blocks j0 .. m-1, as the sign count
// of its block LDL^H factorisation: M_j = A_j - sigma - B_j X_{j-1},
// X_{j-1} = M_{j-1}^{-1} B_j^H, each M_j factorised without pivoting (a
// pivot below `tiny` in magnitude is replaced by +-tiny, as in the host
// form).  One block of 256 threads; shared memory M, L, X (p^2 each) and the
// pivots.
struct BandTask {
  double sigma, tiny;
  int q, j0;
};

__global__ void __launch_bounds__(256) k_band_sturm(BandDims d, const double2* __restrict__ A,
                                                    const double2* __restrict__ B,
                                                    const int* __restrict__ mq,
                                                    const BandTask* __restrict__ tasks,
                                                    int* __restrict__ counts) {
  extern __shared__ double2 sm[];
  const int p = d.p;
  const int pp = p * p;
  double2* M = sm;
  double2* L = sm + pp;
  double2* X = sm + 2 * pp;
  double* dg = reinterpret_cast<double*>(sm + 3 * pp);
  __shared__ int s_neg;
  const BandTask tk = tasks[blockIdx.x];
  const int q = tk.q, m = mq[q];
  const int tid = threadIdx.x, nt = blockDim.x;
  if (tid == 0) s_neg = 0;
  bool have_x = false;
  for (int j = tk.j0; j < m; ++j) {
    const double2* Aj = A + ((size_t)q * d.mmax + j) * pp;
    for (int e = tid; e < pp; e += nt) {
      double2 v = Aj[e];
      if (e % (p + 1) == 0) v.x -= tk.sigma;  // the diagonal entries a (p + 1)
      M[e] = v;
      if (have_x) L[e] = B[((size_t)q * d.mmax + j) * pp + e];  // B_j, staged
    }
    __syncthreads();
    if (have_x) {  // M -= B_j X
      for (int e = tid; e < pp; e += nt) {
        const int a = e % p, c = e / p;
        double sr = 0.0, si = 0.0;
        for (int t = 0; t < p; ++t) {
          const double2 b = L[a + t * p], x = X[t + c * p];
          sr += b.x * x.x - b.y * x.y;
          si += b.x * x.y + b.y * x.x;
        }
        M[e].x -= sr;
        M[e].y -= si;
      }
      __syncthreads();
    }
    // right-looking LDL^H on the lower triangle: L(i, k) for i > k, pivots dg
    for (int k = 0; k < p; ++k) {
      if (tid == 0) {
        double dk = M[k + k * p].x;
        if (fabs(dk) < tk.tiny) dk = dk < 0 ? -tk.tiny : tk.tiny;
        dg[k] = dk;
        if (dk < 0) ++s_neg;
      }
      __syncthreads();
      const double dk = dg[k];
      for (int i = k + 1 + tid; i < p; i += nt) {
        const double2 v = M[i + k * p];
        L[i + k * p] = make_double2(v.x / dk, v.y / dk);
      }
      __syncthreads();
      const int r = p - k - 1;
      for (int e = tid; e < r * r; e += nt) {
        const int i = k + 1 + e % r, jj = k + 1 + e / r;
        if (jj > i) continue;
        const double2 li = L[i + k * p], lj = L[jj + k * p];
        // M(i, jj) -= L(i, k) dk conj(L(jj, k))
        M[i + jj * p].x -= dk * (li.x * lj.x + li.y * lj.y);
        M[i + jj * p].y -= dk * (li.y * lj.x - li.x * lj.y);
      }
      __syncthreads();
    }
    if (j + 1 < m) {
      // X = M^{-1} B_{j+1}^H: column c (four lanes of one warp each, p a
      // multiple of 8 so a warp's columns are all inside or all outside)
      const double2* Bn = B + ((size_t)q * d.mmax + j + 1) * pp;
      const int c = tid >> 2, part = tid & 3;
      if (c < p) {
        double2* x = X + (size_t)c * p;
        for (int a = part; a < p; a += 4) {  // rhs(a) = conj(B(c, a))
          const double2 b = Bn[c + (size_t)a * p];
          x[a] = make_double2(b.x, -b.y);
        }
        __syncwarp();
        for (int a = 0; a < p; ++a) {  // L y = rhs (unit lower)
          double sr = 0.0, si = 0.0;
          for (int t = part; t < a; t += 4) {
            const double2 l = L[a + t * p], y = x[t];
            sr += l.x * y.x - l.y * y.y;
            si += l.x * y.y + l.y * y.x;
          }
          sr += __shfl_xor_sync(0xffffffffu, sr, 1);
          si += __shfl_xor_sync(0xffffffffu, si, 1);
          sr += __shfl_xor_sync(0xffffffffu, sr, 2);
          si += __shfl_xor_sync(0xffffffffu, si, 2);
          if (part == 0) x[a] = make_double2(x[a].x - sr, x[a].y - si);
          __syncwarp();
        }
        for (int a = part; a < p; a += 4) x[a] = make_double2(x[a].x / dg[a], x[a].y / dg[a]);
        __syncwarp();
        for (int a = p - 1; a >= 0; --a) {  // L^H z = y
          double sr = 0.0, si = 0.0;
          for (int t = a + 1 + part; t < p; t += 4) {
            const double2 l = L[t + a * p], y = x[t];  // conj(L(t, a)) y_t
            sr += l.x * y.x + l.y * y.y;
            si += l.x * y.y - l.y * y.x;
          }
          sr += __shfl_xor_sync(0xffffffffu, sr, 1);
          si += __shfl_xor_sync(0xffffffffu, si, 1);
          sr += __shfl_xor_sync(0xffffffffu, sr, 2);
          si += __shfl_xor_sync(0xffffffffu, si, 2);
          if (part == 0) x[a] = make_double2(x[a].x - sr, x[a].y - si);
          __syncwarp();
        }
      }
      __syncthreads();
      have_x = true;
    }
  }
  if (tid == 0) counts[blockIdx.x] = s_neg;
}

}  // namespace

edk_status band_lowest_device(int p, int nev, const std::vector<int>& m,
                              const std::vector<std::vector<const double*>>& A,
                              const std::vector<std::vector<const double*>>& B,
                              cudaStream_t st, std::vector<std::vector<double>>& out) {
  const int nops = (int)m.size();
  out.assign(nops, std::vector<double>(nev, NAN));
  if (nops == 0) return EDK_OK;
  if (p < 8 || p > 64 || p % 8 != 0) {
    set_error("block eigenvalue step: block must be a multiple of 8 between 8 and 64");
    return EDK_INVALID_ARG;
  }
  BandDims d;
  d.p = p;
  d.mmax = std::max(1, *std::max_element(m.begin(), m.end()));
  d.nmax = (int64_t)p * d.mmax;
  const int kmax = (int)std::min<int64_t>(d.nmax, kBandSteps);
  d.vcols = kmax + 1;
  const size_t pp = (size_t)p * p;
  // T's blocks on the device
  std::vector<double2> hAB((size_t)nops * d.mmax * pp);
  DevBuf dA, dB, V, w, s1, s2, alpha, beta, invb, stop, nq, mqd;
  EDK_RETURN_IF(dA.alloc_async(hAB.size() * sizeof(double2), st));
  EDK_RETURN_IF(dB.alloc_async(hAB.size() * sizeof(double2), st));
  for (int pass = 0; pass < 2; ++pass) {
    std::fill(hAB.begin(), hAB.end(), make_double2(0.0, 0.0));
    for (int q = 0; q < nops; ++q)
      for (int j = 0; j < m[q]; ++j) {
        const double* src = pass == 0 ? A[q][j] : (j >= 1 ? B[q][j] : nullptr);
        if (src) std::memcpy(&hAB[((size_t)q * d.mmax + j) * pp], src, pp * sizeof(double2));
      }
    EDK_TRY_CUDA(cudaMemcpyAsync(pass == 0 ? dA.p : dB.p, hAB.data(), hAB.size() * sizeof(double2),
                                 cudaMemcpyHostToDevice, st));
    EDK_TRY_CUDA(cudaStreamSynchronize(st));  // hAB is refilled next pass
  }
  std::vector<int> hn(nops);
  for (int q = 0; q < nops; ++q) hn[q] = p * m[q];
  EDK_RETURN_IF(V.alloc_async((size_t)nops * d.vcols * d.nmax * sizeof(double2), st));
  EDK_RETURN_IF(w.alloc_async((size_t)nops * d.nmax * sizeof(double2), st));
  EDK_RETURN_IF(s1.alloc_async((size_t)nops * d.vcols * sizeof(double2), st));
  EDK_RETURN_IF(s2.alloc_async((size_t)nops * d.vcols * sizeof(double2), st));
  EDK_RETURN_IF(alpha.alloc_async((size_t)nops * d.vcols * sizeof(double), st));
  EDK_RETURN_IF(beta.alloc_async((size_t)nops * d.vcols * sizeof(double), st));
  EDK_RETURN_IF(invb.alloc_async((size_t)nops * sizeof(double), st));
  EDK_RETURN_IF(stop.alloc_async((size_t)nops * sizeof(int), st));
  EDK_RETURN_IF(nq.alloc_async((size_t)nops * sizeof(int), st));
  EDK_RETURN_IF(mqd.alloc_async((size_t)nops * sizeof(int), st));
  EDK_TRY_CUDA(cudaMemcpyAsync(nq.p, hn.data(), nops * sizeof(int), cudaMemcpyHostToDevice, st));
  EDK_TRY_CUDA(cudaMemcpyAsync(mqd.p, m.data(), nops * sizeof(int), cudaMemcpyHostToDevice, st));
  EDK_TRY_CUDA(cudaMemsetAsync(stop.p, 0, nops * sizeof(int), st));
  EDK_TRY_CUDA(cudaMemsetAsync(V.p, 0, (size_t)nops * d.vcols * d.nmax * sizeof(double2), st));
  // start vectors: the host form's seeded sequence, normalised, in column 0
  {
    std::vector<double2> v0((size_t)nops * d.nmax, make_double2(0.0, 0.0));
    for (int q = 0; q < nops; ++q) {
      uint64_t s = 0x12345678abcdefull;
      auto rnd = [&]() {
        s ^= s << 13;
        s ^= s >> 7;
        s ^= s << 17;
        return ((s >> 11) * (1.0 / 9007199254740992.0)) - 0.5;
      };
      double nr = 0.0;
      double2* v = v0.data() + (size_t)q * d.nmax;
      for (int i = 0; i < hn[q]; ++i) {
        const double re = rnd(), im = rnd();
        v[i] = make_double2(re, im);
        nr += re * re + im * im;
      }
      nr = std::sqrt(nr);
      for (int i = 0; i < hn[q]; ++i) v[i] = make_double2(v[i].x / nr, v[i].y / nr);
      EDK_TRY_CUDA(cudaMemcpyAsync(V.as<double2>() + (size_t)q * d.vcols * d.nmax, v,
                                   (size_t)d.nmax * sizeof(double2), cudaMemcpyHostToDevice, st));
    }
    EDK_TRY_CUDA(cudaStreamSynchronize(st));
  }
  // Lanczos on every T in lockstep; the host looks every 10 steps (and at
  // each operator's own last step), as the host form does
  std::vector<std::vector<double>> prev(nops), cand(nops);
  std::vector<int> finished(nops, 0), hstop(nops, 0);
  std::vector<double> ha((size_t)nops * d.vcols), hb((size_t)nops * d.vcols);
  const unsigned rows = (unsigned)((d.nmax + 255) / 256);
  int left = nops;
  for (int k = 0; k < kmax && left > 0; ++k) {
    k_band_mv<<<dim3(d.mmax, nops), p, 3 * p * sizeof(double2), st>>>(
        d, dA.as<double2>(), dB.as<double2>(), mqd.as<int>(), V.as<double2>(), k, w.as<double2>(),
        stop.as<int>());
    for (int pass = 0; pass < 2; ++pass) {
      double2* s = pass == 0 ? s1.as<double2>() : s2.as<double2>();
      k_band_dots<<<dim3((k + 8) / 8, nops), 256, 0, st>>>(d, nq.as<int>(), V.as<double2>(), k,
                                                          w.as<double2>(), s, stop.as<int>());
      k_band_update<<<dim3(rows, nops), 256, (k + 1) * sizeof(double2), st>>>(
          d, nq.as<int>(), V.as<double2>(), k, s, w.as<double2>(), stop.as<int>());
    }
    k_band_norm<<<nops, 256, 0, st>>>(d, nq.as<int>(), k, w.as<double2>(), s1.as<double2>(),
                                      alpha.as<double>(), beta.as<double>(), invb.as<double>(),
                                      stop.as<int>());
    k_band_scale<<<dim3(rows, nops), 256, 0, st>>>(d, nq.as<int>(), k, w.as<double2>(),
                                                   invb.as<double>(), V.as<double2>(),
                                                   stop.as<int>());
    EDK_TRY_CUDA(cudaGetLastError());
    bool look = (k + 1) % 10 == 0 || k + 1 == kmax;
    for (int q = 0; q < nops && !look; ++q)
      look = !finished[q] && k + 1 == std::min(hn[q], kBandSteps);
    if (!look) continue;
    EDK_TRY_CUDA(cudaMemcpyAsync(ha.data(), alpha.p, ha.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    EDK_TRY_CUDA(cudaMemcpyAsync(hb.data(), beta.p, hb.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    EDK_TRY_CUDA(cudaMemcpyAsync(hstop.data(), stop.p, nops * sizeof(int), cudaMemcpyDeviceToHost, st));
    EDK_TRY_CUDA(cudaStreamSynchronize(st));
    bool changed = false;
    for (int q = 0; q < nops; ++q) {
      if (finished[q]) continue;
      const int own = std::min(hn[q], kBandSteps);
      const int mm = hstop[q] > 0 ? hstop[q] : k + 1;
      const bool last = hstop[q] > 0 || k + 1 >= own;
      if (!last && (k + 1) % 10 != 0) continue;
      std::vector<double> ev(mm);
      tridiag_eigvals(mm, ha.data() + (size_t)q * d.vcols, hb.data() + (size_t)q * d.vcols,
                      ev.data());
      std::vector<double> dd;  // distinct values: closer than 1e-12 relative merge
      for (double x : ev)
        if (dd.empty() || x - dd.back() > 1e-12 * std::max(1.0, std::fabs(x))) dd.push_back(x);
      bool conv = last;
      if (!conv && (int)dd.size() >= nev + 4 && (int)prev[q].size() >= nev + 4) {
        conv = true;
        for (int t = 0; t < nev + 4; ++t)
          if (std::fabs(dd[t] - prev[q][t]) > 1e-13 * std::max(1.0, std::fabs(dd[0]))) conv = false;
      }
      prev[q] = dd;
      if (conv) {
        cand[q].assign(dd.begin(), dd.begin() + std::min<size_t>(dd.size(), nev + 4));
        finished[q] = 1;
        --left;
        if (hstop[q] == 0) {
          hstop[q] = k + 1;
          changed = true;
        }
      }
    }
    if (changed)
      EDK_TRY_CUDA(cudaMemcpyAsync(stop.p, hstop.data(), nops * sizeof(int), cudaMemcpyHostToDevice, st));
  }
  for (int q = 0; q < nops; ++q)
    if (!finished[q]) cand[q] = prev[q].size() > (size_t)nev + 4
                                    ? std::vector<double>(prev[q].begin(), prev[q].begin() + nev + 4)
                                    : prev[q];
  // Sturm counts at both edges of every candidate cluster, for T and T-hat
  struct Cluster { int q; double lo, hi, dl; };
  std::vector<Cluster> cl;
  std::vector<BandTask> tasks;
  for (int q = 0; q < nops; ++q) {
    double tiny[2];
    for (int j0 = 0; j0 < 2; ++j0) {
      double scale = 1.0;
      for (int j = j0; j < m[q]; ++j)
        for (int a = 0; a < p; ++a) scale = std::max(scale, std::fabs(A[q][j][2 * ((size_t)a * p + a)]));
      tiny[j0] = 1e-300 + 1e-15 * scale;
    }
    const std::vector<double>& c = cand[q];
    for (size_t i = 0; i < c.size();) {
      const double lo = c[i], dl = 1e-10 * std::max(1.0, std::fabs(lo));
      double hi = lo;
      size_t e = i + 1;
      while (e < c.size() && c[e] - hi <= dl) hi = c[e++];
      cl.push_back({q, lo, hi, dl});
      for (int j0 = 0; j0 < (m[q] > 1 ? 2 : 1); ++j0) {
        tasks.push_back({hi + dl, tiny[j0], q, j0});
        tasks.push_back({lo - dl, tiny[j0], q, j0});
      }
      i = e;
    }
  }
  std::vector<int> hc(tasks.size(), 0);
  if (!tasks.empty()) {
    DevBuf dt, dc;
    EDK_RETURN_IF(dt.alloc_async(tasks.size() * sizeof(BandTask), st));
    EDK_RETURN_IF(dc.alloc_async(tasks.size() * sizeof(int), st));
    EDK_TRY_CUDA(cudaMemcpyAsync(dt.p, tasks.data(), tasks.size() * sizeof(BandTask),
                                 cudaMemcpyHostToDevice, st));
    const size_t smem = 3 * pp * sizeof(double2) + p * sizeof(double);
    EDK_TRY_CUDA(cudaFuncSetAttribute(k_band_sturm, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem));
    k_band_sturm<<<(unsigned)tasks.size(), 256, smem, st>>>(d, dA.as<double2>(), dB.as<double2>(),
                                                             mqd.as<int>(), dt.as<BandTask>(),
                                                             dc.as<int>());
    EDK_TRY_CUDA(cudaGetLastError());
    EDK_TRY_CUDA(cudaMemcpyAsync(hc.data(), dc.p, hc.size() * sizeof(int), cudaMemcpyDeviceToHost, st));
    EDK_TRY_CUDA(cudaStreamSynchronize(st));
  }
  // keep a cluster when T has more eigenvalues in its window than T-hat
  std::vector<int> got(nops, 0);
  size_t t = 0;
  for (const Cluster& c : cl) {
    const int q = c.q;
    const int nt = hc[t] - hc[t + 1];
    const int nh = m[q] > 1 ? hc[t + 2] - hc[t + 3] : 0;
    t += m[q] > 1 ? 4 : 2;
    if (got[q] < nev && nt - nh >= 1) out[q][got[q]++] = c.lo;
  }
  return EDK_OK;
}

}  // namespace edk
