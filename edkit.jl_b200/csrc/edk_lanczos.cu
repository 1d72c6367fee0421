// edk_lanczos.cu — Lanczos ground state and adaptive Krylov exp(-iHt) on the
// device.
//
// The Krylov basis V (D x (m+1), column-major) lives in HBM in the storage
// precision (f64/c128, or f32/c64 for the mixed path); the working vector w,
// every inner product and the Gram-Schmidt coefficients are FP64.  One
// Lanczos step is
//   wt = H v_j                        (row-gather matvec)
//   s  = V^H wt ; alpha_j = Re s_j     (pass 1 over V, FP64 block partials)
//   w  = wt - V s                      (pass 2)
//   u  = V^H w                         (pass 3)
//   w  = w - V u ; beta_j = ||w||      (pass 4, norm fused)
//   v_{j+1} = w / beta_j
// i.e. classical Gram-Schmidt applied twice against the whole basis, the
// reorthogonalisation of _lanczos_build! (src/algorithms/TimeEvolution.jl:
// 250-306) with its three-term recurrence folded into the first sweep, and
// the same lucky-breakdown rule beta <= sqrt(eps) * max(1, |alpha|).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <complex>
#include <memory>
#include <numeric>
#include <vector>

#include "edk_internal.cuh"

namespace edk {

template <class T> struct CxT;
template <> struct CxT<double> { static constexpr bool cx = false; };
template <> struct CxT<double2> { static constexpr bool cx = true; };
template <> struct CxT<float> { static constexpr bool cx = false; };
template <> struct CxT<float2> { static constexpr bool cx = true; };

__device__ __forceinline__ double2 ld2(const double* p) { return make_double2(*p, 0.0); }
__device__ __forceinline__ double2 ld2(const double2* p) { return *p; }
__device__ __forceinline__ double2 ld2(const float* p) { return make_double2((double)*p, 0.0); }
__device__ __forceinline__ double2 ld2(const float2* p) {
  float2 v = *p;
  return make_double2((double)v.x, (double)v.y);
}
__device__ __forceinline__ void st2(double* p, double2 v) { *p = v.x; }
__device__ __forceinline__ void st2(double2* p, double2 v) { *p = v; }
__device__ __forceinline__ void st2(float* p, double2 v) { *p = (float)v.x; }
__device__ __forceinline__ void st2(float2* p, double2 v) { *p = make_float2((float)v.x, (float)v.y); }

constexpr int kRowsPerThread = 4;
constexpr int kDotThreads = 256;
constexpr int kRowsPerBlock = kRowsPerThread * kDotThreads;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// part[c * nblk + blk] = sum_{rows of blk} conj(V[r, c]) * w[r]
template <class VV, class WV>
__global__ void __launch_bounds__(kDotThreads) k_dots(const VV* __restrict__ V, int64_t ld, int ncols,
                                                      const WV* __restrict__ w, int64_t D,
                                                      double2* __restrict__ part) {
  extern __shared__ double2 s_part[];  // [8 warps][ncols]
  constexpr bool CX = CxT<VV>::cx || CxT<WV>::cx;
  const int64_t r0 = (int64_t)blockIdx.x * kRowsPerBlock;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double2 wv[kRowsPerThread];
  int64_t rows[kRowsPerThread];
#pragma unroll
  for (int k = 0; k < kRowsPerThread; ++k) {
    rows[k] = r0 + threadIdx.x + (int64_t)k * kDotThreads;
    wv[k] = rows[k] < D ? ld2(w + rows[k]) : make_double2(0.0, 0.0);
  }
  for (int c = 0; c < ncols; ++c) {
    const VV* Vc = V + (int64_t)c * ld;
    double ar = 0.0, ai = 0.0;
#pragma unroll
    for (int k = 0; k < kRowsPerThread; ++k) {
      if (rows[k] < D) {
        double2 v = ld2(Vc + rows[k]);
        ar += v.x * wv[k].x + v.y * wv[k].y;
        if (CX) ai += v.x * wv[k].y - v.y * wv[k].x;
      }
    }
    ar = warp_sum(ar);
    if (CX) ai = warp_sum(ai);
    if (lane == 0) s_part[warp * ncols + c] = make_double2(ar, ai);
  }
  __syncthreads();
  const int nw = blockDim.x >> 5;
  for (int c = threadIdx.x; c < ncols; c += blockDim.x) {
    double sr = 0.0, si = 0.0;
    for (int q = 0; q < nw; ++q) {
      sr += s_part[q * ncols + c].x;
      si += s_part[q * ncols + c].y;
    }
    part[(int64_t)c * gridDim.x + blockIdx.x] = make_double2(sr, si);
  }
}

// out[c] = sum_b part[c * nblk + b]  (one block per column)
__global__ void k_reduce_cols(const double2* __restrict__ part, int nblk, int ncols,
                              double2* __restrict__ out) {
  const int c = blockIdx.x;
  double sr = 0.0, si = 0.0;
  for (int b = threadIdx.x; b < nblk; b += blockDim.x) {
    double2 v = part[(int64_t)c * nblk + b];
    sr += v.x;
    si += v.y;
  }
  __shared__ double s_r[32], s_i[32];
  sr = warp_sum(sr);
  si = warp_sum(si);
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) { s_r[warp] = sr; s_i[warp] = si; }
  __syncthreads();
  if (warp == 0) {
    int nw = blockDim.x >> 5;
    sr = lane < nw ? s_r[lane] : 0.0;
    si = lane < nw ? s_i[lane] : 0.0;
    sr = warp_sum(sr);
    si = warp_sum(si);
    if (lane == 0) out[c] = make_double2(sr, si);
  }
}

// wout[r] = win[r] - sum_c V[r, c] * coef[c];  optional per-block ||wout||^2.
template <class VV, class WI, class WO>
__global__ void __launch_bounds__(256) k_update(const VV* __restrict__ V, int64_t ld, int ncols,
                                                const double2* __restrict__ coef,
                                                const WI* __restrict__ win, WO* __restrict__ wout,
                                                int64_t D, double* __restrict__ normpart) {
  extern __shared__ double2 s_coef[];
  constexpr bool CX = CxT<VV>::cx || CxT<WI>::cx;
  for (int c = threadIdx.x; c < ncols; c += blockDim.x) s_coef[c] = coef[c];
  __syncthreads();
  double nrm = 0.0;
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < D;
       r += (int64_t)gridDim.x * blockDim.x) {
    double2 acc = ld2(win + r);
    int c = 0;
    for (; c + 4 <= ncols; c += 4) {
      double2 v0 = ld2(V + (int64_t)(c + 0) * ld + r);
      double2 v1 = ld2(V + (int64_t)(c + 1) * ld + r);
      double2 v2 = ld2(V + (int64_t)(c + 2) * ld + r);
      double2 v3 = ld2(V + (int64_t)(c + 3) * ld + r);
      double2 k0 = s_coef[c], k1 = s_coef[c + 1], k2 = s_coef[c + 2], k3 = s_coef[c + 3];
      acc.x -= v0.x * k0.x + v1.x * k1.x + v2.x * k2.x + v3.x * k3.x;
      if (CX) {
        acc.x += v0.y * k0.y + v1.y * k1.y + v2.y * k2.y + v3.y * k3.y;
        acc.y -= v0.x * k0.y + v0.y * k0.x + v1.x * k1.y + v1.y * k1.x + v2.x * k2.y + v2.y * k2.x +
                 v3.x * k3.y + v3.y * k3.x;
      }
    }
    for (; c < ncols; ++c) {
      double2 v = ld2(V + (int64_t)c * ld + r);
      double2 k = s_coef[c];
      acc.x -= v.x * k.x;
      if (CX) {
        acc.x += v.y * k.y;
        acc.y -= v.x * k.y + v.y * k.x;
      }
    }
    st2(wout + r, acc);
    if (normpart) nrm += acc.x * acc.x + (CX ? acc.y * acc.y : 0.0);
  }
  if (normpart) {
    __shared__ double s_n[32];
    nrm = warp_sum(nrm);
    int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) s_n[warp] = nrm;
    __syncthreads();
    if (warp == 0) {
      int nw = blockDim.x >> 5;
      nrm = lane < nw ? s_n[lane] : 0.0;
      nrm = warp_sum(nrm);
      if (lane == 0) normpart[blockIdx.x] = nrm;
    }
  }
}

// sum of per-block norms -> out[0]
__global__ void k_sum(const double* __restrict__ p, int n, double* __restrict__ out) {
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s += p[i];
  __shared__ double sh[32];
  s = warp_sum(s);
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) sh[warp] = s;
  __syncthreads();
  if (warp == 0) {
    int nw = blockDim.x >> 5;
    s = lane < nw ? sh[lane] : 0.0;
    s = warp_sum(s);
    if (lane == 0) out[0] = s;
  }
}

// out[r] = scale * w[r]
template <class WI, class VO>
__global__ void k_scale(const WI* __restrict__ w, int64_t D, double scale, VO* __restrict__ out) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < D;
       r += (int64_t)gridDim.x * blockDim.x) {
    double2 v = ld2(w + r);
    st2(out + r, make_double2(v.x * scale, v.y * scale));
  }
}

// out[r] = scale * sum_c V[r, c] * coef[c]
template <class VV, class OV>
__global__ void __launch_bounds__(256) k_gemv(const VV* __restrict__ V, int64_t ld, int ncols,
                                              const double2* __restrict__ coef, double scale,
                                              OV* __restrict__ out, int64_t D) {
  extern __shared__ double2 s_coef[];
  for (int c = threadIdx.x; c < ncols; c += blockDim.x) s_coef[c] = coef[c];
  __syncthreads();
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < D;
       r += (int64_t)gridDim.x * blockDim.x) {
    double ar = 0.0, ai = 0.0;
    for (int c = 0; c < ncols; ++c) {
      double2 v = ld2(V + (int64_t)c * ld + r);
      double2 k = s_coef[c];
      ar += v.x * k.x - v.y * k.y;
      ai += v.x * k.y + v.y * k.x;
    }
    st2(out + r, make_double2(ar * scale, ai * scale));
  }
}

namespace {

int vec_grid(int64_t D) {
  int64_t g = (D + 255) / 256;
  if (g < 1) g = 1;
  if (g > 148 * 16) g = 148 * 16;
  return (int)g;
}

size_t esize(int dt) {
  switch (dt) {
    case EDK_F64: return 8;
    case EDK_C128: return 16;
    case EDK_F32: return 4;
    case EDK_C64: return 8;
  }
  return 0;
}
bool is_cx(int dt) { return dt == EDK_C128 || dt == EDK_C64; }
int w_dtype(int vdt) { return is_cx(vdt) ? EDK_C128 : EDK_F64; }

// type dispatch helpers ------------------------------------------------------
template <class F> edk_status with_type(int dt, F&& f) {
  switch (dt) {
    case EDK_F64: return f((double*)nullptr);
    case EDK_C128: return f((double2*)nullptr);
    case EDK_F32: return f((float*)nullptr);
    case EDK_C64: return f((float2*)nullptr);
  }
  set_error("unknown dtype");
  return EDK_INVALID_ARG;
}

// ----------------------------------------------------------------------------
// Lanczos engine: owns V, w and the reduction scratch for one operator.
// ----------------------------------------------------------------------------
struct Engine {
  edk_operator* op = nullptr;
  cudaStream_t st = nullptr;
  int64_t D = 0;
  int vdt = EDK_F64;   // storage dtype of V (and of the matvec)
  int wdt = EDK_F64;   // FP64 working dtype (F64 / C128)
  int mcap = 0;        // columns of V
  DevBuf V, w, wt, part, coef, normpart, scal;
  int nblk = 0, ngrid = 0;
  cudaEvent_t e0 = nullptr, e1 = nullptr, e2 = nullptr;
  double t_matvec = 0.0, t_reorth = 0.0;
  int matvecs = 0;

  ~Engine() {
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (e2) cudaEventDestroy(e2);
  }

  edk_status init(edk_operator* o, int vdtype, int ncols, cudaStream_t s) {
    op = o;
    st = s;
    D = o->b->D;
    vdt = vdtype;
    wdt = w_dtype(vdt);
    mcap = ncols;
    EDK_RETURN_IF(V.alloc((size_t)D * ncols * esize(vdt)));
    EDK_RETURN_IF(w.alloc((size_t)D * esize(wdt)));
    EDK_RETURN_IF(wt.alloc((size_t)D * esize(vdt)));
    nblk = (int)std::max<int64_t>(1, (D + kRowsPerBlock - 1) / kRowsPerBlock);
    ngrid = vec_grid(D);
    EDK_RETURN_IF(part.alloc((size_t)nblk * ncols * sizeof(double2)));
    EDK_RETURN_IF(coef.alloc((size_t)ncols * sizeof(double2)));
    EDK_RETURN_IF(normpart.alloc((size_t)ngrid * sizeof(double)));
    EDK_RETURN_IF(scal.alloc(64));
    EDK_TRY_CUDA(cudaEventCreate(&e0));
    EDK_TRY_CUDA(cudaEventCreate(&e1));
    EDK_TRY_CUDA(cudaEventCreate(&e2));
    return EDK_OK;
  }
  void* col(int j) const { return (char*)V.p + (size_t)j * D * esize(vdt); }

  // coef[0..ncols) = V[:, 0:ncols]^H x   (x of dtype xdt)
  edk_status dots(int ncols, const void* x, int xdt) {
    size_t smem = (size_t)(kDotThreads / 32) * ncols * sizeof(double2);
    edk_status s = with_type(vdt, [&](auto vp) {
      using VV = std::remove_pointer_t<decltype(vp)>;
      return with_type(xdt, [&](auto xp) {
        using XV = std::remove_pointer_t<decltype(xp)>;
        auto kern = k_dots<VV, XV>;
        if (smem > 48 * 1024)
          cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        kern<<<nblk, kDotThreads, smem, st>>>((const VV*)V.p, D, ncols, (const XV*)x, D,
                                               part.as<double2>());
        return EDK_OK;
      });
    });
    EDK_RETURN_IF(s);
    k_reduce_cols<<<ncols, 256, 0, st>>>(part.as<double2>(), nblk, ncols, coef.as<double2>());
    EDK_TRY_CUDA(cudaGetLastError());
    return EDK_OK;
  }
  // wout = win - V[:, 0:ncols] coef ; optional ||wout||^2 into scal[0]
  edk_status update(int ncols, const void* win, int wint, void* wout, bool norm) {
    size_t smem = (size_t)ncols * sizeof(double2);
    edk_status s = with_type(vdt, [&](auto vp) {
      using VV = std::remove_pointer_t<decltype(vp)>;
      return with_type(wint, [&](auto ip) {
        using WI = std::remove_pointer_t<decltype(ip)>;
        return with_type(wdt, [&](auto op_) {
          using WO = std::remove_pointer_t<decltype(op_)>;
          k_update<VV, WI, WO><<<ngrid, 256, smem, st>>>(
              (const VV*)V.p, D, ncols, coef.as<double2>(), (const WI*)win, (WO*)wout, D,
              norm ? normpart.as<double>() : nullptr);
          return EDK_OK;
        });
      });
    });
    EDK_RETURN_IF(s);
    if (norm) k_sum<<<1, 256, 0, st>>>(normpart.as<double>(), ngrid, scal.as<double>());
    EDK_TRY_CUDA(cudaGetLastError());
    return EDK_OK;
  }
  // V[:, j] = scale * src (src dtype sdt)
  edk_status store_col(int j, const void* src, int sdt, double scale) {
    return with_type(sdt, [&](auto sp) {
      using SV = std::remove_pointer_t<decltype(sp)>;
      return with_type(vdt, [&](auto vp) {
        using VV = std::remove_pointer_t<decltype(vp)>;
        k_scale<SV, VV><<<ngrid, 256, 0, st>>>((const SV*)src, D, scale, (VV*)col(j));
        return EDK_OK;
      });
    });
  }
  // out (dtype odt) = scale * V[:, 0:ncols] c  (c host, complex)
  edk_status combine(int ncols, const std::vector<std::complex<double>>& c, double scale,
                     void* out, int odt) {
    EDK_TRY_CUDA(cudaMemcpyAsync(coef.p, c.data(), ncols * sizeof(double2),
                                 cudaMemcpyHostToDevice, st));
    size_t smem = (size_t)ncols * sizeof(double2);
    return with_type(vdt, [&](auto vp) {
      using VV = std::remove_pointer_t<decltype(vp)>;
      return with_type(odt, [&](auto op_) {
        using OV = std::remove_pointer_t<decltype(op_)>;
        k_gemv<VV, OV><<<ngrid, 256, smem, st>>>((const VV*)V.p, D, ncols, coef.as<double2>(),
                                                  scale, (OV*)out, D);
        return EDK_OK;
      });
    });
  }
  edk_status read_scal(double* h, int n) {
    EDK_TRY_CUDA(cudaMemcpyAsync(h, scal.p, n * sizeof(double), cudaMemcpyDeviceToHost, st));
    EDK_TRY_CUDA(cudaStreamSynchronize(st));
    return EDK_OK;
  }
  // normalise src (dtype sdt, device) into V[:, 0]; returns the norm
  edk_status set_start(const void* src, int sdt, double* nrm) {
    // ||src||^2 via a zero-column update: wout = src, norm fused
    EDK_RETURN_IF(update(0, src, sdt, w.p, true));
    double n2 = 0.0;
    EDK_RETURN_IF(read_scal(&n2, 1));
    *nrm = std::sqrt(n2);
    if (!(*nrm > 0.0)) return EDK_OK;
    return store_col(0, w.p, wdt, 1.0 / *nrm);
  }

};

// Lanczos run with per-step host bookkeeping.  Returns alphas/betas.
struct RunResult {
  std::vector<double> a, b;
  int steps = 0;
  bool breakdown = false;
};

edk_status lanczos_run(Engine& E, int max_steps, int nev, double tol, int check_every,
                       bool reorth, RunResult& R, std::vector<double>* evals_out) {
  R.a.assign(max_steps, 0.0);
  R.b.assign(max_steps, 0.0);
  std::vector<double> prev(nev, 0.0), cur(max_steps);
  const double seps = std::sqrt(std::numeric_limits<double>::epsilon());
  int last_check = -1;
  for (int j = 0; j < max_steps; ++j) {
    // step: matvec + CGS2
    EDK_TRY_CUDA(cudaEventRecord(E.e0, E.st));
    EDK_RETURN_IF(apply_device(E.op, E.vdt, E.col(j), E.wt.p, 1, E.D, E.D, 0, E.st));
    EDK_TRY_CUDA(cudaEventRecord(E.e1, E.st));
    ++E.matvecs;
    double2 s_j;
    if (reorth) {
      EDK_RETURN_IF(E.dots(j + 1, E.wt.p, E.vdt));
      EDK_TRY_CUDA(cudaMemcpyAsync(&s_j, E.coef.as<double2>() + j, sizeof(double2),
                                   cudaMemcpyDeviceToHost, E.st));
      EDK_RETURN_IF(E.update(j + 1, E.wt.p, E.vdt, E.w.p, false));
      EDK_RETURN_IF(E.dots(j + 1, E.w.p, E.wdt));
      EDK_RETURN_IF(E.update(j + 1, E.w.p, E.wdt, E.w.p, true));
    } else {
      // plain three-term recurrence: project out v_{j-1}, v_j only
      int c0 = std::max(0, j - 1);
      EDK_RETURN_IF(E.dots(j + 1, E.wt.p, E.vdt));
      EDK_TRY_CUDA(cudaMemcpyAsync(&s_j, E.coef.as<double2>() + j, sizeof(double2),
                                   cudaMemcpyDeviceToHost, E.st));
      // zero all but the last two coefficients
      std::vector<double2> keep(j + 1);
      EDK_TRY_CUDA(cudaMemcpyAsync(keep.data(), E.coef.p, (j + 1) * sizeof(double2),
                                   cudaMemcpyDeviceToHost, E.st));
      EDK_TRY_CUDA(cudaStreamSynchronize(E.st));
      for (int q = 0; q < c0; ++q) keep[q] = make_double2(0.0, 0.0);
      EDK_TRY_CUDA(cudaMemcpyAsync(E.coef.p, keep.data(), (j + 1) * sizeof(double2),
                                   cudaMemcpyHostToDevice, E.st));
      EDK_RETURN_IF(E.update(j + 1, E.wt.p, E.vdt, E.w.p, true));
    }
    EDK_TRY_CUDA(cudaEventRecord(E.e2, E.st));
    double n2 = 0.0;
    EDK_RETURN_IF(E.read_scal(&n2, 1));
    E.t_matvec += elapsed_ms(E.e0, E.e1) * 1e-3;
    E.t_reorth += elapsed_ms(E.e1, E.e2) * 1e-3;
    double alpha = s_j.x;
    double beta = std::sqrt(n2);
    R.a[j] = alpha;
    R.b[j] = beta;
    R.steps = j + 1;
    if (beta <= seps * std::max(1.0, std::fabs(alpha))) {
      R.b[j] = 0.0;
      R.breakdown = true;
      break;
    }
    if (j + 1 < E.mcap) EDK_RETURN_IF(E.store_col(j + 1, E.w.p, E.wdt, 1.0 / beta));
    // convergence check on the lowest nev Ritz values
    if (tol > 0 && check_every > 0 && ((j + 1) % check_every == 0) && j + 1 >= nev) {
      int m = j + 1;
      if (tridiag_eigvals(m, R.a.data(), R.b.data(), cur.data()) == 0) {
        bool conv = last_check >= 0;
        for (int q = 0; q < nev && q < m; ++q)
          conv &= std::fabs(cur[q] - prev[q]) <= tol * std::max(1.0, std::fabs(cur[q]));
        for (int q = 0; q < nev && q < m; ++q) prev[q] = cur[q];
        last_check = j;
        if (conv) break;
      }
    }
  }
  if (evals_out) {
    int m = R.steps;
    std::vector<double> w(m);
    tridiag_eigvals(m, R.a.data(), R.b.data(), w.data());
    evals_out->assign(w.begin(), w.begin() + std::min(m, nev));
  }
  return EDK_OK;
}

// copy / convert a caller vector to a device buffer of dtype dst_dt
edk_status stage_vector(const void* src, int src_dt, int ptr_kind, int64_t D, int dst_dt,
                        DevBuf& out, cudaStream_t st) {
  EDK_RETURN_IF(out.alloc((size_t)D * esize(dst_dt)));
  DevBuf tmp;
  const void* dsrc = src;
  if (ptr_kind == EDK_HOST) {
    EDK_RETURN_IF(tmp.alloc((size_t)D * esize(src_dt)));
    EDK_TRY_CUDA(cudaMemcpyAsync(tmp.p, src, (size_t)D * esize(src_dt), cudaMemcpyHostToDevice, st));
    dsrc = tmp.p;
  }
  edk_status s = with_type(src_dt, [&](auto sp) {
    using SV = std::remove_pointer_t<decltype(sp)>;
    return with_type(dst_dt, [&](auto dp) {
      using DV = std::remove_pointer_t<decltype(dp)>;
      k_scale<SV, DV><<<vec_grid(D), 256, 0, st>>>((const SV*)dsrc, D, 1.0, (DV*)out.p);
      return EDK_OK;
    });
  });
  EDK_RETURN_IF(s);
  EDK_TRY_CUDA(cudaStreamSynchronize(st));
  return EDK_OK;
}

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

}  // namespace

// lowest Ritz vector of the run (FP64 working dtype, device) into out
static edk_status ritz_vector(Engine& E, const RunResult& R, void* out) {
  int m = R.steps;
  std::vector<double> w(m), Q((size_t)m * m);
  if (tridiag_eigen(m, R.a.data(), R.b.data(), w.data(), Q.data()) != 0) {
    set_error("tridiagonal eigensolver did not converge");
    return EDK_NOT_CONVERGED;
  }
  std::vector<std::complex<double>> c(m);
  for (int q = 0; q < m; ++q) c[q] = Q[q];  // column 0 = lowest
  return E.combine(m, c, 1.0, out, E.wdt);
}

}  // namespace edk

using namespace edk;

// gs_out (optional, device, D elements of the FP64 working dtype): the lowest
// Ritz vector, normalised
static edk_status lanczos_common(edk_operator* op, const edk_lanczos_opts* opts, const void* v0,
                                 int32_t v0_dtype, int32_t ptr_kind, double* evals,
                                 double* alpha, double* beta, edk_lanczos_diag* diag,
                                 void* gs_out);

extern "C" edk_status edk_lanczos_e0(edk_operator* op, const edk_lanczos_opts* opts,
                                     const void* v0, int32_t v0_dtype, int32_t ptr_kind,
                                     double* evals, double* alpha, double* beta,
                                     edk_lanczos_diag* diag) {
  return lanczos_common(op, opts, v0, v0_dtype, ptr_kind, evals, alpha, beta, diag, nullptr);
}

namespace edk {
namespace gs_detail {
template <class T>
__global__ void k_sumsq(const T* __restrict__ v, int64_t n, double* __restrict__ out) {
  double acc = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    acc += (double)v[i] * (double)v[i];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(out, acc);
}
__global__ void k_scale_d(double* __restrict__ v, int64_t n, const double* __restrict__ ss) {
  const double s = 1.0 / sqrt(*ss);
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    v[i] *= s;
}
}  // namespace gs_detail
}  // namespace edk

extern "C" edk_status edk_lanczos_ground_state(edk_operator* op, const edk_lanczos_opts* opts,
                                               const void* v0, int32_t v0_dtype,
                                               int32_t ptr_kind, double* evals, void* psi,
                                               int32_t psi_dtype, edk_lanczos_diag* diag) {
  EDK_CHECK_ARG(op && opts && v0 && evals && psi, "edk_lanczos_ground_state: NULL argument");
  EDK_CHECK_ARG(v0_dtype >= EDK_F64 && v0_dtype <= EDK_C64, "edk_lanczos_ground_state: bad v0 dtype");
  const bool cx = op->is_complex || opts->complex_vectors || is_cx(v0_dtype);
  const int wdt = cx ? EDK_C128 : EDK_F64;
  if (psi_dtype != wdt) {
    set_error(cx ? "edk_lanczos_ground_state: the ground state is complex here; psi must be EDK_C128"
                 : "edk_lanczos_ground_state: the ground state is real here; psi must be EDK_F64");
    return EDK_INVALID_ARG;
  }
  const int64_t D = op->b->D;
  EDK_CHECK_ARG(D >= 1, "edk_lanczos_ground_state: empty basis");
  DevBuf gs, ss;
  EDK_RETURN_IF(gs.alloc((size_t)D * esize(wdt)));
  EDK_RETURN_IF(ss.alloc(sizeof(double)));
  EDK_RETURN_IF(lanczos_common(op, opts, v0, v0_dtype, ptr_kind, evals, nullptr, nullptr, diag,
                               gs.p));
  std::lock_guard<std::mutex> lk(op->mu);
  cudaStream_t st = op->stream;
  const int64_t nd = D * (cx ? 2 : 1);  // real doubles
  EDK_TRY_CUDA(cudaMemsetAsync(ss.p, 0, sizeof(double), st));
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((nd + 255) / 256, 148 * 8));
  gs_detail::k_sumsq<double><<<grid, 256, 0, st>>>(gs.as<double>(), nd, ss.as<double>());
  gs_detail::k_scale_d<<<grid, 256, 0, st>>>(gs.as<double>(), nd, ss.as<double>());
  EDK_TRY_CUDA(cudaGetLastError());
  EDK_TRY_CUDA(cudaMemcpyAsync(psi, gs.p, (size_t)D * esize(wdt),
                               ptr_kind == EDK_DEVICE ? cudaMemcpyDeviceToDevice
                                                      : cudaMemcpyDeviceToHost, st));
  EDK_TRY_CUDA(cudaStreamSynchronize(st));
  return EDK_OK;
}

static edk_status lanczos_common(edk_operator* op, const edk_lanczos_opts* opts, const void* v0,
                                 int32_t v0_dtype, int32_t ptr_kind, double* evals,
                                 double* alpha, double* beta, edk_lanczos_diag* diag,
                                 void* gs_out) {
  EDK_CHECK_ARG(op && opts && v0 && evals, "edk_lanczos_e0: NULL argument");
  EDK_CHECK_ARG(opts->max_steps >= 1, "edk_lanczos_e0: max_steps < 1");
  EDK_CHECK_ARG(opts->nev >= 1, "edk_lanczos_e0: nev < 1");
  EDK_CHECK_ARG(v0_dtype >= EDK_F64 && v0_dtype <= EDK_C64, "edk_lanczos_e0: bad v0 dtype");
  if (!op->gather) {
    set_error("edk_lanczos_e0: the operator is not Hermitian in this basis");
    return EDK_NOT_HERMITIAN;
  }
  std::lock_guard<std::mutex> lk(op->mu);
  double t0 = now_s();
  cudaStream_t st = op->stream;
  const int64_t D = op->b->D;
  EDK_CHECK_ARG(D >= 1, "edk_lanczos_e0: empty basis");
  if (((op->b->L <= 32 && op->b->dev.bk != BK_ABELIAN) || op->sell_ok) && opts->reorth) {
    // batch of one: device-side recurrence, graph-replayed steps
    DevBuf v0d;
    size_t es = (v0_dtype == EDK_F64 || v0_dtype == EDK_C64) ? 8 : (v0_dtype == EDK_C128 ? 16 : 4);
    const void* src = v0;
    if (ptr_kind == EDK_HOST) {
      EDK_RETURN_IF(v0d.alloc((size_t)D * es));
      EDK_TRY_CUDA(cudaMemcpyAsync(v0d.p, v0, (size_t)D * es, cudaMemcpyHostToDevice, st));
      src = v0d.p;
    }
    edk_lanczos_opts o = *opts;
    o.max_steps = (int)std::min<int64_t>(o.max_steps, D);
    std::vector<OpResult> res;
    std::vector<edk_operator*> one(1, op);
    EDK_RETURN_IF(batch_lanczos(one, o, src, v0_dtype, st, res, diag, gs_out));
    const OpResult& r = res[0];
    for (int q = 0; q < opts->nev; ++q) evals[q] = q < (int)r.ev.size() ? r.ev[q] : NAN;
    if (alpha) for (int q = 0; q < r.steps; ++q) alpha[q] = r.a[q];
    if (beta) for (int q = 0; q < r.steps; ++q) beta[q] = r.b[q];
    return EDK_OK;
  }
  bool cx = op->is_complex || opts->complex_vectors || is_cx(v0_dtype);
  int m = std::min<int64_t>(opts->max_steps, D);
  bool mixed = opts->precision == EDK_PREC_MIXED;
  int vdt = mixed ? (cx ? EDK_C64 : EDK_F32) : (cx ? EDK_C128 : EDK_F64);
  Engine E;
  EDK_RETURN_IF(E.init(op, vdt, m + 1, st));
  DevBuf start;
  EDK_RETURN_IF(stage_vector(v0, v0_dtype, ptr_kind, D, E.wdt, start, st));
  double nrm = 0.0;
  EDK_RETURN_IF(E.set_start(start.p, E.wdt, &nrm));
  if (!std::isfinite(nrm)) {
    set_error("Initial state has non-finite entries (NaN or Inf)");
    return EDK_INVALID_ARG;
  }
  if (!(nrm > 0.0)) {
    set_error("Initial state has zero norm");
    return EDK_ZERO_NORM;
  }
  RunResult R;
  std::vector<double> ev;
  int check = opts->check_every > 0 ? opts->check_every : 10;
  double tol = opts->tol;
  double tol1 = mixed ? std::max(tol, 1e-7) : tol;
  EDK_RETURN_IF(lanczos_run(E, m, opts->nev, tol1, check, opts->reorth != 0, R, &ev));
  int steps_low = R.steps;
  double tmv = E.t_matvec, tro = E.t_reorth;
  int mvs = E.matvecs;
  bool bd = R.breakdown;
  if (mixed) {
    // FP64 refinement: restart a short FP64 Lanczos from the FP64 Ritz vector
    DevBuf y;
    EDK_RETURN_IF(y.alloc((size_t)D * esize(E.wdt)));
    EDK_RETURN_IF(ritz_vector(E, R, y.p));
    int mr = std::min<int64_t>(opts->refine_steps > 0 ? opts->refine_steps : 20, D);
    int rounds = 0;
    while (true) {
      Engine F;
      EDK_RETURN_IF(F.init(op, E.wdt, mr + 1, st));
      double n0 = 0.0;
      EDK_RETURN_IF(F.set_start(y.p, E.wdt, &n0));
      RunResult R2;
      std::vector<double> ev2;
      EDK_RETURN_IF(lanczos_run(F, mr, opts->nev, tol, 5, true, R2, &ev2));
      tmv += F.t_matvec;
      tro += F.t_reorth;
      mvs += F.matvecs;
      bool done = R2.breakdown || ++rounds >= 8 || opts->nev > 1;
      double change = std::fabs(ev2[0] - ev[0]) / std::max(1.0, std::fabs(ev2[0]));
      ev = ev2;
      R = R2;
      if (done || change <= tol) {
        bd = R2.breakdown;
        if (gs_out) EDK_RETURN_IF(ritz_vector(F, R2, gs_out));
        break;
      }
      EDK_RETURN_IF(ritz_vector(F, R2, y.p));
    }
  }
  if (!mixed && gs_out) EDK_RETURN_IF(ritz_vector(E, R, gs_out));
  for (int q = 0; q < opts->nev; ++q) evals[q] = q < (int)ev.size() ? ev[q] : NAN;
  if (alpha) for (int q = 0; q < R.steps; ++q) alpha[q] = R.a[q];
  if (beta) for (int q = 0; q < R.steps; ++q) beta[q] = R.b[q];
  if (diag) {
    diag->steps = R.steps;
    diag->steps_low = mixed ? steps_low : R.steps;
    diag->matvecs = mvs;
    diag->breakdown = bd ? 1 : 0;
    diag->seconds_matvec = tmv;
    diag->seconds_reorth = tro;
    int mm = R.steps;
    std::vector<double> w(mm), Q((size_t)mm * mm);
    diag->residual = NAN;
    if (tridiag_eigen(mm, R.a.data(), R.b.data(), w.data(), Q.data()) == 0)
      diag->residual = std::fabs(R.b[mm - 1] * Q[(size_t)mm - 1]);
    diag->seconds = now_s() - t0;
  }
  return EDK_OK;
}

// ---------------------------------------------------------------------------
// Adaptive Krylov exp(-iHt) psi — TimeEvolution.jl:166-649
// ---------------------------------------------------------------------------
namespace edk {

struct KrylovCacheDev {
  Engine E;
  edk_krylov_opts o;
  int m = 0, m_max = 0, m_init = 0;
  double t_anchor = 0.0, t_latest = 0.0, norm_anchor = 0.0;
  std::vector<double> alpha, beta, lam, Q, Qe1, Qem;
  edk_krylov_diag* dg = nullptr;
  DevBuf anchor;  // FP64 complex anchor state

  edk_status build(int m_target) {  // _lanczos_build! :250-306
    m_target = std::min(m_target, m_max);
    const double seps = std::sqrt(std::numeric_limits<double>::epsilon());
    for (int j = m; j < m_target; ++j) {
      EDK_RETURN_IF(apply_device(E.op, E.vdt, E.col(j), E.wt.p, 1, E.D, E.D, 0, E.st));
      ++E.matvecs;
      dg->matvecs += 1;
      EDK_RETURN_IF(E.dots(j + 1, E.wt.p, E.vdt));
      double2 s_j;
      EDK_TRY_CUDA(cudaMemcpyAsync(&s_j, E.coef.as<double2>() + j, sizeof(double2),
                                   cudaMemcpyDeviceToHost, E.st));
      EDK_RETURN_IF(E.update(j + 1, E.wt.p, E.vdt, E.w.p, false));
      EDK_RETURN_IF(E.dots(j + 1, E.w.p, E.wdt));
      EDK_RETURN_IF(E.update(j + 1, E.w.p, E.wdt, E.w.p, true));
      double n2;
      EDK_RETURN_IF(E.read_scal(&n2, 1));
      double aj = s_j.x, bj = std::sqrt(n2);
      alpha[j] = aj;
      beta[j] = bj;
      if (bj <= seps * std::max(1.0, std::fabs(aj))) {
        m = j + 1;
        beta[j] = 0.0;
        return EDK_OK;
      }
      m = j + 1;
      if (j + 1 < E.mcap) EDK_RETURN_IF(E.store_col(j + 1, E.w.p, E.wdt, 1.0 / bj));
    }
    return EDK_OK;
  }
  edk_status reduced() {  // _build_reduced! :311-323
    lam.assign(m, 0.0);
    Q.assign((size_t)m * m, 0.0);
    if (tridiag_eigen(m, alpha.data(), beta.data(), lam.data(), Q.data()) != 0) {
      set_error("tridiagonal eigensolver did not converge");
      return EDK_NOT_CONVERGED;
    }
    Qe1.resize(m);
    Qem.resize(m);
    for (int k = 0; k < m; ++k) {
      Qe1[k] = Q[0 + (size_t)k * m];
      Qem[k] = Q[(m - 1) + (size_t)k * m];
    }
    return EDK_OK;
  }
  std::vector<std::complex<double>> coeffs(double tau) const {  // :329-338
    std::vector<std::complex<double>> ph(m), c(m, 0.0);
    for (int k = 0; k < m; ++k) ph[k] = std::polar(1.0, -tau * lam[k]) * Qe1[k];
    for (int r = 0; r < m; ++r) {
      std::complex<double> s = 0.0;
      for (int k = 0; k < m; ++k) s += Q[r + (size_t)k * m] * ph[k];
      c[r] = s;
    }
    return c;
  }
  double monitor(double tau) const {  // :341-350
    double bm = beta[m - 1];
    if (bm == 0.0) return 0.0;
    std::complex<double> acc = 0.0;
    for (int k = 0; k < m; ++k) acc += Qem[k] * std::polar(1.0, -tau * lam[k]) * Qe1[k];
    return std::fabs(bm) * std::abs(acc);
  }
  edk_status reconstruct(double tau, void* out) {  // :352-362 (out: C128 device)
    auto c = coeffs(tau);
    EDK_RETURN_IF(E.combine(m, c, norm_anchor, out, EDK_C128));
    if (o.normalize_output) {
      EDK_RETURN_IF(E.update(0, out, EDK_C128, E.w.p, true));
      double n2;
      EDK_RETURN_IF(E.read_scal(&n2, 1));
      double n = std::sqrt(n2);
      if (n > 0) {
        edk_status s = with_type(EDK_C128, [&](auto) {
          k_scale<double2, double2><<<vec_grid(E.D), 256, 0, E.st>>>(
              (const double2*)out, E.D, 1.0 / n, (double2*)out);
          return EDK_OK;
        });
        EDK_RETURN_IF(s);
      }
    }
    return EDK_OK;
  }
  int nsample_eff(double tau_try) const {  // :383-394
    int base_n = o.nsample;
    if (lam.empty() || m <= 1) return base_n;
    double om = lam[m - 1] - lam[0];
    if (om <= 0) return base_n;
    long n_nyq = (long)std::ceil(4 * om * tau_try / M_PI) + 1;
    long v = std::max<long>(base_n, n_nyq);
    return (int)std::min<long>(std::max<long>(v, base_n), 513);
  }
  double max_valid(double tau_try) const {  // :396-429
    if (!(tau_try > 0)) return 0.0;
    if (std::fabs(beta[m - 1]) <= o.tol) return tau_try;
    int n = nsample_eff(tau_try);
    for (int k = 0; k < n; ++k) {
      double xk = (n == 1) ? 0.0 : tau_try * (double)k / (double)(n - 1);
      double eta = monitor(xk);
      if (!std::isfinite(eta) || eta > o.tol) {
        if (k == 0) return 0.0;
        double lo = tau_try * (double)(k - 1) / (double)(n - 1), hi = xk;
        for (int q = 0; q < o.bisect_iters; ++q) {
          double mid = 0.5 * (lo + hi);
          if (monitor(mid) > o.tol) hi = mid; else lo = mid;
        }
        return lo;
      }
    }
    return tau_try;
  }
  edk_status extend(bool& ok) {  // :434-447
    ok = false;
    if (!o.extend_basis || m >= m_max) return EDK_OK;
    int old = m;
    EDK_RETURN_IF(build(std::min(m + o.extend_step, m_max)));
    if (m > old) {
      EDK_RETURN_IF(reduced());
      dg->basis_extensions += 1;
      dg->max_dim_used = std::max(dg->max_dim_used, m);
      ok = true;
    }
    return EDK_OK;
  }
  edk_status restart(double tau_valid) {  // :449-477
    EDK_RETURN_IF(reconstruct(tau_valid, anchor.p));
    t_anchor += tau_valid;
    EDK_RETURN_IF(E.update(0, anchor.p, EDK_C128, E.w.p, true));
    double n2;
    EDK_RETURN_IF(E.read_scal(&n2, 1));
    double nrm = std::sqrt(n2);
    if (!(nrm > 0)) {
      set_error("Restart failed: anchor state has zero norm");
      return EDK_ZERO_NORM;
    }
    norm_anchor = nrm;
    std::fill(alpha.begin(), alpha.end(), 0.0);
    std::fill(beta.begin(), beta.end(), 0.0);
    m = 0;
    EDK_RETURN_IF(E.store_col(0, anchor.p, EDK_C128, 1.0 / nrm));
    EDK_RETURN_IF(build(m_init));
    EDK_RETURN_IF(reduced());
    dg->basis_builds += 1;
    dg->restarts += 1;
    dg->max_dim_used = std::max(dg->max_dim_used, m);
    return EDK_OK;
  }
  edk_status ensure(double tau_target) {  // :486-520
    double rem = tau_target;
    if (rem <= 0) return EDK_OK;
    while (true) {
      double tv = max_valid(rem);
      if (tv >= rem) return EDK_OK;
      if (o.extend_basis && m < m_max) {
        bool ok;
        EDK_RETURN_IF(extend(ok));
        if (ok) continue;
      }
      if (tv <= 0) {
        if (m < m_max) {
          bool ok;
          EDK_RETURN_IF(extend(ok));
          if (ok) continue;
        }
        set_error("KrylovEvolutionCache: basis at m=" + std::to_string(m) +
                  " is not valid at τ=0; consider increasing m_max or loosening tol");
        return EDK_NOT_CONVERGED;
      }
      if (dg->n_intervals < 64) dg->accepted_intervals[dg->n_intervals] = tv;
      dg->n_intervals += 1;
      EDK_RETURN_IF(restart(tv));
      rem -= tv;
    }
  }
};

extern "C" void edk_krylov_default_opts(edk_krylov_opts* o) {
  if (!o) return;
  o->tol = 1e-10;
  o->m_init = 30;
  o->m_max = 60;
  o->extend_step = 10;
  o->nsample = 13;
  o->bisect_iters = 12;
  o->reuse_basis = 1;
  o->extend_basis = 1;
  o->normalize_output = 0;
  o->precision = EDK_PREC_FP64;
}

// checks of the KrylovEvolutionCache constructor (TimeEvolution.jl:178-189)
static edk_status krylov_check(edk_operator* op, const edk_krylov_opts* opts) {
  if (!op->gather) {
    set_error("edk_krylov_evolve: the propagator is Hermitian-only; the operator is not "
              "Hermitian in this basis");
    return EDK_NOT_HERMITIAN;
  }
  EDK_CHECK_ARG(op->b->D > 0, "Initial state must be non-empty");
  EDK_CHECK_ARG(opts->m_init >= 1, "m_init must be ≥ 1");
  EDK_CHECK_ARG(opts->m_max >= opts->m_init, "m_max must be ≥ m_init");
  EDK_CHECK_ARG(opts->nsample >= 2, "nsample must be ≥ 2");
  EDK_CHECK_ARG(opts->bisect_iters >= 0, "bisect_iters must be ≥ 0");
  EDK_CHECK_ARG(opts->extend_step >= 1, "extend_step must be ≥ 1");
  return EDK_OK;
}

// the constructor's set-up: anchor = psi0, V[:, 1] = psi0 / |psi0|, first basis
static edk_status krylov_start(KrylovCacheDev& K, edk_operator* op, const edk_krylov_opts* opts,
                               const void* psi0, int32_t ptr_kind, edk_krylov_diag* dg) {
  const int64_t D = op->b->D;
  cudaStream_t st = op->stream;
  K.o = *opts;
  K.dg = dg;
  K.m_max = (int)std::min<int64_t>(opts->m_max, D);
  K.m_init = std::min(opts->m_init, K.m_max);
  int vdt = opts->precision == EDK_PREC_MIXED ? EDK_C64 : EDK_C128;
  EDK_RETURN_IF(K.E.init(op, vdt, K.m_max + 1, st));
  K.alpha.assign(K.m_max, 0.0);
  K.beta.assign(K.m_max, 0.0);
  EDK_RETURN_IF(stage_vector(psi0, EDK_C128, ptr_kind, D, EDK_C128, K.anchor, st));
  double nrm = 0.0;
  EDK_RETURN_IF(K.E.set_start(K.anchor.p, EDK_C128, &nrm));
  if (!std::isfinite(nrm)) {
    set_error("Initial state has non-finite entries (NaN or Inf)");
    return EDK_INVALID_ARG;
  }
  if (!(nrm > 0)) {
    set_error("Initial state has zero norm");
    return EDK_ZERO_NORM;
  }
  K.norm_anchor = nrm;
  EDK_RETURN_IF(K.build(K.m_init));
  EDK_RETURN_IF(K.reduced());
  dg->basis_builds += 1;
  dg->max_dim_used = std::max(dg->max_dim_used, K.m);
  return EDK_OK;
}

// timeevolve!(cache, t) for each t of a non-decreasing sequence (:586-636):
// column p of out (device) or of the host array receives the state at ts[p]
static edk_status krylov_serve(KrylovCacheDev& K, edk_operator* op, const double* ts, int64_t nts,
                               const int64_t* perm, void* out, int32_t ptr_kind, DevBuf& psi) {
  const int64_t D = op->b->D;
  cudaStream_t st = op->stream;
  for (int64_t q = 0; q < nts; ++q) {
    const int64_t p = perm ? perm[q] : q;
    const double tf = ts[p];
    const double tau = tf - K.t_anchor;
    EDK_RETURN_IF(K.ensure(tau));
    void* dst = (ptr_kind == EDK_DEVICE) ? (void*)((double2*)out + (size_t)p * D) : psi.p;
    EDK_RETURN_IF(K.reconstruct(tf - K.t_anchor, dst));
    if (ptr_kind == EDK_HOST)
      EDK_TRY_CUDA(cudaMemcpyAsync((double2*)out + (size_t)p * D, psi.p, (size_t)D * 16,
                                   cudaMemcpyDeviceToHost, st));
    K.t_latest = tf;
    K.dg->total_times_served += 1;
  }
  EDK_TRY_CUDA(cudaStreamSynchronize(st));
  return EDK_OK;
}

}  // namespace edk

struct edk_krylov_cache {
  edk_operator* op = nullptr;
  edk::KrylovCacheDev K;
  edk_krylov_diag diag{};
  edk::DevBuf psi;  // staging column of the host path
  double seconds = 0.0;
};

extern "C" edk_status edk_krylov_evolve(edk_operator* op, const edk_krylov_opts* opts,
                                        const void* psi0, const double* ts, int64_t nts,
                                        void* out, int32_t ptr_kind, edk_krylov_diag* diag) {
  EDK_CHECK_ARG(op && opts && psi0 && ts && out, "edk_krylov_evolve: NULL argument");
  EDK_CHECK_ARG(nts >= 0, "edk_krylov_evolve: nts < 0");
  EDK_CHECK_ARG(ptr_kind == EDK_HOST || ptr_kind == EDK_DEVICE, "edk_krylov_evolve: bad ptr_kind");
  for (int64_t q = 0; q < nts; ++q)
    if (ts[q] < 0) {
      set_error("timeevolve: all times in ts must be non-negative; backward evolution is not "
                "supported");
      return EDK_BACKWARD_TIME;
    }
  EDK_RETURN_IF(krylov_check(op, opts));
  std::lock_guard<std::mutex> lk(op->mu);
  double t0 = now_s();
  const int64_t D = op->b->D;
  edk_krylov_diag local{};
  edk_krylov_diag* dg = diag ? diag : &local;
  *dg = edk_krylov_diag{};
  KrylovCacheDev K;
  EDK_RETURN_IF(krylov_start(K, op, opts, psi0, ptr_kind, dg));
  // serve times in sorted order, write columns in the caller's order
  std::vector<int64_t> perm(nts);
  std::iota(perm.begin(), perm.end(), 0);
  std::stable_sort(perm.begin(), perm.end(), [&](int64_t a, int64_t b) { return ts[a] < ts[b]; });
  DevBuf psi;
  if (ptr_kind == EDK_HOST) EDK_RETURN_IF(psi.alloc((size_t)D * 16));
  EDK_RETURN_IF(krylov_serve(K, op, ts, nts, perm.data(), out, ptr_kind, psi));
  dg->seconds = now_s() - t0;
  return EDK_OK;
}

extern "C" edk_status edk_krylov_cache_create(edk_operator* op, const edk_krylov_opts* opts,
                                              const void* psi0, int32_t ptr_kind,
                                              edk_krylov_cache** out) {
  EDK_CHECK_ARG(out != nullptr, "edk_krylov_cache_create: out is NULL");
  *out = nullptr;
  EDK_CHECK_ARG(op && opts && psi0, "edk_krylov_cache_create: NULL argument");
  EDK_CHECK_ARG(ptr_kind == EDK_HOST || ptr_kind == EDK_DEVICE,
                "edk_krylov_cache_create: bad ptr_kind");
  EDK_RETURN_IF(krylov_check(op, opts));
  std::lock_guard<std::mutex> lk(op->mu);
  double t0 = now_s();
  auto* c = new edk_krylov_cache;
  std::unique_ptr<edk_krylov_cache> guard(c);
  c->op = op;
  EDK_RETURN_IF(krylov_start(c->K, op, opts, psi0, ptr_kind, &c->diag));
  c->seconds = now_s() - t0;
  c->diag.seconds = c->seconds;
  *out = guard.release();
  return EDK_OK;
}

extern "C" edk_status edk_krylov_cache_evolve(edk_krylov_cache* c, const double* ts, int64_t nts,
                                              void* out, int32_t ptr_kind) {
  EDK_CHECK_ARG(c && ts && out, "edk_krylov_cache_evolve: NULL argument");
  EDK_CHECK_ARG(nts >= 0, "edk_krylov_cache_evolve: nts < 0");
  EDK_CHECK_ARG(ptr_kind == EDK_HOST || ptr_kind == EDK_DEVICE,
                "edk_krylov_cache_evolve: bad ptr_kind");
  for (int64_t q = 1; q < nts; ++q)
    if (ts[q] < ts[q - 1]) {
      set_error("timeevolve!: ts must be sorted in ascending order");
      return EDK_INVALID_ARG;
    }
  for (int64_t q = 0; q < nts; ++q) {
    if (!(ts[q] >= c->K.t_latest)) {
      char msg[256];
      std::snprintf(msg, sizeof msg,
                    "timeevolve!: requested time %.17g precedes the last served time %.17g; "
                    "backward evolution is not supported", ts[q], c->K.t_latest);
      set_error(msg);
      return EDK_BACKWARD_TIME;
    }
  }
  edk_operator* op = c->op;
  std::lock_guard<std::mutex> lk(op->mu);
  double t0 = now_s();
  if (ptr_kind == EDK_HOST && !c->psi.p) EDK_RETURN_IF(c->psi.alloc((size_t)op->b->D * 16));
  c->K.dg = &c->diag;
  edk_status rc = krylov_serve(c->K, op, ts, nts, nullptr, out, ptr_kind, c->psi);
  c->seconds += now_s() - t0;
  c->diag.seconds = c->seconds;
  return rc;
}

extern "C" edk_status edk_krylov_cache_info(const edk_krylov_cache* c, double* t_anchor,
                                            double* t_latest, int32_t* m, edk_krylov_diag* diag) {
  EDK_CHECK_ARG(c != nullptr, "edk_krylov_cache_info: NULL cache");
  if (t_anchor) *t_anchor = c->K.t_anchor;
  if (t_latest) *t_latest = c->K.t_latest;
  if (m) *m = c->K.m;
  if (diag) *diag = c->diag;
  return EDK_OK;
}

extern "C" edk_status edk_krylov_cache_destroy(edk_krylov_cache* c) {
  if (!c) return EDK_OK;
  std::lock_guard<std::mutex> lk(c->op->mu);  // device buffers go back while the operator is locked
  delete c;
  return EDK_OK;
}
