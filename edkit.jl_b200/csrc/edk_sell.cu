// edk_sell.cu — materialised operator: the device counterpart of EDKit's
// sparse!(opt) cache (src/Operator.jl:221-285).
//
// The matrix-free kernels recompute every nonzero (orbit canonicalisation and
// table probe) on every application.  An iterative solver applies the same H
// hundreds of times, so it pays to expand the rows once: two passes of the
// expansion (count, then fill) write a sliced-ELLPACK matrix (32-row slices,
// rows sorted by length inside 256-row windows) whose entries are a 4-byte
// target row and a 2-byte coefficient code.  The code indexes a small table of
// distinct values val * phase * R[target]; 1/R[row] is applied per row from a
// table of the norm classes.  The product is then a streaming read of 6 bytes
// per nonzero (4 when the row and the code share one word) and 12 per row
// (slot word, real diagonal) plus the psi gather.
#include <algorithm>
#include <vector>

#include "edk_rows.cuh"
#include "edk_tma.cuh"

namespace edk {

namespace {

// (row, norm class, phase index) of one off-diagonal target, or false where
// index() returns (0, 1).  Same canonicalisation as the matvec kernels.
template <int BK>
__device__ __forceinline__ bool sell_target(const BasisDev& b, uint32_t s, const uint32_t* binom,
                                            int64_t& pos, int& cls, int& ph) {
  const uint32_t mask = (uint32_t)b.maskL;
  cls = 0;
  ph = 0;
  uint32_t key = s;
  if constexpr (BK == BK_TENSOR) {
    pos = s;
    return true;
  } else if constexpr (BK == BK_PROJ_RANK) {
    if (__popc(s) != b.K) return false;
    pos = colex_rank(s, binom);
    return true;
  } else {
    if constexpr (BK == BK_TRANS0) {
      key = canon_min32(s, b.L, b.A, b.len, mask);
    } else if constexpr (BK == BK_TRANS) {
      int M;
      key = canon_arg32(s, b.L, b.A, b.len, mask, M);
      ph = M;
    } else if constexpr (BK == BK_TRANSPAR) {
      uint32_t Iam, Ibm;
      int Rr, M;
      canon_par32(s, b.L, b.A, b.len, mask, Iam, Rr, Ibm, M);
      double n;
      if (Ibm < Iam) { key = Ibm; n = (double)b.P * __ldg(b.phase + M).x; }
      else { key = Iam; n = __ldg(b.phase + Rr).x; }
      ph = n < 0 ? 1 : 0;
    }
    uint32_t v;
    if (!hash_find(b, key, v)) return false;
    if (b.packed) { pos = (int64_t)(v >> 5); cls = (int)(v & 31u); }
    else { pos = (int64_t)v; cls = 0; }
    return true;
  }
}

template <int BK>
__global__ void __launch_bounds__(256) k_sell_count(BasisDev b, OpDev op, FFParams ff,
                                                    uint8_t* __restrict__ cnt,
                                                    double2* __restrict__ diag) {
  __shared__ uint32_t s_binom[32 * 33];
  if constexpr (BK == BK_PROJ_RANK) {
    fill_binom32(s_binom);
    __syncthreads();
  }
  const uint32_t mask = (uint32_t)b.maskL;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < b.D;
       i += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t st = (BK == BK_TENSOR) ? (uint32_t)i : (uint32_t)__ldg(b.I + i);
    double dr = 0.0, di = 0.0;
    int n = 0;
    for (int f = 0; f < ff.nfam; ++f) {
      const uint32_t X = st, Y = rotl_L(st, ff.d[f], b.L, mask), V = ff.valid[f];
      const uint32_t m1 = ~X & Y & V, m2 = X & ~Y & V;
      const int c0 = __popc(~X & ~Y & V), c1 = __popc(m1), c2 = __popc(m2), c3 = __popc(X & Y & V);
      dr += ff.dval[f][0].x * c0 + ff.dval[f][1].x * c1 + ff.dval[f][2].x * c2 + ff.dval[f][3].x * c3;
      di += ff.dval[f][0].y * c0 + ff.dval[f][1].y * c1 + ff.dval[f][2].y * c2 + ff.dval[f][3].y * c3;
      uint32_t bits = m1 | m2;
      while (bits) {
        const int p = __ffs(bits) - 1;
        bits &= bits - 1;
        const int q = p >= ff.d[f] ? p - ff.d[f] : p - ff.d[f] + b.L;
        int64_t pos;
        int cls, ph;
        if (sell_target<BK>(b, st ^ (1u << p) ^ (1u << q), s_binom, pos, cls, ph)) ++n;
      }
    }
    for (int t = 0; t < op.nterm; ++t) {
      const TermDev* T = op.term + t;
      int c = 0;
      for (int k = 0; k < T->nsites; ++k) c = (c << 1) | (int)((st >> T->bitpos[k]) & 1u);
      const double2 dv = __ldg(op.dval + T->diag_off + c);
      dr += dv.x;
      di += dv.y;
    }
    cnt[i] = (uint8_t)n;
    diag[i] = make_double2(dr, di);
  }
}

template <int BK>
__global__ void __launch_bounds__(256) k_sell_fill(BasisDev b, FFParams ff, int64_t nslices,
                                                   int* __restrict__ rowid,
                                                   const double2* __restrict__ diag_rows,
                                                   double* __restrict__ diag,
                                                   double2* __restrict__ diagc, int rbits,
                                                   const int64_t* __restrict__ off,
                                                   const int* __restrict__ width,
                                                   int* __restrict__ col,
                                                   uint16_t* __restrict__ code, int nph,
                                                   int ncls, int packed) {
  __shared__ uint32_t s_binom[32 * 33];
  if constexpr (BK == BK_PROJ_RANK) {
    fill_binom32(s_binom);
    __syncthreads();
  }
  const uint32_t mask = (uint32_t)b.maskL;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < nslices * 32;
       g += (int64_t)gridDim.x * blockDim.x) {
    const int64_t slice = g >> 5;
    const int lane = (int)(g & 31);
    const int row = rowid[g];
    const int w = width[slice];
    const int64_t base = off[slice] + lane;
    int k = 0;
    if (row >= 0) {
      const uint32_t st = (BK == BK_TENSOR) ? (uint32_t)row : (uint32_t)__ldg(b.I + row);
      // slot word: the row and its own norm class (the class that index() of
      // the representative returns); the diagonal moves to slot order
      int64_t own;
      int cls = 0, ph;
      if constexpr (BK == BK_TRANS0 || BK == BK_TRANS || BK == BK_TRANSPAR) {
        sell_target<BK>(b, st, nullptr, own, cls, ph);
      }
      rowid[g] = (int)((unsigned)row | ((unsigned)cls << rbits));
      const double2 dv = diag_rows[row];
      if (diagc) diagc[g] = dv;
      else diag[g] = dv.x;
      for (int f = 0; f < ff.nfam; ++f) {
        const uint32_t X = st, Y = rotl_L(st, ff.d[f], b.L, mask), V = ff.valid[f];
        uint32_t bits = (~X & Y & V) | (X & ~Y & V);
        while (bits) {
          const int p = __ffs(bits) - 1;
          bits &= bits - 1;
          const int q = p >= ff.d[f] ? p - ff.d[f] : p - ff.d[f] + b.L;
          int64_t pos;
          int cls, ph;
          if (sell_target<BK>(b, st ^ (1u << p) ^ (1u << q), s_binom, pos, cls, ph) && k < w) {
            const int val_id = 2 * f + (int)((st >> p) & 1u);
            const int cd = 1 + (val_id * nph + ph) * ncls + cls;
            if (packed) {
              col[base + (int64_t)k * 32] = (int)(((unsigned)pos << packed) | (unsigned)cd);
            } else {
              col[base + (int64_t)k * 32] = (int)pos;
              code[base + (int64_t)k * 32] = (uint16_t)cd;
            }
            ++k;
          }
        }
      }
    }
    if (row < 0) {
      if (diagc) diagc[g] = make_double2(0.0, 0.0);
      else diag[g] = 0.0;
    }
    for (; k < w; ++k) {  // padding: coefficient 0 on a valid row
      const int r = row >= 0 ? row : 0;
      if (packed) {
        col[base + (int64_t)k * 32] = (int)((unsigned)r << packed);
      } else {
        col[base + (int64_t)k * 32] = r;
        code[base + (int64_t)k * 32] = 0;
      }
    }
  }
}

template <class VT, int PACKED>
__global__ void __launch_bounds__(256) k_sell_apply(BasisDev b, SellDev sd,
                                                    const VT* __restrict__ x, VT* __restrict__ y,
                                                    int64_t ldx, int64_t ldy, int accumulate,
                                                    int64_t blk0) {
  const int64_t slice = (blk0 + blockIdx.x) * 8 + (threadIdx.x >> 5);
  if (slice >= sd.nslices) return;
  sell_slice<VT, PACKED>(b, sd, slice, threadIdx.x & 31, x + (int64_t)blockIdx.y * ldx,
                         y + (int64_t)blockIdx.y * ldy, accumulate);
}

// Failure-detection self-test of the bounded waits the staged kernel uses: one
// block waits on a shared-memory mbarrier whose phase nothing completes (it
// expects two arrivals and receives one), with the same bounded poll; the
// wait runs out, the block records the time-out in *err and returns.  No copy
// is issued, so nothing is in flight when the block exits.
__global__ void k_wait_selftest(uint32_t polls, int* __restrict__ err) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 2);
    mbar_fence_init();
  }
  __syncthreads();
  if (threadIdx.x == 0) mbar_arrive(&bar);
  const bool ok = mbar_wait_bounded(&bar, 0u, polls);
  if (__syncthreads_or(!ok) && threadIdx.x == 0) atomicExch(err, 1);
}

// Materialised product with the entry stream staged through shared memory:
// a persistent block walks windows wbeg + blockIdx.x + i * gridDim.x; thread 0
// copies each window's packed entries (8 slices, contiguous in `col`) with one
// bulk asynchronous copy into one of two stages, two windows ahead, so the
// lanes read their entries from shared memory and only the psi gathers stay
// in the dependent-latency chain.  Waits are bounded: a wait that runs out
// raises *err and the block stops.
template <class VT>
__global__ void __launch_bounds__(256) k_sell_tma(BasisDev b, SellDev sd,
                                                  const VT* __restrict__ x, VT* __restrict__ y,
                                                  int accumulate, int64_t wbeg, int64_t wend,
                                                  int cap_words, int* __restrict__ err) {
  using A = typename VTraits<VT>::A;
  constexpr bool CX = VTraits<VT>::cx;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw);  // two barriers, then the stages
  unsigned* const stage0 = reinterpret_cast<unsigned*>(smem_raw + 128);
  auto stage_buf = [&](int stage) { return stage0 + (stage ? cap_words : 0); };
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  if (t == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_fence_init();
  }
  __syncthreads();
  auto window_end = [&](int64_t w) -> int64_t {  // entry offset past window w
    const int64_t s1 = min(w * 8 + 8, sd.nslices);
    return __ldg(sd.off + s1 - 1) + (int64_t)__ldg(sd.width + s1 - 1) * 32;
  };
  auto issue = [&](int64_t w, int stage) {  // thread 0
    const int64_t e0 = __ldg(sd.off + w * 8);
    const uint32_t bytes = (uint32_t)((window_end(w) - e0) * 4);
    if (bytes) {
      mbar_arrive_expect_tx(&bar[stage], bytes);
      bulk_copy_g2s(stage_buf(stage), reinterpret_cast<const unsigned*>(sd.col) + e0, bytes,
                    &bar[stage]);
    } else {
      mbar_arrive(&bar[stage]);
    }
  };
  const int64_t step = gridDim.x;
  const int64_t w0 = wbeg + blockIdx.x;
  if (t == 0) {
    if (w0 < wend) issue(w0, 0);
    if (w0 + step < wend) issue(w0 + step, 1);
  }
  const int sh = sd.packed;
  const unsigned cm = (1u << sh) - 1u;
  int i = 0;
  for (int64_t w = w0; w < wend; w += step, ++i) {
    const int stage = i & 1;
    const bool ok = mbar_wait_bounded(&bar[stage], (uint32_t)((i >> 1) & 1), 1u << 20);
    if (__syncthreads_or(!ok)) {
      // a copy that does not complete means the device is already in a bad
      // state; record it, give this block's copies in flight (this window's
      // and, when one was issued, the next window's) another bounded wait, and
      // stop
      if (t == 0) atomicExch(err, 1);
      mbar_wait_bounded(&bar[stage], (uint32_t)((i >> 1) & 1), 1u << 20);
      if (w + step < wend)
        mbar_wait_bounded(&bar[stage ^ 1], (uint32_t)(((i + 1) >> 1) & 1), 1u << 20);
      __syncthreads();
      return;
    }
    const int64_t slice = w * 8 + warp;
    if (slice < sd.nslices) {
      const int64_t eoff = __ldg(sd.off + slice) - __ldg(sd.off + w * 8);
      const unsigned* ep = stage_buf(stage) + eoff + lane;
      const int wd = __ldg(sd.width + slice);
      const unsigned rc = __ldg(sd.rowid + slice * 32 + lane);
      A ar = 0, ai = 0;
      auto term = [&](unsigned e) {
        const int c = (int)(e >> sh), code = (int)(e & cm);
        const Cx<A> xv = ldv(x + c);
        if constexpr (CX) {
          A vr, vi;
          if constexpr (sizeof(A) == 8) {
            const double2 v = __ldg(sd.vt64 + code);
            vr = v.x; vi = v.y;
          } else {
            const float2 v = __ldg(sd.vt32 + code);
            vr = v.x; vi = v.y;
          }
          ar += vr * xv.r + vi * xv.i;  // conj(v) * x
          ai += vr * xv.i - vi * xv.r;
        } else {
          A vr;
          if constexpr (sizeof(A) == 8)
            vr = __ldg(reinterpret_cast<const double*>(sd.vt64) + 2 * code);
          else
            vr = __ldg(reinterpret_cast<const float*>(sd.vt32) + 2 * code);
          ar += vr * xv.r;
        }
      };
      int k = 0;
      for (; k + 4 <= wd; k += 4) {
        const unsigned e0 = ep[(k + 0) * 32], e1 = ep[(k + 1) * 32];
        const unsigned e2 = ep[(k + 2) * 32], e3 = ep[(k + 3) * 32];
        term(e0);
        term(e1);
        term(e2);
        term(e3);
      }
      for (; k < wd; ++k) term(ep[k * 32]);
      if (rc != ~0u) {
        const int64_t row = rc & ((1u << sd.rbits) - 1u);
        const A invR = (A)__ldg(sd.rinv + (rc >> sd.rbits));
        const double2 d =
            sd.diagc ? __ldg(sd.diagc + slice * 32 + lane) : make_double2(__ldg(sd.diag + slice * 32 + lane), 0.0);
        const Cx<A> xi = ldv(x + row);
        Cx<A> out{ar * invR + (A)d.x * xi.r + (A)d.y * xi.i, (A)0};
        if constexpr (CX) out.i = ai * invR + (A)d.x * xi.i - (A)d.y * xi.r;
        if (accumulate) {
          const Cx<A> yo = ldout(y + row);
          out.r += yo.r;
          out.i += yo.i;
        }
        stv(y + row, out);
      }
    }
    __syncthreads();  // every lane is done with this stage
    if (t == 0 && w + 2 * step < wend) {
      fence_proxy_async_smem();
      issue(w + 2 * step, stage);
    }
  }
}

// Value mode (any operator in the row-gather form, any basis): the row
// expansion of the generic kernel, stored with explicit coefficients
// c = v * phase * R[target] / R[row], y_row += conj(c) x[target].
template <int BK, class S>
__global__ void __launch_bounds__(256) k_vsell_count(BasisDev b, OpDev op, int* __restrict__ cnt,
                                                     double2* __restrict__ diag) {
  __shared__ uint32_t s_binom[(BK == BK_PROJ_RANK) ? 32 * 33 : 1];
  if constexpr (BK == BK_PROJ_RANK) {
    fill_binom32(s_binom);
    __syncthreads();
  }
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < b.D;
       i += (int64_t)gridDim.x * blockDim.x) {
    const S s = (BK == BK_TENSOR) ? (S)i : (S)__ldg(b.I + i);
    double dr = 0.0, di = 0.0;
    int n = 0;
    expand_row<BK, S>(b, op, s, s_binom, dr, di, [&](const Hit&, double, double) { ++n; });
    cnt[i] = n;
    diag[i] = make_double2(dr, di);
  }
}

template <int BK, class S>
__global__ void __launch_bounds__(256) k_vsell_fill(BasisDev b, OpDev op, int64_t nslices,
                                                    const int* __restrict__ rowid,
                                                    const int64_t* __restrict__ off,
                                                    const int* __restrict__ width,
                                                    const double2* __restrict__ drows,
                                                    double* __restrict__ diag,
                                                    double2* __restrict__ diagc,
                                                    int* __restrict__ col,
                                                    double2* __restrict__ val) {
  __shared__ uint32_t s_binom[(BK == BK_PROJ_RANK) ? 32 * 33 : 1];
  if constexpr (BK == BK_PROJ_RANK) {
    fill_binom32(s_binom);
    __syncthreads();
  }
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < nslices * 32;
       g += (int64_t)gridDim.x * blockDim.x) {
    const int64_t slice = g >> 5;
    const int row = rowid[g];
    const int w = width[slice];
    const int64_t base = off[slice] + (g & 31);
    int k = 0;
    if (row >= 0) {
      const S s = (BK == BK_TENSOR) ? (S)row : (S)__ldg(b.I + row);
      const double invRi = b.R ? 1.0 / __ldg(b.R + row) : 1.0;
      double dr = 0.0, di = 0.0;
      expand_row<BK, S>(b, op, s, s_binom, dr, di, [&](const Hit& h, double vr, double vi) {
        if (k >= w) return;
        const double ratio = h.rpos * invRi;
        col[base + (int64_t)k * 32] = (int)h.pos;
        val[base + (int64_t)k * 32] = make_double2((vr * h.pre - vi * h.pim) * ratio,
                                                   (vr * h.pim + vi * h.pre) * ratio);
        ++k;
      });
      const double2 d = drows[row];
      if (diagc) diagc[g] = d;
      else diag[g] = d.x;
    } else {
      if (diagc) diagc[g] = make_double2(0.0, 0.0);
      else diag[g] = 0.0;
    }
    for (; k < w; ++k) {  // padding: coefficient 0 on a valid row
      col[base + (int64_t)k * 32] = row >= 0 ? row : 0;
      val[base + (int64_t)k * 32] = make_double2(0.0, 0.0);
    }
  }
}

int gridn(int64_t n) {
  int64_t g = (n + 255) / 256;
  return (int)std::max<int64_t>(1, std::min<int64_t>(g, 148 * 32));
}

}  // namespace

// the staged kernel for windows [w0, w1); false when it does not apply
template <class VT>
static bool launch_sell_tma(edk_operator* op, const void* x, void* y, int accumulate,
                            int64_t w0, int64_t w1, cudaStream_t st, edk_status& rc) {
  const SellDev& sd = op->dev.sell;
  rc = EDK_OK;
  if (!sd.packed || !op->sell_tma || !op->sell_tma_ok || w1 <= w0) return false;
  const size_t smem = 128 + 2 * (size_t)op->sell_wincap * 4;
  static thread_local int attr_dev = -1;
  int dev = 0;
  cudaGetDevice(&dev);
  if (attr_dev != dev) {
    cudaFuncSetAttribute(k_sell_tma<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
    cudaFuncSetAttribute(k_sell_tma<double2>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
    cudaFuncSetAttribute(k_sell_tma<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
    cudaFuncSetAttribute(k_sell_tma<float2>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
    attr_dev = dev;
  }
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sell_tma<VT>, 256, smem) !=
          cudaSuccess || per_sm < 1)
    return false;
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const int64_t grid = std::min<int64_t>(w1 - w0, (int64_t)nsm * per_sm);
  k_sell_tma<VT><<<(unsigned)grid, 256, smem, st>>>(op->b->dev, sd, static_cast<const VT*>(x),
                                                    static_cast<VT*>(y), accumulate, w0, w1,
                                                    (int)op->sell_wincap, op->s_err.as<int>());
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error(std::string("k_sell_tma launch failed: ") + cudaGetErrorString(e));
    rc = EDK_CUDA_ERROR;
  }
  return true;
}

template <class VT>
static edk_status launch_sell(const BasisDev& b, const SellDev& sd, const void* x, void* y,
                              int64_t nvec, int64_t ldx, int64_t ldy, int accumulate,
                              cudaStream_t st) {
  for (int64_t k0 = 0; k0 < nvec; k0 += 65535) {
    int64_t nk = std::min<int64_t>(nvec - k0, 65535);
    dim3 grid((unsigned)((sd.nslices + 7) / 8), (unsigned)nk);
    const VT* xs = static_cast<const VT*>(x) + k0 * ldx;
    VT* ys = static_cast<VT*>(y) + k0 * ldy;
    if (sd.val)
      k_sell_apply<VT, 2><<<grid, 256, 0, st>>>(b, sd, xs, ys, ldx, ldy, accumulate, 0);
    else if (sd.packed)
      k_sell_apply<VT, 1><<<grid, 256, 0, st>>>(b, sd, xs, ys, ldx, ldy, accumulate, 0);
    else
      k_sell_apply<VT, 0><<<grid, 256, 0, st>>>(b, sd, xs, ys, ldx, ldy, accumulate, 0);
    EDK_TRY_CUDA(cudaGetLastError());
  }
  return EDK_OK;
}

// one block = one 256-row window (8 slices), so rows [row0, row1) with
// row0 a multiple of 256 are windows row0/256 ..
template <class VT>
static edk_status launch_sell_rows(const BasisDev& b, const SellDev& sd, const void* x, void* y,
                                   int64_t row0, int64_t row1, int accumulate, cudaStream_t st) {
  const int64_t w0 = row0 / 256, w1 = (row1 + 255) / 256;
  if (w1 <= w0) return EDK_OK;
  const VT* xs = static_cast<const VT*>(x);
  VT* ys = static_cast<VT*>(y);
  const int64_t D = b.D;
  if (sd.val)
    k_sell_apply<VT, 2><<<(unsigned)(w1 - w0), 256, 0, st>>>(b, sd, xs, ys, D, D, accumulate, w0);
  else if (sd.packed)
    k_sell_apply<VT, 1><<<(unsigned)(w1 - w0), 256, 0, st>>>(b, sd, xs, ys, D, D, accumulate, w0);
  else
    k_sell_apply<VT, 0><<<(unsigned)(w1 - w0), 256, 0, st>>>(b, sd, xs, ys, D, D, accumulate, w0);
  EDK_TRY_CUDA(cudaGetLastError());
  return EDK_OK;
}

edk_status apply_sell_rows(edk_operator* op, int dtype, const void* x, void* y, int64_t row0,
                           int64_t row1, int accumulate, cudaStream_t st) {
  const BasisDev& b = op->b->dev;
  const SellDev& sd = op->dev.sell;
  {
    const int64_t w0 = row0 / 256, w1 = (row1 + 255) / 256;
    edk_status rc = EDK_OK;
    bool done = false;
    switch (dtype) {
      case EDK_F64: done = launch_sell_tma<double>(op, x, y, accumulate, w0, w1, st, rc); break;
      case EDK_C128: done = launch_sell_tma<double2>(op, x, y, accumulate, w0, w1, st, rc); break;
      case EDK_F32: done = launch_sell_tma<float>(op, x, y, accumulate, w0, w1, st, rc); break;
      case EDK_C64: done = launch_sell_tma<float2>(op, x, y, accumulate, w0, w1, st, rc); break;
    }
    if (done) return rc;
  }
  switch (dtype) {
    case EDK_F64: return launch_sell_rows<double>(b, sd, x, y, row0, row1, accumulate, st);
    case EDK_C128: return launch_sell_rows<double2>(b, sd, x, y, row0, row1, accumulate, st);
    case EDK_F32: return launch_sell_rows<float>(b, sd, x, y, row0, row1, accumulate, st);
    case EDK_C64: return launch_sell_rows<float2>(b, sd, x, y, row0, row1, accumulate, st);
  }
  set_error("apply: unknown dtype");
  return EDK_INVALID_ARG;
}

edk_status apply_sell(edk_operator* op, int dtype, const void* x, void* y, int64_t nvec,
                      int64_t ldx, int64_t ldy, int accumulate, cudaStream_t st) {
  const BasisDev& b = op->b->dev;
  const SellDev& sd = op->dev.sell;
  if (nvec == 1) {
    const int64_t nwin = (sd.nslices + 7) / 8;
    edk_status rc = EDK_OK;
    bool done = false;
    switch (dtype) {
      case EDK_F64: done = launch_sell_tma<double>(op, x, y, accumulate, 0, nwin, st, rc); break;
      case EDK_C128: done = launch_sell_tma<double2>(op, x, y, accumulate, 0, nwin, st, rc); break;
      case EDK_F32: done = launch_sell_tma<float>(op, x, y, accumulate, 0, nwin, st, rc); break;
      case EDK_C64: done = launch_sell_tma<float2>(op, x, y, accumulate, 0, nwin, st, rc); break;
    }
    if (done) return rc;
  }
  switch (dtype) {
    case EDK_F64: return launch_sell<double>(b, sd, x, y, nvec, ldx, ldy, accumulate, st);
    case EDK_C128: return launch_sell<double2>(b, sd, x, y, nvec, ldx, ldy, accumulate, st);
    case EDK_F32: return launch_sell<float>(b, sd, x, y, nvec, ldx, ldy, accumulate, st);
    case EDK_C64: return launch_sell<float2>(b, sd, x, y, nvec, ldx, ldy, accumulate, st);
  }
  set_error("apply: unknown dtype");
  return EDK_INVALID_ARG;
}

static edk_status materialize_values(edk_operator* op);

static edk_status materialize(edk_operator* op) {
  edk_basis* bb = op->b;
  const BasisDev& b = bb->dev;
  const int bk = b.bk;
  if (!op->gather) {
    set_error("edk_operator_materialize: the operator is not Hermitian (or not symmetric) in "
              "this basis; only the row-gather form is materialised");
    return EDK_UNSUPPORTED;
  }
  const bool coded = op->ff_ok && bb->L <= 32 &&
                     (bk == BK_TENSOR || bk == BK_PROJ_RANK || bk == BK_PROJ_HASH ||
                      bk == BK_TRANS0 || bk == BK_TRANS || bk == BK_TRANSPAR);
  const bool symm = bk == BK_TRANS0 || bk == BK_TRANS || bk == BK_TRANSPAR;
  // bond-family operators: coefficient codes; everything else: explicit values
  if (!coded || (symm && !b.packed)) return materialize_values(op);
  const FFParams& ff = *reinterpret_cast<const FFParams*>(op->ff_params.data());
  const int nval = 2 * ff.nfam;
  const int nph = (bk == BK_TRANS) ? b.len : (bk == BK_TRANSPAR ? 2 : 1);
  const int ncls = symm ? std::max(1, b.nclass) : 1;
  const int64_t ncode = 1 + (int64_t)nval * nph * ncls;
  if (ncode > 65535) return materialize_values(op);
  cudaStream_t st = op->stream;
  const int64_t D = b.D;
  // slot word row | class << rbits: 27 row bits under translations (<= 32
  // norm classes), 31 otherwise (one class, R = 1)
  const int rbits = symm ? 27 : 31;
  if (D >= (int64_t(1) << rbits)) {
    set_error("edk_operator_materialize: basis dimension too large for the sliced-ELL row index");
    return EDK_UNSUPPORTED;
  }
  DevBuf cnt, drows;
  EDK_RETURN_IF(cnt.alloc(std::max<int64_t>(D, 1)));
  EDK_RETURN_IF(drows.alloc(std::max<int64_t>(D, 1) * sizeof(double2)));
#define EDK_CNT(BK)                                                                             \
  case BK:                                                                                      \
    k_sell_count<BK><<<gridn(D), 256, 0, st>>>(b, op->dev, ff, cnt.as<uint8_t>(),              \
                                               drows.as<double2>());                           \
    break;
  switch (bk) {
    EDK_CNT(BK_TENSOR)
    EDK_CNT(BK_PROJ_RANK)
    EDK_CNT(BK_PROJ_HASH)
    EDK_CNT(BK_TRANS0)
    EDK_CNT(BK_TRANS)
    EDK_CNT(BK_TRANSPAR)
  }
#undef EDK_CNT
  EDK_TRY_CUDA(cudaGetLastError());
  std::vector<uint8_t> hc(D);
  if (D > 0) EDK_TRY_CUDA(cudaMemcpyAsync(hc.data(), cnt.p, D, cudaMemcpyDeviceToHost, st));
  EDK_TRY_CUDA(cudaStreamSynchronize(st));
  // rows sorted by length (descending) inside windows of 256 rows
  const int64_t nwin = (D + 255) / 256;
  const int64_t nslices = nwin * 8;
  std::vector<int> rowid((size_t)nslices * 32, -1), width(nslices, 0);
  std::vector<int64_t> off(nslices, 0);
  int64_t E = 0;
  for (int64_t wdx = 0; wdx < nwin; ++wdx) {
    const int64_t r0 = wdx * 256, r1 = std::min<int64_t>(D, r0 + 256);
    int bins[257] = {0};
    for (int64_t r = r0; r < r1; ++r) bins[256 - hc[r]]++;
    int start[257];
    int acc = 0;
    for (int k = 0; k < 257; ++k) { start[k] = acc; acc += bins[k]; }
    for (int64_t r = r0; r < r1; ++r) rowid[(size_t)wdx * 256 + start[256 - hc[r]]++] = (int)r;
    for (int sl = 0; sl < 8; ++sl) {
      const int64_t s = wdx * 8 + sl;
      const int first = rowid[(size_t)s * 32];
      width[s] = first >= 0 ? hc[first] : 0;
      off[s] = E;
      E += (int64_t)width[s] * 32;
    }
  }
  EDK_RETURN_IF(op->s_rowid.alloc(rowid.size() * sizeof(int)));
  EDK_RETURN_IF(op->s_width.alloc(width.size() * sizeof(int)));
  EDK_RETURN_IF(op->s_off.alloc(off.size() * sizeof(int64_t)));
  // packed entries: code in the low `cbits` bits, target row above them
  int cbits = 1;
  while ((int64_t(1) << cbits) < ncode) ++cbits;
  const int packed = (D <= (int64_t(1) << (32 - cbits))) ? cbits : 0;
  EDK_RETURN_IF(op->s_col.alloc(std::max<int64_t>(E, 1) * sizeof(int)));
  if (!packed) EDK_RETURN_IF(op->s_code.alloc(std::max<int64_t>(E, 1) * sizeof(uint16_t)));
  else op->s_code.release();
  EDK_TRY_CUDA(cudaMemcpyAsync(op->s_rowid.p, rowid.data(), rowid.size() * sizeof(int),
                               cudaMemcpyHostToDevice, st));
  EDK_TRY_CUDA(cudaMemcpyAsync(op->s_width.p, width.data(), width.size() * sizeof(int),
                               cudaMemcpyHostToDevice, st));
  EDK_TRY_CUDA(cudaMemcpyAsync(op->s_off.p, off.data(), off.size() * sizeof(int64_t),
                               cudaMemcpyHostToDevice, st));
  const bool dcx = op->is_complex;
  EDK_RETURN_IF(op->s_diag.alloc(nslices * 32 * (dcx ? sizeof(double2) : sizeof(double))));
  double* dre = dcx ? nullptr : op->s_diag.as<double>();
  double2* dcp = dcx ? op->s_diag.as<double2>() : nullptr;
#define EDK_FILL(BK)                                                                            \
  case BK:                                                                                      \
    k_sell_fill<BK><<<gridn(nslices * 32), 256, 0, st>>>(                                       \
        b, ff, nslices, op->s_rowid.as<int>(), drows.as<double2>(), dre, dcp, rbits,           \
        op->s_off.as<int64_t>(), op->s_width.as<int>(),                                         \
        op->s_col.as<int>(), op->s_code.as<uint16_t>(), nph, ncls, packed);                    \
    break;
  switch (bk) {
    EDK_FILL(BK_TENSOR)
    EDK_FILL(BK_PROJ_RANK)
    EDK_FILL(BK_PROJ_HASH)
    EDK_FILL(BK_TRANS0)
    EDK_FILL(BK_TRANS)
    EDK_FILL(BK_TRANSPAR)
  }
#undef EDK_FILL
  EDK_TRY_CUDA(cudaGetLastError());
  // coefficient table val * phase * R[target]
  std::vector<double2> ph(nph, make_double2(1.0, 0.0));
  if (bk == BK_TRANS && b.len > 0)
    EDK_TRY_CUDA(cudaMemcpyAsync(ph.data(), b.phase, nph * sizeof(double2), cudaMemcpyDeviceToHost, st));
  if (bk == BK_TRANSPAR) ph[1] = make_double2(-1.0, 0.0);
  EDK_TRY_CUDA(cudaStreamSynchronize(st));
  std::vector<double2> vt((size_t)ncode, make_double2(0.0, 0.0));
  std::vector<float2> vt32((size_t)ncode, make_float2(0.f, 0.f));
  for (int v = 0; v < nval; ++v) {
    const int f = v / 2;
    const double2 val = (v % 2 == 0) ? ff.v1[f] : ff.v2[f];
    for (int p = 0; p < nph; ++p)
      for (int c = 0; c < ncls; ++c) {
        const double r = symm ? b.Rcls[c] : 1.0;
        const double re = (val.x * ph[p].x - val.y * ph[p].y) * r;
        const double im = (val.x * ph[p].y + val.y * ph[p].x) * r;
        const size_t code = 1 + ((size_t)v * nph + p) * ncls + c;
        vt[code] = make_double2(re, im);
        vt32[code] = make_float2((float)re, (float)im);
      }
  }
  std::vector<double> rinv(32, 1.0);
  for (int c = 0; c < ncls; ++c) rinv[c] = symm ? 1.0 / b.Rcls[c] : 1.0;
  EDK_RETURN_IF(op->s_rinv.alloc(rinv.size() * sizeof(double)));
  EDK_TRY_CUDA(cudaMemcpyAsync(op->s_rinv.p, rinv.data(), rinv.size() * sizeof(double),
                               cudaMemcpyHostToDevice, st));
  EDK_RETURN_IF(op->s_vt64.alloc(vt.size() * sizeof(double2)));
  EDK_RETURN_IF(op->s_vt32.alloc(vt32.size() * sizeof(float2)));
  EDK_TRY_CUDA(cudaMemcpyAsync(op->s_vt64.p, vt.data(), vt.size() * sizeof(double2),
                               cudaMemcpyHostToDevice, st));
  EDK_TRY_CUDA(cudaMemcpyAsync(op->s_vt32.p, vt32.data(), vt32.size() * sizeof(float2),
                               cudaMemcpyHostToDevice, st));
  EDK_TRY_CUDA(cudaStreamSynchronize(st));
  op->s_val.release();
  SellDev& sd = op->dev.sell;
  sd = SellDev{};
  sd.nslices = nslices;
  sd.packed = packed;
  sd.rbits = rbits;
  sd.rowid = op->s_rowid.as<unsigned>();
  sd.off = op->s_off.as<int64_t>();
  sd.width = op->s_width.as<int>();
  sd.col = op->s_col.as<int>();
  sd.code = op->s_code.as<uint16_t>();
  sd.diag = dre;
  sd.diagc = dcp;
  sd.rinv = op->s_rinv.as<double>();
  sd.vt64 = op->s_vt64.as<double2>();
  sd.vt32 = op->s_vt32.as<float2>();
  // largest window (8 slices) in entries: the stage size of the staged kernel
  int64_t wincap = 0;
  for (int64_t wdx = 0; wdx < nwin; ++wdx) {
    int64_t ew = 0;
    for (int sl = 0; sl < 8; ++sl) ew += (int64_t)width[wdx * 8 + sl] * 32;
    wincap = std::max(wincap, ew);
  }
  op->sell_wincap = wincap;
  op->sell_tma_ok = packed != 0 && 128 + 2 * wincap * 4 <= 200 * 1024;
  op->sell_tma = false;  // the autotuner enables it where it measures faster
  EDK_RETURN_IF(op->s_err.alloc(sizeof(int)));
  EDK_TRY_CUDA(cudaMemsetAsync(op->s_err.p, 0, sizeof(int), st));
  EDK_TRY_CUDA(cudaStreamSynchronize(st));
  op->sell_entries = E;
  op->sell_ok = true;
  return EDK_OK;
}

}  // namespace edk

using namespace edk;

namespace edk {
// Explicit-value sliced ELL for any operator in the row-gather form.
static edk_status materialize_values(edk_operator* op) {
  edk_basis* bb = op->b;
  const BasisDev& b = bb->dev;
  const int bk = b.bk;
  cudaStream_t st = op->stream;
  const int64_t D = b.D;
  if (D >= (int64_t(1) << 31)) {
    set_error("edk_operator_materialize: basis dimension too large for the sliced-ELL row index");
    return EDK_UNSUPPORTED;
  }
  EDK_RETURN_IF(check_basis_dev(b));
  const bool wide = bb->L > 32;
  DevBuf cnt, drows;
  EDK_RETURN_IF(cnt.alloc(std::max<int64_t>(D, 1) * sizeof(int)));
  EDK_RETURN_IF(drows.alloc(std::max<int64_t>(D, 1) * sizeof(double2)));
#define EDK_VCNT(BK)                                                                            \
  case BK:                                                                                      \
    if (wide) k_vsell_count<BK, uint64_t><<<gridn(D), 256, 0, st>>>(b, op->dev, cnt.as<int>(),  \
                                                                   drows.as<double2>());       \
    else k_vsell_count<BK, uint32_t><<<gridn(D), 256, 0, st>>>(b, op->dev, cnt.as<int>(),       \
                                                              drows.as<double2>());            \
    break;
  switch (bk) {
    EDK_VCNT(BK_TENSOR)
    EDK_VCNT(BK_PROJ_RANK)
    EDK_VCNT(BK_PROJ_HASH)
    EDK_VCNT(BK_TRANS0)
    EDK_VCNT(BK_TRANS)
    EDK_VCNT(BK_TRANSPAR)
    EDK_VCNT(BK_ABELIAN)
    default:
      set_error("edk_operator_materialize: unknown lookup kind");
      return EDK_INVALID_ARG;
  }
#undef EDK_VCNT
  EDK_TRY_CUDA(cudaGetLastError());
  std::vector<int> hc(D);
  if (D > 0) EDK_TRY_CUDA(cudaMemcpyAsync(hc.data(), cnt.p, D * sizeof(int), cudaMemcpyDeviceToHost, st));
  EDK_TRY_CUDA(cudaStreamSynchronize(st));
  const int64_t nwin = (D + 255) / 256;
  const int64_t nslices = nwin * 8;
  std::vector<int> rowid((size_t)nslices * 32, -1), width(nslices, 0);
  std::vector<int64_t> off(nslices, 0);
  int64_t E = 0;
  std::vector<int> order;
  for (int64_t wdx = 0; wdx < nwin; ++wdx) {
    const int64_t r0 = wdx * 256, r1 = std::min<int64_t>(D, r0 + 256);
    order.clear();
    for (int64_t r = r0; r < r1; ++r) order.push_back((int)r);
    std::stable_sort(order.begin(), order.end(), [&](int a, int c) { return hc[a] > hc[c]; });
    for (size_t q = 0; q < order.size(); ++q) rowid[(size_t)wdx * 256 + q] = order[q];
    for (int sl = 0; sl < 8; ++sl) {
      const int64_t s = wdx * 8 + sl;
      const int first = rowid[(size_t)s * 32];
      width[s] = first >= 0 ? hc[first] : 0;
      off[s] = E;
      E += (int64_t)width[s] * 32;
    }
  }
  if (E >= (int64_t(1) << 40)) {
    set_error("edk_operator_materialize: too many entries");
    return EDK_UNSUPPORTED;
  }
  EDK_RETURN_IF(op->s_rowid.alloc(rowid.size() * sizeof(int)));
  EDK_RETURN_IF(op->s_width.alloc(width.size() * sizeof(int)));
  EDK_RETURN_IF(op->s_off.alloc(off.size() * sizeof(int64_t)));
  EDK_RETURN_IF(op->s_col.alloc(std::max<int64_t>(E, 1) * sizeof(int)));
  EDK_RETURN_IF(op->s_val.alloc(std::max<int64_t>(E, 1) * sizeof(double2)));
  op->s_code.release();
  const bool dcx = op->is_complex;
  EDK_RETURN_IF(op->s_diag.alloc(nslices * 32 * (dcx ? sizeof(double2) : sizeof(double))));
  double* dre = dcx ? nullptr : op->s_diag.as<double>();
  double2* dcp = dcx ? op->s_diag.as<double2>() : nullptr;
  EDK_TRY_CUDA(cudaMemcpyAsync(op->s_rowid.p, rowid.data(), rowid.size() * sizeof(int),
                               cudaMemcpyHostToDevice, st));
  EDK_TRY_CUDA(cudaMemcpyAsync(op->s_width.p, width.data(), width.size() * sizeof(int),
                               cudaMemcpyHostToDevice, st));
  EDK_TRY_CUDA(cudaMemcpyAsync(op->s_off.p, off.data(), off.size() * sizeof(int64_t),
                               cudaMemcpyHostToDevice, st));
#define EDK_VFILL(BK)                                                                           \
  case BK:                                                                                      \
    if (wide)                                                                                   \
      k_vsell_fill<BK, uint64_t><<<gridn(nslices * 32), 256, 0, st>>>(                          \
          b, op->dev, nslices, op->s_rowid.as<int>(), op->s_off.as<int64_t>(),                 \
          op->s_width.as<int>(), drows.as<double2>(), dre, dcp, op->s_col.as<int>(),           \
          op->s_val.as<double2>());                                                            \
    else                                                                                        \
      k_vsell_fill<BK, uint32_t><<<gridn(nslices * 32), 256, 0, st>>>(                          \
          b, op->dev, nslices, op->s_rowid.as<int>(), op->s_off.as<int64_t>(),                 \
          op->s_width.as<int>(), drows.as<double2>(), dre, dcp, op->s_col.as<int>(),           \
          op->s_val.as<double2>());                                                            \
    break;
  switch (bk) {
    EDK_VFILL(BK_TENSOR)
    EDK_VFILL(BK_PROJ_RANK)
    EDK_VFILL(BK_PROJ_HASH)
    EDK_VFILL(BK_TRANS0)
    EDK_VFILL(BK_TRANS)
    EDK_VFILL(BK_TRANSPAR)
    EDK_VFILL(BK_ABELIAN)
  }
#undef EDK_VFILL
  EDK_TRY_CUDA(cudaGetLastError());
  std::vector<double> rinv(32, 1.0);
  EDK_RETURN_IF(op->s_rinv.alloc(rinv.size() * sizeof(double)));
  EDK_TRY_CUDA(cudaMemcpyAsync(op->s_rinv.p, rinv.data(), rinv.size() * sizeof(double),
                               cudaMemcpyHostToDevice, st));
  std::vector<double2> vt(1, make_double2(0.0, 0.0));
  std::vector<float2> vt32(1, make_float2(0.f, 0.f));
  EDK_RETURN_IF(op->s_vt64.alloc(sizeof(double2)));
  EDK_RETURN_IF(op->s_vt32.alloc(sizeof(float2)));
  EDK_TRY_CUDA(cudaMemcpyAsync(op->s_vt64.p, vt.data(), sizeof(double2), cudaMemcpyHostToDevice, st));
  EDK_TRY_CUDA(cudaMemcpyAsync(op->s_vt32.p, vt32.data(), sizeof(float2), cudaMemcpyHostToDevice, st));
  EDK_RETURN_IF(op->s_err.alloc(sizeof(int)));
  EDK_TRY_CUDA(cudaMemsetAsync(op->s_err.p, 0, sizeof(int), st));
  EDK_TRY_CUDA(cudaStreamSynchronize(st));
  SellDev& sd = op->dev.sell;
  sd = SellDev{};
  sd.nslices = nslices;
  sd.packed = 0;
  sd.rbits = 31;
  sd.rowid = op->s_rowid.as<unsigned>();
  sd.off = op->s_off.as<int64_t>();
  sd.width = op->s_width.as<int>();
  sd.col = op->s_col.as<int>();
  sd.code = nullptr;
  sd.val = op->s_val.as<double2>();
  sd.diag = dre;
  sd.diagc = dcp;
  sd.rinv = op->s_rinv.as<double>();
  sd.vt64 = op->s_vt64.as<double2>();
  sd.vt32 = op->s_vt32.as<float2>();
  op->sell_wincap = 0;
  op->sell_tma_ok = false;
  op->sell_tma = false;
  op->sell_entries = E;
  op->sell_ok = true;
  return EDK_OK;
}
}  // namespace edk

extern "C" edk_status edk_operator_materialize(edk_operator* op, int32_t enable,
                                               int64_t* entries) {
  EDK_CHECK_ARG(op != nullptr, "edk_operator_materialize: NULL operator");
  std::lock_guard<std::mutex> lk(op->mu);
  if (!enable) {
    op->sell_ok = false;
    op->dev.sell = SellDev{};
    op->s_rowid.release(); op->s_off.release(); op->s_width.release(); op->s_col.release();
    op->s_code.release(); op->s_diag.release(); op->s_vt64.release(); op->s_vt32.release();
    op->s_rinv.release(); op->s_val.release();
    op->sell_entries = 0;
    if (entries) *entries = 0;
    return EDK_OK;
  }
  if (!op->sell_ok) EDK_RETURN_IF(materialize(op));
  if (entries) *entries = op->sell_entries;
  return EDK_OK;
}

extern "C" edk_status edk_selftest_bounded_wait(uint32_t polls) {
  EDK_CHECK_ARG(polls >= 1 && polls <= (1u << 24),
                "edk_selftest_bounded_wait: polls out of 1..2^24");
  DevBuf err;
  EDK_RETURN_IF(err.alloc(sizeof(int)));
  cudaStream_t st = nullptr;
  EDK_TRY_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  int flag = 0;
  cudaError_t e = cudaMemsetAsync(err.p, 0, sizeof(int), st);
  if (e == cudaSuccess) {
    edk::k_wait_selftest<<<1, 128, 0, st>>>(polls, err.as<int>());
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(&flag, err.p, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaStreamDestroy(st);
  if (e != cudaSuccess) {
    set_error(std::string("edk_selftest_bounded_wait: ") + cudaGetErrorString(e));
    return EDK_CUDA_ERROR;
  }
  if (flag) {
    set_error("bounded wait ran out after " + std::to_string(polls) +
              " polls: the awaited barrier phase never completed (self-test)");
    return EDK_TIMEOUT;
  }
  return EDK_OK;
}
