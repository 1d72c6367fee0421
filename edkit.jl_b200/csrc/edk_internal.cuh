// edk_internal.cuh — device-side data layout shared by the libedk sources.
//
// HBM layout of one basis (sector):
//   I     uint64[D]   sorted 0-based representative states (EDKit's I - 1)
//   R     f64[D]      orbit norms (symmetric kinds only)
//   htab  slots       open-addressing table state -> (row << 5 | norm class)
//   phase c128[len]   translation phase table C (or generator phase tables)
// Vectors are column-major blocks x[row + k*ld] of f64 / c128 / f32 / c64.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/edk.h"

namespace edk {

void set_error(const std::string& msg);
const std::string& get_error();

#define EDK_TRY_CUDA(call)                                                          \
  do {                                                                              \
    cudaError_t e_ = (call);                                                        \
    if (e_ != cudaSuccess) {                                                        \
      edk::set_error(std::string(#call) + " failed: " + cudaGetErrorString(e_));    \
      return (e_ == cudaErrorMemoryAllocation) ? EDK_OOM : EDK_CUDA_ERROR;          \
    }                                                                               \
  } while (0)

#define EDK_CHECK_ARG(cond, msg)                 \
  do {                                           \
    if (!(cond)) {                               \
      edk::set_error(msg);                       \
      return EDK_INVALID_ARG;                    \
    }                                            \
  } while (0)

#define EDK_RETURN_IF(st) \
  do {                    \
    edk_status s_ = (st); \
    if (s_ != EDK_OK) return s_; \
  } while (0)

// Owning device buffer.  alloc() uses cudaMalloc; alloc_async() takes the
// memory from the device's stream-ordered pool on stream `s` (workspace of the
// Lanczos/Krylov drivers, reused across calls without new allocations).
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  cudaStream_t pool_stream = nullptr;
  bool pooled = false;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  void release() {
    if (p) {
      if (pooled) cudaFreeAsync(p, pool_stream);
      else cudaFree(p);
    }
    p = nullptr;
    bytes = 0;
    pooled = false;
  }
  edk_status alloc_async(size_t n, cudaStream_t s);
  edk_status alloc(size_t n) {
    release();
    if (n == 0) return EDK_OK;
    cudaError_t e = cudaMalloc(&p, n);
    if (e != cudaSuccess) {
      cudaGetLastError();  // an allocation failure is not sticky: clear it for later checks
      p = nullptr;
      set_error(std::string("cudaMalloc(") + std::to_string(n) + " bytes) failed: " +
                cudaGetErrorString(e));
      return EDK_OOM;
    }
    bytes = n;
    return EDK_OK;
  }
  template <class T> T* as() const { return reinterpret_cast<T*>(p); }
};

// keep freed pool memory cached in the process (set once per device)
inline void keep_pool_memory() {
  static bool done[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64 || done[dev]) return;
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
    uint64_t thr = ~0ull;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
  }
  done[dev] = true;
}

inline edk_status DevBuf::alloc_async(size_t n, cudaStream_t s) {
  release();
  if (n == 0) return EDK_OK;
  keep_pool_memory();
  cudaError_t e = cudaMallocAsync(&p, n, s);
  if (e != cudaSuccess) {
    cudaGetLastError();  // an allocation failure is not sticky: clear it for later checks
    p = nullptr;
    set_error(std::string("cudaMallocAsync(") + std::to_string(n) + " bytes) failed: " +
              cudaGetErrorString(e));
    return EDK_OOM;
  }
  bytes = n;
  pool_stream = s;
  pooled = true;
  return EDK_OK;
}

// ---------------------------------------------------------------------------
// lookup / canonicalisation kinds (compile-time dispatch)
// ---------------------------------------------------------------------------
enum LookupKind : int {
  BK_TENSOR = 0,     // row = state
  BK_PROJ_RANK = 1,  // row = colex rank among fixed-popcount states
  BK_PROJ_HASH = 2,  // row = hash(state)
  BK_TRANS0 = 3,     // translation, trivial phase (k = 0): min over rotations
  BK_TRANS = 4,      // translation, phase C[M] from the first-minimum shift M
  BK_TRANSPAR = 5,   // translation + reflection
  BK_ABELIAN = 6,    // generic odometer over commuting generators
  // BK_TRANS0 basis searched through its rank table (EDK_SEARCH_RANK); only
  // the bond-family fast path instantiates it, every other path keeps the hash
  BK_TRANS0_RANK = 7,
  // BK_TRANS basis searched through its rank table (entries carry the shift M)
  BK_TRANS_RANK = 8,
  // BK_TRANSPAR basis searched through its rank table (entries carry the sign)
  BK_TRANSPAR_RANK = 9
};

constexpr int kMaxGen = 8;
constexpr int kMaxLayers = 64;
constexpr int kNormClasses = 32;
constexpr uint32_t kHashEmpty32 = 0xFFFFFFFFu;

enum GenKind : int { GEN_PERM = 0, GEN_ROTL = 1, GEN_REV = 2, GEN_ID = 3 };

struct GenDev {
  int kind;      // GenKind
  int order;     // cyclic order
  int shift;     // rotation amount for GEN_ROTL
  int nlayers;   // delta-swap layers for GEN_PERM
  uint64_t inv_mask;
  int phase_off; // offset into the phase table
  int pad;
  uint64_t lmask[kMaxLayers];
  int lshift[kMaxLayers];
};

// Everything a kernel needs to know about a basis; passed by value.
struct BasisDev {
  int bk;          // LookupKind
  int L, A, len;   // sites, unit cell, number of translations
  int64_t D;
  uint64_t maskL;  // (1 << L) - 1
  const uint64_t* I;     // states (nullptr for TensorBasis)
  const double* R;       // norms (nullptr for onsite kinds)
  // hash table (BK_PROJ_HASH / translation kinds / abelian)
  const void* htab;
  uint64_t hmask;        // slots - 1
  int hbits;             // log2(slots)
  int packed;            // 1: value = row << 5 | class; 0: value = row, R gathered
  // sorted-array search (edk_basis_set_search): two-level binary search over
  // the ascending representatives instead of the hash table
  int search;              // 0: hash table, 1: sorted array
  const uint32_t* keys32;  // representatives as 32-bit words (L <= 32), else null
  const uint32_t* fence;   // keys32[32 j]: first level of the search
  int64_t nfence;
  const uint8_t* rcls8;    // norm class of each row (packed values), else null
  // rank table (edk_basis_set_search(EDK_SEARCH_RANK), search == 2): for every
  // state with the sector's popcount, indexed by its colex rank, the entry
  // row << rank_shift | M << 5 | norm class of its representative (M, the
  // first-minimum shift, only when rank_shift == 10; for translation + parity
  // sectors rank_shift == 6 and bit 5 is the sign of the coefficient), or ~0u
  // when the orbit is not in the basis; binom32[p * 33 + k] = C(p, k), p < 32
  int rank_shift;            // 5 (row < 2^27), 6 (row < 2^26, sign), 10 (row < 2^22, M)
  const uint32_t* rankmap;
  const uint32_t* binom32;
  const uint32_t* rowrank;   // colex rank of each representative I[i]
  int nclass;
  double Rcls[kNormClasses];
  // BK_PROJ_RANK
  int K;                 // popcount of every state
  // phases
  const double2* phase;  // translation: len entries; abelian: concatenated tables
  int P;                 // parity sign (TranslationParityBasis)
  int phase_real;        // 1 when every phase is real
  int runs_canon;        // 1: canonicalise from zero-run tops (unit cell 1, phase-free)
  // abelian generators
  int ngen;
  const GenDev* gens;
};

// Local terms compiled for the device.
// Family: 2-site terms (i, i+d mod L) sharing one 4x4 matrix, evaluated on
// whole bit planes: X = s, Y = rotl(s, d), local column c = 2*X_p + Y_p.
struct FamDev {
  int d;
  int nnz[4];         // off-diagonal entries per local column
  uint64_t valid;     // bit p set when the family has a term with site i at bit p
  double2 dval[4];    // diagonal values M[c][c]
  int xr[4][3];       // c ^ r for each off-diagonal entry (bit1: site i, bit0: site j)
  double2 val[4][3];  // M[r][c]
};
// Generic term on up to 8 sites (bit positions, most significant site first).
struct TermDev {
  int nsites;
  int bitpos[8];
  int col_off;        // offset into colptr (2^nsites + 1 entries)
  int diag_off;       // offset into dval (2^nsites entries)
};
// Flip-flop bond families for the fast path (all 2-site off-diagonal terms
// swap the two digits; every other term is diagonal).
constexpr int kMaxFF = 4;
struct FFParams {
  int nfam;
  int d[kMaxFF];
  uint32_t valid[kMaxFF];
  double2 dval[kMaxFF][4];
  double2 v1[kMaxFF];  // M[2][1]: local column "01" -> row "10"
  double2 v2[kMaxFF];  // M[1][2]: local column "10" -> row "01"
  int same[kMaxFF];    // 1 when v1 == v2 (one accumulator for both directions)
};

// Materialised operator (the device counterpart of sparse!(opt)): sliced
// ELLPACK with 32-row slices.  Rows are sorted by their number of nonzeros
// inside windows of 256 rows; slice s holds rows rowid[32 s .. 32 s + 31] and
// its entries k = 0..w_s-1 at off_s + 32 k + lane (lane = row in the slice):
// col = target row, code = index into vt (vt[0] = 0 pads short rows); when
// the code's bits and the row's bits fit together, both share one 32-bit word.
// y[r] = (1/R_r) sum conj(vt[code]) x[col] + conj(diag[r]) x[r].
struct SellDev {
  int64_t nslices;
  int packed;              // > 0: entry = row << packed | code, both in `col`
  int rbits;               // slot word = row | norm class << rbits; ~0u past the last row
  const unsigned* rowid;   // 32 per slice, in slot order
  const int64_t* off;      // entry offset of each slice
  const int* width;        // entries per lane of each slice
  const int* col;          // target rows
  const uint16_t* code;    // coefficient codes
  const double2* val;      // value mode (any operator): the entry's coefficient c, y += conj(c) x;
                           // col holds the row, no codes (null in code mode)
  const double* diag;      // real diagonal per slot (Hermitian operators with real terms)
  const double2* diagc;    // complex diagonal per slot, or null
  const double* rinv;      // 1 / R of each norm class (1 for bases without norms)
  const double2* vt64;     // coefficient table, FP64
  const float2* vt32;      // the same table rounded to FP32
};

constexpr int kPlanWindow = 256;  // rows per window of a row plan (and per thread block)
// Device view of a row plan: slot k of window w describes row
// rw[k] & kPlanRowMask of that window (rows sorted by their number of hits).
struct RowPlanDev {
  // one 16-byte slot per row, read with one load:
  //   x = row | norm class << 27 (~0u pads the last window)
  //   y = row state (L <= 32)
  //   z = colex rank of the row state (the row itself for complete sectors)
  //   w = rank of the state with bits 0 and L-1 exchanged (the wrap-around
  //       bond of a nearest-neighbour family), or ~0u
  const uint4* slot;
  const double* dg;       // diagonal of the row (operators with diagonal-only generic terms), or null
  const uint32_t* binom;  // binom[p * 33 + k] = C(p, k), p < 32
  int64_t nslots;         // windows * 256
};
constexpr uint32_t kPlanRowMask = (1u << 27) - 1u;

struct OpDev {
  SellDev sell;
  RowPlanDev plan;          // row plan of the rank-searched fast path (plan.slot null: none)
  int nfam;
  const FamDev* fam;
  int nterm;
  const TermDev* term;
  const int* colptr;        // per term: start of the off-diagonal list of each column
  const uint64_t* xmask;    // XOR mask turning the row state into the column state
  const double2* val;       // matrix element M[r][c]
  const double2* dval;      // diagonal M[c][c]
};

}  // namespace edk

// Opaque handles of the C ABI.
struct edk_basis {
  edk_basis_desc desc{};
  int kind = 0;
  int L = 0, A = 1, len = 1, K = -1, P = 1, Kmom = 0;  // Kmom = mod(-k, len)
  int64_t D = 0;
  edk::DevBuf I, R, htab, phase, gens;
  edk::DevBuf keys32, fence, rcls8;  // sorted-array search tables (built on demand)
  edk::DevBuf rankmap, binom32, rowrank;  // rank table of EDK_SEARCH_RANK (built on demand)
  edk::BasisDev dev{};
  std::vector<edk::GenDev> gens_host;
  std::vector<int> gen_order, gen_q;
  std::vector<std::vector<int>> gen_perm;
  std::vector<std::vector<uint8_t>> gen_inv;
  bool phase_complex = false;
  bool pairnorm = false;  // TranslationFlipBasis norms on the abelian path
  int device = 0;  // CUDA device the tables live on
  cudaStream_t stream = nullptr;
  std::mutex mu;
  ~edk_basis();
};

struct edk_operator {
  edk_basis* b = nullptr;
  edk::DevBuf fam, term, colptr, xmask, val, dval;
  edk::DevBuf hx, hy;  // staging buffers of edk_apply's host-pointer path (grow only)
  // materialised matrix (edk_operator_materialize)
  edk::DevBuf s_rowid, s_off, s_width, s_col, s_code, s_diag, s_vt64, s_vt32, s_rinv, s_err, s_val;
  int64_t sell_wincap = 0;  // entries of the largest 256-row window
  bool sell_tma_ok = false;  // the staged (bulk-copy) product applies (stages fit in shared memory)
  bool sell_tma = false;     // ... and is used (set by the autotuner)
  bool sell_ok = false;
  int64_t sell_entries = 0;
  edk::OpDev dev{};
  bool gather = true;
  bool is_complex = false;
  bool ff_ok = false;     // flip-flop bond-family fast path applies
  bool use_ff = true;     // callers may switch the fast path off (A/B checks)
  int tps = 1;            // threads per state of the fast path (1, 2 or 4; autotuned)
  // row plan of the fast path on rank-searched sectors (edk_plan.cu): built on
  // first use; plan_state 0 not built, 1 built, -1 not available
  edk::DevBuf p_slot, p_dg, p_binom, p_bad;
  int plan_state = 0;
  bool use_plan = true;   // tps == 1 on a rank-searched sector runs the plan kernel
  int use_block = -1;     // several right-hand sides through one SpMM: 1 yes, 0 no, -1 auto
                          // (yes unless materialised or on a row plan, whose one-column
                          // products already stream faster)
  std::vector<unsigned char> ff_params;
  int max_hits = 0;
  int nfam = 0, ngeneric = 0;
  // host copy of the merged terms (used by the invariance check)
  std::vector<std::vector<int>> sites;
  std::vector<std::vector<double>> dense_re, dense_im;  // local matrices, row-major
  cudaStream_t stream = nullptr;
  edk::DevBuf bx, by, bop;               // row-major blocks and operator record of the SpMM path
  std::vector<unsigned char> bop_host;   // the record as last uploaded
  cudaStream_t cstream = nullptr;        // copy stream of the pipelined host path
  std::vector<cudaEvent_t> cevents;      // one per row chunk of that path
  std::mutex mu;
  ~edk_operator();
};

namespace edk {
// implemented in edk_basis.cu
edk_status check_basis_dev(const BasisDev& b);
edk_status index_device(const BasisDev& dv, int64_t n, const uint64_t* s_d, int64_t* p_d,
                        double2* c_d, cudaStream_t st);
// rows [row0, row1) of y = H x (row0, row1 multiples of 256 or row1 = D)
// for one vector, on the row-gather fast or materialised paths; false when the
// operator runs on another path
bool rows_apply_ok(const edk_operator* op);
edk_status apply_rows(edk_operator* op, int dtype, const void* x, void* y, int64_t row0,
                      int64_t row1, int accumulate, cudaStream_t st);
// implemented in edk_plan.cu
bool plan_applies(const edk_operator* op);
edk_status plan_ensure(edk_operator* op);
edk_status apply_plan(edk_operator* op, int dtype, const void* x, void* y, int64_t nvec,
                      int64_t ldx, int64_t ldy, int accumulate, cudaStream_t st, int64_t row0,
                      int64_t row1);
// implemented in edk_sell.cu
edk_status apply_sell_rows(edk_operator* op, int dtype, const void* x, void* y, int64_t row0,
                           int64_t row1, int accumulate, cudaStream_t st);
edk_status apply_sell(edk_operator* op, int dtype, const void* x, void* y, int64_t nvec,
                      int64_t ldx, int64_t ldy, int accumulate, cudaStream_t st);
// implemented in edk_apply.cu
edk_status apply_device(edk_operator* op, int dtype, const void* x, void* y, int64_t nvec,
                        int64_t ldx, int64_t ldy, int accumulate, cudaStream_t st);
// implemented in edk_batch.cu
struct OpResult {
  std::vector<double> a, b, ev;  // recurrence coefficients and lowest Ritz values
  int steps = 0;
  int status = 0;  // 0 ran to the step limit, 1 converged, 2 breakdown, 3 zero norm,
                   // 4 non-finite start
};
// ritz_out (optional, device): every operator's lowest Ritz vector in the
// FP64 working dtype (F64 or C128), concatenated in operator order
edk_status batch_lanczos(const std::vector<edk_operator*>& ops, const edk_lanczos_opts& o,
                         const void* v0_dev, int v0_dt, cudaStream_t st,
                         std::vector<OpResult>& res, edk_lanczos_diag* diag,
                         void* ritz_out = nullptr);
// implemented in edk_util.cpp
int tridiag_eigvals(int m, const double* a, const double* b, double* w);
// The lowest `nev` distinct eigenvalues of block-tridiagonal Hermitian
// matrices (operator q: m[q] blocks of p x p, A[q][j] on the diagonal and
// B[q][j], j >= 1, below it, column-major interleaved complex on the host),
// on the device (edk_band.cu); NaN where fewer are found.
edk_status band_lowest_device(int p, int nev, const std::vector<int>& m,
                              const std::vector<std::vector<const double*>>& A,
                              const std::vector<std::vector<const double*>>& B,
                              cudaStream_t st, std::vector<std::vector<double>>& out);
int tridiag_eigen(int m, const double* a, const double* b, double* w, double* Q);
double elapsed_ms(cudaEvent_t a, cudaEvent_t b);
}  // namespace edk
