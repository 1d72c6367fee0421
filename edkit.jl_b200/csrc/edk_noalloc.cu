// edk_noalloc.cu — index() for host-side states without any device allocation.
//
// edk_basis_index with host pointers stages the states and the results in
// device buffers it allocates for the call.  Some callers cannot allocate
// device memory at the point where they need a lookup: host runtimes that
// call in from contexts where they forbid allocation (for example a garbage
// collector's finaliser or a callback that must not block), latency-sensitive
// loops that must not pay for the allocator's implicit synchronisation, and
// processes in which another component has already reserved all device
// memory for its own pool.  edk_basis_index_noalloc serves them from a fixed
// scratch area that is part of the library image.
//
// The scratch is a file-scope __device__ array of kNoAllocBytes (2 MiB): room
// for kNoAllocMaxStates states with their positions and coefficients.  Every
// GPU that loads libedk keeps those 2 MiB reserved until the process exits.
// All calls share it: a host mutex serialises the calls and each call waits
// for its own copies before returning, so calls never overlap on the GPU;
// a caller that bypassed this function and launched work on the same array
// concurrently would race.  The results are fully overwritten on every call,
// so no part of the array has to be cleared between calls.
//
// In host code the name `g_noalloc_scratch` denotes a host-side stand-in, not
// a device address.  The device address is obtained once per device with
// cudaGetSymbolAddress, with that device current, on the first call made for a
// basis living on that device; that first call should therefore happen
// before any stream capture begins.
#include <mutex>

#include "edk_internal.cuh"

namespace {

constexpr int64_t kNoAllocMaxStates = 65536;
constexpr size_t kNoAllocBytes = (size_t)kNoAllocMaxStates * (8 + 8 + 16);
constexpr int kMaxDevices = 64;

__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

std::mutex g_noalloc_mu;
void* g_noalloc_ptr[kMaxDevices] = {};

// device address of the scratch on `dev` (which must be current)
edk_status scratch_on(int dev, unsigned char** out) {
  if (dev < 0 || dev >= kMaxDevices) {
    edk::set_error("edk_basis_index_noalloc: device ordinal out of range");
    return EDK_INVALID_ARG;
  }
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr) {
      edk::set_error(std::string("edk_basis_index_noalloc: cudaGetSymbolAddress failed: ") +
                     cudaGetErrorString(e));
      return EDK_CUDA_ERROR;
    }
    g_noalloc_ptr[dev] = p;
  }
  *out = static_cast<unsigned char*>(g_noalloc_ptr[dev]);
  return EDK_OK;
}

}  // namespace

// Same results as edk_basis_index(b, n, states, pos, coeff, EDK_HOST), with n
// limited to 65536 states per call and no device allocation.
extern "C" edk_status edk_basis_index_noalloc(const edk_basis* bc, int64_t n,
                                              const uint64_t* states, int64_t* pos,
                                              double* coeff) {
  EDK_CHECK_ARG(bc && states && pos && coeff, "edk_basis_index_noalloc: NULL argument");
  EDK_CHECK_ARG(n >= 0, "edk_basis_index_noalloc: n < 0");
  if (n > kNoAllocMaxStates) {
    edk::set_error("edk_basis_index_noalloc: n = " + std::to_string(n) +
                   " exceeds the fixed scratch of 65536 states per call; split the batch or "
                   "use edk_basis_index");
    return EDK_INVALID_ARG;
  }
  if (n == 0) return EDK_OK;
  edk_basis* b = const_cast<edk_basis*>(bc);
  std::lock_guard<std::mutex> glk(g_noalloc_mu);
  std::lock_guard<std::mutex> lk(b->mu);
  int prev = 0;
  EDK_TRY_CUDA(cudaGetDevice(&prev));
  if (prev != b->device) EDK_TRY_CUDA(cudaSetDevice(b->device));
  unsigned char* base = nullptr;
  edk_status st = scratch_on(b->device, &base);
  if (st == EDK_OK) {
    uint64_t* s_d = reinterpret_cast<uint64_t*>(base);
    int64_t* p_d = reinterpret_cast<int64_t*>(base + (size_t)kNoAllocMaxStates * 8);
    double2* c_d = reinterpret_cast<double2*>(base + (size_t)kNoAllocMaxStates * 16);
    cudaStream_t s = b->stream;
    cudaError_t e = cudaMemcpyAsync(s_d, states, n * 8, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) {
      st = edk::index_device(b->dev, n, s_d, p_d, c_d, s);
      if (st == EDK_OK) {
        e = cudaMemcpyAsync(pos, p_d, n * 8, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(coeff, c_d, n * 16, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
      }
    }
    if (st == EDK_OK && e != cudaSuccess) {
      edk::set_error(std::string("edk_basis_index_noalloc: ") + cudaGetErrorString(e));
      st = EDK_CUDA_ERROR;
    }
  }
  if (prev != b->device) cudaSetDevice(prev);
  return st;
}
