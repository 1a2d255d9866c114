// noalloc.cu — the canonical 2m reduction for callers that cannot allocate.
//
// hl_tree_sum_noalloc computes the same fixed-shape pairwise sum the update
// path uses for 2m (tiles of 1024 values padded with +0.0, each folded by
// stride halving, the tile sums folded again until one value is left), over a
// device array the caller owns, writing the result to a device address the
// caller owns.  It allocates nothing: the tile sums live in the file-scope
// array below, which every GPU that loads the library holds until exit.
//
// Who needs this: code that must not call cudaMalloc or the stream-ordered
// allocator — a caller running inside a region that forbids allocation (for
// example a host callback or a real-time loop with a fixed memory budget), or
// an embedding runtime that owns all device memory and hands the library only
// its input and output buffers.
//
// Limits and sharing: at most HL_NOALLOC_MAX_ELEMS values per call.  All calls
// on one GPU share the scratch array and it keeps the last call's contents;
// two calls whose work overlaps on the GPU (different streams, or different
// host threads without ordering) race on it and must be serialised by the
// caller.  Every call made outside stream capture resolves the array's device
// address with cudaGetSymbolAddress, with the device current, and keeps it per
// device; a call made while its stream is being captured uses the kept address
// instead.  So the first call on a device must come before any capture, and a
// capture after cudaDeviceReset must again follow an uncaptured call (the
// address is only valid for the life of the primary context).
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/hl.h"

namespace {

constexpr unsigned long long kTile = 1024;
constexpr unsigned long long kMaxTiles1 = HL_NOALLOC_MAX_ELEMS / kTile;   // 262144
constexpr unsigned long long kMaxTiles2 = (kMaxTiles1 + kTile - 1) / kTile;  // 256

// level-1 tile sums, then level-2 tile sums
static __device__ __align__(256) double g_tree_scratch[kMaxTiles1 + kMaxTiles2];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double* g_scratch_ptr[kMaxDevices] = {nullptr};

__global__ void k_tree_tile_noalloc(const double* x, unsigned long long n, double* out) {
  __shared__ double s[1024];
  unsigned long long base = (unsigned long long)blockIdx.x * 1024;
  for (unsigned i = threadIdx.x; i < 1024; i += blockDim.x) {
    unsigned long long idx = base + i;
    s[i] = idx < n ? x[idx] : 0.0;
  }
  __syncthreads();
  for (unsigned st = 512; st >= 1; st >>= 1) {
    for (unsigned i = threadIdx.x; i < st; i += blockDim.x) s[i] = __dadd_rn(s[i], s[i + st]);
    __syncthreads();
  }
  if (threadIdx.x == 0) out[blockIdx.x] = s[0];
}

__global__ void k_store_zero(double* out) { *out = 0.0; }

}  // namespace

// Error text for hl_last_error (defined with the rest of the C ABI).
void hl_set_error_message(const std::string& m);

extern "C" HL_API hl_status hl_tree_sum_noalloc(const double* d_x, uint64_t n, double* d_out,
                                                void* stream) {
  if (!d_out || (n && !d_x)) {
    hl_set_error_message("hl_tree_sum_noalloc: NULL device pointer");
    return HL_ERR_INVALID_INPUT;
  }
  if (n > HL_NOALLOC_MAX_ELEMS) {
    hl_set_error_message("hl_tree_sum_noalloc: " + std::to_string(n) +
                         " values exceed the fixed scratch limit of " +
                         std::to_string((unsigned long long)HL_NOALLOC_MAX_ELEMS));
    return HL_ERR_INVALID_INPUT;
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    hl_set_error_message(std::string("hl_tree_sum_noalloc: no usable current device: ") +
                         cudaGetErrorString(e));
    return HL_ERR_CUDA;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  e = cudaStreamIsCapturing(st, &cap);
  if (e != cudaSuccess) {
    hl_set_error_message(std::string("hl_tree_sum_noalloc: cudaStreamIsCapturing failed: ") +
                         cudaGetErrorString(e));
    return HL_ERR_CUDA;
  }
  double* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    if (cap == cudaStreamCaptureStatusNone) {
      // Host code only knows a stand-in for the array; its device address is
      // resolved with the device current.  Resolving it on every uncaptured
      // call keeps the kept address right after a context reset.
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_tree_scratch);
      if (e != cudaSuccess || !p) {
        hl_set_error_message(std::string("hl_tree_sum_noalloc: cudaGetSymbolAddress failed: ") +
                             cudaGetErrorString(e));
        return HL_ERR_CUDA;
      }
      g_scratch_ptr[dev] = static_cast<double*>(p);
    } else if (!g_scratch_ptr[dev]) {
      hl_set_error_message(
          "hl_tree_sum_noalloc: first call on this device made during stream capture; make an "
          "uncaptured call first");
      return HL_ERR_INVALID_INPUT;
    }
    scratch = g_scratch_ptr[dev];
  }
  if (n == 0) {
    k_store_zero<<<1, 1, 0, st>>>(d_out);
  } else {
    unsigned long long t1 = (n + kTile - 1) / kTile;
    if (t1 == 1) {
      k_tree_tile_noalloc<<<1, 256, 0, st>>>(d_x, n, d_out);
    } else {
      double* lvl1 = scratch;
      double* lvl2 = scratch + kMaxTiles1;
      k_tree_tile_noalloc<<<(unsigned)t1, 256, 0, st>>>(d_x, n, lvl1);
      unsigned long long t2 = (t1 + kTile - 1) / kTile;
      if (t2 == 1) {
        k_tree_tile_noalloc<<<1, 256, 0, st>>>(lvl1, t1, d_out);
      } else {
        k_tree_tile_noalloc<<<(unsigned)t2, 256, 0, st>>>(lvl1, t1, lvl2);
        k_tree_tile_noalloc<<<1, 256, 0, st>>>(lvl2, t2, d_out);  // t2 <= 256
      }
    }
  }
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    hl_set_error_message(std::string("hl_tree_sum_noalloc: launch failed: ") +
                         cudaGetErrorString(e));
    return HL_ERR_CUDA;
  }
  return HL_OK;
}
