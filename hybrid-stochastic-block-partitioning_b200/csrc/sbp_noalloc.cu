// Allocation-free MDL entry point (sbp_mdl_device_noalloc in include/sbp_b200.h).
//
// For callers that cannot allocate GPU memory: code that runs under a device-memory budget
// fixed at start-up, or that must not call cudaMalloc/cudaFree because those synchronize the
// whole device (a pipeline with work in flight on other streams, a host callback, a caller that
// owns every allocation itself).  The caller passes the block counts and degrees already on the
// device and a device pointer for the result; the only scratch memory is the file-scope array
// below, which every GPU that loads this library holds until the process exits.
//
// Limits and sharing:
//   * at most kNoAllocMaxBlocks blocks (one FP64 partial sum per block row: 256 KB);
//   * every call writes the array before reading it, so stale contents from an earlier call
//     are never used, but the array is shared by all calls: calls that overlap on the GPU
//     (different streams, or different host threads) race on it and must be serialised;
//   * the first call on a device looks up the array's device address on that device (see
//     scratch_for_current_device); make that first call before any stream capture.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "../../include/sbp_b200.h"
#include "sbp_error.h"

namespace sbpb_noalloc {

constexpr int kNoAllocMaxBlocks = 32768;
constexpr int kMaxDevices = 64;
constexpr int kFinalThreads = 256;   // CTA size of k_noalloc_final (its reduction array is sized from it)
static_assert(kFinalThreads % 32 == 0 && kFinalThreads <= 1024, "k_noalloc_final needs whole warps");

// Per-row partial sums of M log M.  In host code this name is only a handle for
// cudaGetSymbolAddress, never a device address.
static __device__ __align__(256) double g_row_scratch[kNoAllocMaxBlocks];

__device__ __forceinline__ double na_xlogx(double x) { return x > 0.0 ? x * log(x) : 0.0; }

// One warp per block row: rows[row] = sum_col g(M[row, col]).
__global__ void k_noalloc_rows(const int* __restrict__ M, int B, long long ld, double* rows) {
  const int lane = threadIdx.x & 31;
  const int wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int row = wid; row < B; row += nw) {
    double acc = 0.0;
    const int* p = M + (size_t)row * (size_t)ld;
    for (int col = lane; col < B; col += 32) acc += na_xlogx((double)p[col]);
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) rows[row] = acc;
  }
}

// Fixed-order sum of the row partials and the degree terms, then the MDL formula
// (entropy::mdl, src/entropy.cpp:584-589).  One CTA of kFinalThreads threads.
__global__ void __launch_bounds__(kFinalThreads) k_noalloc_final(const double* rows, int B, const int* __restrict__ d_out,
                                                                 const int* __restrict__ d_in, int V, long long E,
                                                                 double* result) {
  __shared__ double red[kFinalThreads / 32];
  double acc = 0.0;
  for (int i = threadIdx.x; i < B; i += blockDim.x)
    acc += rows[i] - na_xlogx((double)d_out[i]) - na_xlogx((double)d_in[i]);
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double L = 0.0;
    for (int w = 0; w < kFinalThreads / 32; ++w) L += red[w];
    const double x = pow((double)B, 2) / (double)E;
    const double h = ((1 + x) * log(1 + x)) - (x * log(x));
    *result = ((double)E * h) + ((double)V * log((double)B)) - L;
  }
}

static std::mutex g_mutex;
static double* g_scratch_ptr[kMaxDevices];

// Device address of g_row_scratch on the current device, looked up once per device.
static cudaError_t scratch_for_current_device(double** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!g_scratch_ptr[dev]) {
    double* p = nullptr;
    e = cudaGetSymbolAddress((void**)&p, g_row_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_ptr[dev] = p;
  }
  *out = g_scratch_ptr[dev];
  return cudaSuccess;
}

// Records a failure for sbp_last_error() (a fixed per-thread buffer: nothing is allocated).
static void fail(const char* what, const char* detail = "") {
  char msg[256];
  snprintf(msg, sizeof msg, "sbp_mdl_device_noalloc: %s%s", what, detail);
  sbpb::set_last_error(msg);
}

}  // namespace sbpb_noalloc

extern "C" SbpStatus sbp_mdl_device_noalloc(const int32_t* d_matrix, int32_t num_blocks, int64_t ld,
                                            const int32_t* d_degrees_out, const int32_t* d_degrees_in,
                                            int32_t num_vertices, int64_t num_edges, double* d_result,
                                            void* stream) {
  using namespace sbpb_noalloc;
  if (!d_matrix || !d_degrees_out || !d_degrees_in || !d_result || num_blocks < 1 || ld < num_blocks ||
      num_vertices < 1 || num_edges < 1) {
    fail("bad argument (NULL pointer, ld < num_blocks or a size below 1)");
    return SBP_ERR_INVALID_ARGUMENT;
  }
  if (num_blocks > kNoAllocMaxBlocks) {
    char what[128];
    snprintf(what, sizeof what, "%d blocks exceed the %d-block limit of its static scratch array", num_blocks,
             kNoAllocMaxBlocks);
    fail(what);
    return SBP_ERR_UNSUPPORTED;
  }
  double* rows = nullptr;
  cudaError_t e = scratch_for_current_device(&rows);
  if (e != cudaSuccess) {
    fail("scratch lookup failed: ", cudaGetErrorString(e));
    return SBP_ERR_CUDA;
  }
  cudaStream_t s = (cudaStream_t)stream;
  const int warps_per_cta = 8;
  int grid = (num_blocks + warps_per_cta - 1) / warps_per_cta;
  if (grid > 4096) grid = 4096;
  k_noalloc_rows<<<grid, 32 * warps_per_cta, 0, s>>>(d_matrix, num_blocks, ld, rows);
  k_noalloc_final<<<1, kFinalThreads, 0, s>>>(rows, num_blocks, d_degrees_out, d_degrees_in, num_vertices, num_edges, d_result);
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    fail("launch failed: ", cudaGetErrorString(e));
    return SBP_ERR_CUDA;
  }
  return SBP_OK;
}
