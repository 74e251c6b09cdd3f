// Exchange energy without any device allocation.
//
// ipie_b200_exchange writes its per-(Cholesky tile, walker) partial sums into
// a workspace the caller allocates.  Some callers cannot allocate device
// memory at the point where they need the exchange energy: a host code whose
// device memory is entirely owned by its own pool allocator (a framework's
// caching allocator, or a preallocated arena sized at start-up), or a hot loop
// that must not pay the implicit device synchronisation of cudaMalloc and
// cudaFree.  For them this file keeps the partials in a fixed file-scope
// device array and reduces them into the caller's output.
//
// Limits and sharing:
//   * the array holds kNoAllocScratchElems complex partials (16 MiB); a call
//     needs rows * W of them, rows = ipie_b200_exchange_rows(W, X, M, N), and
//     larger problems are rejected with cudaErrorInvalidValue before any work;
//   * every GPU that loads this library holds the array until the process exits;
//   * every call shares the one array and leaves its partials there; nothing
//     has to start at zero (each call writes every partial it later reads);
//   * calls that overlap on the GPU (two streams at once) race on the array.
//
// Set-up: every call, with the caller's device current, looks the array's
// device address up with cudaGetSymbolAddress (a host-side table lookup), so
// the address stays right after a device reset or a new primary context.  The
// first call on a device also loads the library's device code there (the set-up
// of the array); make that first call before any stream capture on the device.
#include "../../include/ipie_b200.h"
#include "common.cuh"
#include "kernels.h"

namespace ipie_b200 {

static constexpr size_t kNoAllocScratchBytes = size_t(16) << 20;
static constexpr size_t kNoAllocScratchElems = kNoAllocScratchBytes / sizeof(double2);
static __device__ __align__(256) double2 g_exchange_scratch[kNoAllocScratchElems];

// Device address of g_exchange_scratch on the current device and context.  The
// host-side name of the array is only a stand-in: kernels get this address.
static cudaError_t scratch_address(double2** out) {
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_exchange_scratch);
  if (e != cudaSuccess) return e;
  *out = static_cast<double2*>(p);
  return cudaSuccess;
}

// exx[w] = sum over partial rows t of part[t * W + w], fixed order.
__global__ void reduce_partials_kernel(const double2* __restrict__ part, int rows, int W, double2* __restrict__ exx) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= W) return;
  double2 s = make_double2(0.0, 0.0);
  for (int t = 0; t < rows; ++t) s = cadd(s, part[(size_t)t * W + w]);
  exx[w] = s;
}

}  // namespace ipie_b200

using namespace ipie_b200;

extern "C" int ipie_b200_exchange_noalloc(const double* rchol, const void* ghalf, int W, int X, int M, int N,
                                          void* exx, void* stream) {
  if (W <= 0 || X <= 0 || M <= 0 || N <= 0 || rchol == nullptr || ghalf == nullptr || exx == nullptr)
    return (int)cudaErrorInvalidValue;
  int rows = 0;
  cudaError_t e = launch_exchange(nullptr, nullptr, W, X, M, N, nullptr, &rows, nullptr);
  if (e != cudaSuccess) return (int)e;
  if ((size_t)rows * (size_t)W > kNoAllocScratchElems) return (int)cudaErrorInvalidValue;
  double2* scratch = nullptr;
  e = scratch_address(&scratch);
  if (e != cudaSuccess) return (int)e;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  e = launch_exchange(rchol, reinterpret_cast<const double2*>(ghalf), W, X, M, N, scratch, &rows, st);
  if (e != cudaSuccess) return (int)e;
  reduce_partials_kernel<<<(W + 127) / 128, 128, 0, st>>>(scratch, rows, W, reinterpret_cast<double2*>(exx));
  note_launch();
  return (int)cudaGetLastError();
}
