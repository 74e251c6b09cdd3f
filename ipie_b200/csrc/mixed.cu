// Mixed-precision (TF32 tensor-core) stages of the walker step and their
// host-side plumbing: TMA tensor maps, hi/lo operand splits, launchers.
#include <cudaTypedefs.h>

#include <mutex>

#include "../../include/ipie_b200.h"
#include "../../include/ipie_b200_testing.h"
#include "kernels.h"
#include "umma_gemm.cuh"

namespace ipie_b200 {
namespace umma {

// cuTensorMapEncodeTiled through the runtime's driver entry point (no libcuda link).
static PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

// 3-D batched K-major fp32 operand: `batch` matrices of `rows` x `k` (row stride k, matrix stride
// rows * k elements), tiles of box_rows x 32 of one matrix; rows past `rows` read as 0 (no traffic).
cudaError_t make_map_batched(CUtensorMap* m, const float* base, long long batch, long long rows, long long k,
                             int box_rows) {
  auto fn = encode_fn();
  if (fn == nullptr) return cudaErrorNotSupported;
  if ((reinterpret_cast<uintptr_t>(base) & 15) || (k % 4) || rows <= 0 || k <= 0 || batch <= 0)
    return cudaErrorInvalidValue;
  cuuint64_t dims[3] = {(cuuint64_t)k, (cuuint64_t)rows, (cuuint64_t)batch};
  cuuint64_t strides[2] = {(cuuint64_t)k * 4, (cuuint64_t)rows * k * 4};
  cuuint32_t box[3] = {32, (cuuint32_t)box_rows, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(base), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

// 2-D K-major fp32 operand: `rows` rows of `k` elements, row stride `ld` elements,
// tiles of box_rows x 32 loaded 128B-swizzled; out-of-range elements read as 0.
cudaError_t make_map(CUtensorMap* m, const float* base, long long rows, long long k, long long ld, int box_rows) {
  auto fn = encode_fn();
  if (fn == nullptr) return cudaErrorNotSupported;
  if ((reinterpret_cast<uintptr_t>(base) & 15) || (ld % 4) || rows <= 0 || k <= 0) return cudaErrorInvalidValue;
  cuuint64_t dims[2] = {(cuuint64_t)k, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)ld * 4};
  cuuint32_t box[2] = {32, (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(base), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

// 2-D K-major FP16 operand: `rows` rows of `k` halves, row stride `ld` halves (ld % 8 == 0),
// tiles of box_rows x 64 loaded 128B-swizzled (k32: box_rows x 32, 64B-swizzled, the tiles of
// KIND_F16_K32); out-of-range elements read as 0.
cudaError_t make_map_f16(CUtensorMap* m, const void* base, long long rows, long long k, long long ld, int box_rows,
                         bool k32) {
  auto fn = encode_fn();
  if (fn == nullptr) return cudaErrorNotSupported;
  if ((reinterpret_cast<uintptr_t>(base) & 15) || (ld % 8) || rows <= 0 || k <= 0) return cudaErrorInvalidValue;
  cuuint64_t dims[2] = {(cuuint64_t)k, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
  cuuint32_t box[2] = {k32 ? 32u : 64u, (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2, const_cast<void*>(base), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, k32 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_128B,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}
cudaError_t make_map_f16(CUtensorMap* m, const void* base, long long rows, long long k, long long ld, int box_rows) {
  return make_map_f16(m, base, rows, k, ld, box_rows, false);
}

// Output map of W matrices of rows x ld halves (row stride ld, matrix stride rows x ld) for
// tensor stores of {bx, by, bz} boxes (no swizzle: the staging box is plain row-major).
cudaError_t make_map_f16_store(CUtensorMap* m, void* base, long long W, long long rows, long long ld, int bx, int by,
                               int bz) {
  auto fn = encode_fn();
  if (fn == nullptr) return cudaErrorNotSupported;
  if ((reinterpret_cast<uintptr_t>(base) & 15) || (ld % 8) || rows <= 0 || W <= 0 || (bx * 2) % 16) return cudaErrorInvalidValue;
  cuuint64_t dims[3] = {(cuuint64_t)ld, (cuuint64_t)rows, (cuuint64_t)W};
  cuuint64_t strides[2] = {(cuuint64_t)ld * 2, (cuuint64_t)rows * ld * 2};
  cuuint32_t box[3] = {(cuuint32_t)bx, (cuuint32_t)by, (cuuint32_t)bz};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 3, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                  CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

// 2-D K-major FP16 operand and its remainder as the two planes of one 3-D map: the remainder
// starts `plane` halves after the head (plane % 8 == 0); tiles of box_rows x 64 (k32: x 32) of
// both planes land back to back in shared memory (the head tile, then the remainder tile).
cudaError_t make_map_f16_planes(CUtensorMap* m, const void* base, long long rows, long long k, long long ld,
                                long long plane, int box_rows, bool k32) {
  auto fn = encode_fn();
  if (fn == nullptr) return cudaErrorNotSupported;
  if ((reinterpret_cast<uintptr_t>(base) & 15) || (ld % 8) || (plane % 8) || rows <= 0 || k <= 0 || plane <= 0)
    return cudaErrorInvalidValue;
  cuuint64_t dims[3] = {(cuuint64_t)k, (cuuint64_t)rows, 2};
  cuuint64_t strides[2] = {(cuuint64_t)ld * 2, (cuuint64_t)plane * 2};
  cuuint32_t box[3] = {k32 ? 32u : 64u, (cuuint32_t)box_rows, 2};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 3, const_cast<void*>(base), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, k32 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_128B,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

// The head/remainder pair (hi, lo) of an operand of rows x ld halves as one two-plane map when lo
// sits at a fixed offset >= rows x ld after hi (both halves of one allocation); else two maps.
// Returns the planes flag of GemmMaps.
static cudaError_t map_f16_pair(CUtensorMap* mhi, CUtensorMap* mlo, const void* hi, const void* lo, long long rows,
                                long long k, long long ld, int box_rows, bool k32, int* planes) {
  const uintptr_t h = reinterpret_cast<uintptr_t>(hi), l = reinterpret_cast<uintptr_t>(lo);
  const long long d = l > h ? (long long)((l - h) / 2) : 0;
  if (l > h && (l - h) % 16 == 0 && d >= rows * ld) {
    *planes = 1;
    return make_map_f16_planes(mhi, hi, rows, k, ld, d, box_rows, k32);
  }
  *planes = 0;
  cudaError_t e = make_map_f16(mhi, hi, rows, k, ld, box_rows, k32);
  if (e == cudaSuccess) e = make_map_f16(mlo, lo, rows, k, ld, box_rows, k32);
  return e;
}

// 3-D batched K-major FP16 operand: `batch` matrices of `rows` x `k` halves (row stride ld
// halves, ld % 8 == 0; matrix stride rows * ld), tiles of box_rows x 64 of one matrix; rows past
// `rows` and columns past `k` read as 0 (no traffic).
cudaError_t make_map_f16_batched(CUtensorMap* m, const void* base, long long batch, long long rows, long long k,
                                 long long ld, int box_rows) {
  auto fn = encode_fn();
  if (fn == nullptr) return cudaErrorNotSupported;
  if ((reinterpret_cast<uintptr_t>(base) & 15) || (ld % 8) || rows <= 0 || k <= 0 || batch <= 0 || ld < k)
    return cudaErrorInvalidValue;
  cuuint64_t dims[3] = {(cuuint64_t)k, (cuuint64_t)rows, (cuuint64_t)batch};
  cuuint64_t strides[2] = {(cuuint64_t)ld * 2, (cuuint64_t)rows * ld * 2};
  cuuint32_t box[3] = {64, (cuuint32_t)box_rows, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 3, const_cast<void*>(base), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

// The four VHS planes of every walker as one 4-D map (planes `plane` halves apart in one
// allocation): columns (k), rows, walkers, planes; box 16 columns x box_rows x 1 x 4, 32-byte
// swizzled -- the last 16 columns of all four planes of a walker in one copy.
cudaError_t make_map_f16_tail4(CUtensorMap* m, const void* base, long long batch, long long rows, long long k,
                               long long ld, long long plane, int box_rows) {
  auto fn = encode_fn();
  if (fn == nullptr) return cudaErrorNotSupported;
  if ((reinterpret_cast<uintptr_t>(base) & 15) || (ld % 8) || (plane % 8) || rows <= 0 || k <= 0 || batch <= 0 ||
      ld < k || plane < batch * rows * ld)
    return cudaErrorInvalidValue;
  cuuint64_t dims[4] = {(cuuint64_t)k, (cuuint64_t)rows, (cuuint64_t)batch, 4};
  cuuint64_t strides[3] = {(cuuint64_t)ld * 2, (cuuint64_t)rows * ld * 2, (cuuint64_t)plane * 2};
  cuuint32_t box[4] = {16, (cuuint32_t)box_rows, 1, 4};
  cuuint32_t estr[4] = {1, 1, 1, 1};
  CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 4, const_cast<void*>(base), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_32B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

// hi = FP16(x * scale), lo = FP16(x * scale - hi): the split of the FP16 3-pass product.
__global__ void split_f16_kernel(const double* __restrict__ x, __half* __restrict__ hi, __half* __restrict__ lo,
                                 long long n, double scale) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    __half h, l;
    split_f16(x[i], scale, h, l);
    hi[i] = h;
    if (lo) lo[i] = l;
  }
}

cudaError_t launch_split_f16(const double* x, __half* hi, __half* lo, long long n, double scale, cudaStream_t st) {
  long long blocks = (n + 255) / 256;
  if (blocks > 148 * 32) blocks = 148 * 32;
  if (blocks < 1) blocks = 1;
  split_f16_kernel<<<(unsigned)blocks, 256, 0, st>>>(x, hi, lo, n, scale);
  note_launch();
  return cudaGetLastError();
}

// hi = TF32(x), lo = TF32(x - hi) (both rounded to nearest): the split of the 3-pass product.
__global__ void split_tf32_kernel(const double* __restrict__ x, float* __restrict__ hi, float* __restrict__ lo,
                                  long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    float h, l;
    split_tf32(x[i], h, l);
    hi[i] = h;
    if (lo) lo[i] = l;
  }
}

cudaError_t launch_split_tf32(const double* x, float* hi, float* lo, long long n, cudaStream_t st) {
  long long blocks = (n + 255) / 256;
  if (blocks > 148 * 32) blocks = 148 * 32;
  if (blocks < 1) blocks = 1;
  split_tf32_kernel<<<(unsigned)blocks, 256, 0, st>>>(x, hi, lo, n);
  note_launch();
  return cudaGetLastError();
}

// ---------------------------------------------------------------- test epilogue
// c[z][row][a][col] (row < M, col < N): the raw accumulators, for validation.
template <int BN, int NA>
struct EpiStoreF32 {
  float* c;
  int M, N;
  __device__ __forceinline__ void operator()(int z, int row, int n0, const float* v, uint8_t*) const {
    if (row >= M) return;
    float* base = c + ((size_t)z * M + row) * (size_t)NA * N;
#pragma unroll
    for (int a = 0; a < NA; ++a)
#pragma unroll
      for (int j = 0; j < BN; ++j)
        if (n0 + j < N) base[(size_t)a * N + n0 + j] = v[a * BN + j];
  }
};

// tiles: (column tiles, row tiles, batches) of the output; m_fast orders the tile list with the
// row-tile index fastest (see TileOrder).  persistent: one CTA per SM walks the tile list;
// otherwise one CTA per tile.
template <int BN, int NA, int NSPLIT, int STAGES, class Epi, int KIND = KIND_TF32, int CG = 1>
cudaError_t launch_umma(const GemmMaps& maps, int K, int a_rows_per_batch, int b_rows_per_batch, dim3 tiles, Epi epi,
                        unsigned* status, cudaStream_t st, bool m_fast = false, bool persistent = true,
                        int m_group = 0) {
  using S = GemmShape<BN, NA, NSPLIT, STAGES, EpiSmem<Epi>::value, KIND, CG>;
  auto kern = umma_gemm_kernel<BN, NA, NSPLIT, STAGES, Epi, KIND, CG>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, S::SMEM_BYTES);
  if (e != cudaSuccess) return e;
  int dev = 0, sms = 0;
  if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
  if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
  const TileOrder order{(int)tiles.y, (int)tiles.x, (int)tiles.z, m_fast ? 1 : 0,
                        m_group > 0 ? m_group : (int)tiles.y};
  const long long ntiles = (long long)tiles.x * tiles.y * tiles.z;
  if (ntiles <= 0 || ntiles > 0x7fffffffLL) return cudaErrorInvalidValue;
  if constexpr (CG == 2) {
    // clusters of two CTAs, one per SM pair: as many pairs as can be resident at once (persistent)
    cudaLaunchConfig_t cfg;
    memset(&cfg, 0, sizeof(cfg));
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 2;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.blockDim = dim3(GemmRoles<NA, BN>::kThreads);
    cfg.dynamicSmemBytes = S::SMEM_BYTES;
    cfg.stream = st;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cfg.gridDim = dim3(2 * (sms / 2));
    int pairs = 0;
    if ((e = cudaOccupancyMaxActiveClusters(&pairs, kern, &cfg)) != cudaSuccess) return e;
    if (pairs < 1) return cudaErrorInvalidConfiguration;
    const long long want = persistent && ntiles > pairs ? pairs : ntiles;
    cfg.gridDim = dim3((unsigned)(2 * want));
    e = cudaLaunchKernelEx(&cfg, kern, maps, K, a_rows_per_batch, b_rows_per_batch, order, epi, status);
    note_launch();
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
  }
  const int grid = (int)(persistent && ntiles > sms ? sms : ntiles);
  kern<<<grid, GemmRoles<NA, BN>::kThreads, S::SMEM_BYTES, st>>>(maps, K, a_rows_per_batch, b_rows_per_batch, order,
                                                                 epi, status);
  note_launch();
  return cudaGetLastError();
}

template <int NA, int NSPLIT, int STAGES>
static cudaError_t gemm_test(const float* const* a_hi, const float* const* a_lo, const float* b_hi, const float* b_lo,
                             float* c, int M, int N, int K, unsigned* status, cudaStream_t st) {
  constexpr int BN = NA == 1 ? 128 : 64;
  GemmMaps maps;
  memset(&maps, 0, sizeof(maps));
  cudaError_t e;
  for (int a = 0; a < NA; ++a) {
    if ((e = make_map(&maps.a_hi[a], a_hi[a], M, K, K, kBM)) != cudaSuccess) return e;
    if (NSPLIT == 3 && (e = make_map(&maps.a_lo[a], a_lo[a], M, K, K, kBM)) != cudaSuccess) return e;
  }
  if ((e = make_map(&maps.b_hi, b_hi, N, K, K, BN)) != cudaSuccess) return e;
  if (NSPLIT == 3 && (e = make_map(&maps.b_lo, b_lo, N, K, K, BN)) != cudaSuccess) return e;
  dim3 grid((N + BN - 1) / BN, (M + kBM - 1) / kBM, 1);
  return launch_umma<BN, NA, NSPLIT, STAGES>(maps, K, 0, 0, grid, EpiStoreF32<BN, NA>{c, M, N}, status, st);
}

static cudaError_t gemm_test_f16(const void* a_hi, const void* a_lo, const void* b_hi, const void* b_lo, float* c,
                                 int M, int N, int K, int nsplit, unsigned* status, cudaStream_t st) {
  constexpr int BN = 128;
  GemmMaps maps;
  memset(&maps, 0, sizeof(maps));
  cudaError_t e;
  if ((e = make_map_f16(&maps.a_hi[0], a_hi, M, K, K, kBM)) != cudaSuccess) return e;
  if (nsplit == 3 && (e = make_map_f16(&maps.a_lo[0], a_lo, M, K, K, kBM)) != cudaSuccess) return e;
  if ((e = make_map_f16(&maps.b_hi, b_hi, N, K, K, BN)) != cudaSuccess) return e;
  if (nsplit == 3 && (e = make_map_f16(&maps.b_lo, b_lo, N, K, K, BN)) != cudaSuccess) return e;
  dim3 grid((N + BN - 1) / BN, (M + kBM - 1) / kBM, 1);
  if (nsplit == 3)
    return launch_umma<BN, 1, 3, 3, EpiStoreF32<BN, 1>, KIND_F16>(maps, K, 0, 0, grid, EpiStoreF32<BN, 1>{c, M, N},
                                                                  status, st);
  return launch_umma<BN, 1, 1, 4, EpiStoreF32<BN, 1>, KIND_F16>(maps, K, 0, 0, grid, EpiStoreF32<BN, 1>{c, M, N},
                                                                status, st);
}

}  // namespace umma
}  // namespace ipie_b200

using namespace ipie_b200;

extern "C" int ipie_b200_split_f16(const double* x, void* hi, void* lo, long long n, double scale, void* stream) {
  return (int)umma::launch_split_f16(x, reinterpret_cast<__half*>(hi), reinterpret_cast<__half*>(lo), n, scale,
                                     reinterpret_cast<cudaStream_t>(stream));
}

extern "C" int ipie_b200_umma_gemm_f16_test(const void* a_hi, const void* a_lo, const void* b_hi, const void* b_lo,
                                            float* c, int M, int N, int K, int nsplit, unsigned int* status,
                                            void* stream) {
  if (K % 8 || M <= 0 || N <= 0 || K <= 0 || (nsplit != 1 && nsplit != 3)) return (int)cudaErrorInvalidValue;
  return (int)umma::gemm_test_f16(a_hi, a_lo, b_hi, b_lo, c, M, N, K, nsplit, status,
                                  reinterpret_cast<cudaStream_t>(stream));
}

extern "C" int ipie_b200_split_tf32(const double* x, float* hi, float* lo, long long n, void* stream) {
  return (int)umma::launch_split_tf32(x, hi, lo, n, reinterpret_cast<cudaStream_t>(stream));
}

extern "C" int ipie_b200_umma_gemm_test(const float* a0_hi, const float* a0_lo, const float* a1_hi,
                                        const float* a1_lo, const float* b_hi, const float* b_lo, float* c, int M,
                                        int N, int K, int na, int nsplit, unsigned int* status, void* stream) {
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  if (K % 4 || M <= 0 || N <= 0 || K <= 0) return (int)cudaErrorInvalidValue;
  const float* ah[2] = {a0_hi, a1_hi};
  const float* al[2] = {a0_lo, a1_lo};
  if (na == 1 && nsplit == 1) return (int)umma::gemm_test<1, 1, 4>(ah, al, b_hi, b_lo, c, M, N, K, status, st);
  if (na == 1 && nsplit == 3) return (int)umma::gemm_test<1, 3, 3>(ah, al, b_hi, b_lo, c, M, N, K, status, st);
  if (na == 2 && nsplit == 3) return (int)umma::gemm_test<2, 3, 2>(ah, al, b_hi, b_lo, c, M, N, K, status, st);
  return (int)cudaErrorInvalidValue;
}

// ============================================================================
// Mixed-precision walker-step stages
// ============================================================================
namespace ipie_b200 {
namespace umma {

template <typename T>
__device__ __forceinline__ void store_split(float* hi, float* lo, size_t i, T x) {
  float h, l;
  split_tf32(x, h, l);
  hi[i] = h;
  lo[i] = l;
}

// Force bias with the operands swapped: rows (w, c) of the Green's function, columns x of the
// Cholesky operand; a thread writes component c of vbias[w][x] for its row's columns.
template <int BN>
struct EpiVbiasT {
  double2* vbias;
  int X, W;
  double scale;               // overall factor, divided by the operands' power-of-two scales below
  const double* walker_scale;  // per-walker scale of the Green's-function operand (NULL: 1)
  int accumulate;
  static constexpr int kCols = GemmRoles<1, BN>::kGroupCols;
  __device__ __forceinline__ void operator()(int, int row, int x0, const float* v, uint8_t*) const {
    const int w = row >> 1, c = row & 1;
    if (w >= W) return;
    const double f = walker_scale != nullptr ? scale / walker_scale[w] : scale;
    double* out = reinterpret_cast<double*>(vbias + (size_t)w * X) + c;
#pragma unroll
    for (int q = 0; q < kCols; ++q) {
      const int x = x0 + q;
      if (x < X) {
        double r = f * (double)v[q];
        if (accumulate) r += out[2 * (size_t)x];
        out[2 * (size_t)x] = r;
      }
    }
  }
};

// VHS: rows p of the packed Cholesky (P, X) hi/lo, B rows (w, c) of the shifted
// fields (W, 2, X) hi/lo.  V = i sqrt(dt) (S_re + i S_im) is written to both
// triangles of four planar (W, M, M) fp32 arrays: re/im x hi/lo (the left
// operands of the exp(VHS) products).
template <int BN>
struct EpiVHSSplit {
  float *re_hi, *re_lo, *im_hi, *im_lo;
  const int* ii;
  const int* jj;
  int P, M, W;
  float sdt;
  __device__ __forceinline__ void operator()(int, int p, int n0, const float* v, uint8_t*) const {
    if (p >= P) return;
    const int i = ii[p], j = jj[p];
#pragma unroll
    for (int q = 0; q < BN / 2; ++q) {
      const int w = (n0 >> 1) + q;
      if (w < W) {
        const float vre = -sdt * v[2 * q + 1], vim = sdt * v[2 * q];
        const size_t a = ((size_t)w * M + i) * M + j, b = ((size_t)w * M + j) * M + i;
        store_split(re_hi, re_lo, a, vre);
        store_split(im_hi, im_lo, a, vim);
        if (i != j) {
          store_split(re_hi, re_lo, b, vre);
          store_split(im_hi, im_lo, b, vim);
        }
      }
    }
  }
};

// VHS for the FP16 orbital chain: V x v_scale written to both triangles of four planar
// (W, M, ld) binary16 arrays (re/im x head/remainder; ld = M rounded up to 8, the pad columns
// are not written).  A warp whose 32 pairs form a full 8 x 4 block strictly above the diagonal,
// starting on a row and a column that are multiples of 4 (the packing puts such blocks first),
// trades values by shuffles so that each lane writes one 8-byte
// run per orientation and walker -- lane (r, c): plane c of row i0 + r, columns j0..j0+3, and
// plane r % 4 of row j0 + c, columns i0 + 4 (r / 4) .. +3 -- instead of eight 2-byte stores;
// other warps store pair by pair.
template <int BN>
struct EpiVHSF16 {
  __half *re_hi, *re_lo, *im_hi, *im_lo;
  const int* ii;
  const int* jj;
  int P, M, ld, W;
  float f;  // sqrt(dt) v_scale / (operand scales)
  __device__ __forceinline__ static void put(__half* hi, __half* lo, size_t i, float x) {
    const __half h = __float2half_rn(x);
    hi[i] = h;
    lo[i] = __float2half_rn(x - __half2float(h));
  }
  __device__ __forceinline__ __half* plane(int k) const {
    return k == 0 ? re_hi : k == 1 ? re_lo : k == 2 ? im_hi : im_lo;
  }
  // 16-bit plane k (0 re_hi, 1 re_lo, 2 im_hi, 3 im_lo) out of the packed pairs a = (re_hi, re_lo), b = (im_hi, im_lo)
  __device__ __forceinline__ static uint32_t pick(int k, uint32_t a, uint32_t b) {
    const uint32_t x = k < 2 ? a : b;
    return (k & 1) ? (x >> 16) : (x & 0xffffu);
  }
  __device__ __forceinline__ void operator()(int, int p, int n0, const float* v, uint8_t*) const {
    const unsigned kFull = 0xffffffffu;
    const int lane = threadIdx.x & 31, r = lane >> 2, c = lane & 3;
    const bool live = p < P;
    const int i = live ? ii[p] : 0, j = live ? jj[p] : 0;
    const int i0 = __shfl_sync(kFull, i, 0), j0 = __shfl_sync(kFull, j, 0);
    // the 8-byte runs need i0 and j0 on multiples of 4 (ld is a multiple of 8): blocks elsewhere
    // (a diagonal tile's full rows can line up into one) take the pair-by-pair path
    const bool block =
        __all_sync(kFull, live && i == i0 + r && j == j0 + c && i0 + 7 < j0 && (i0 & 3) == 0 && (j0 & 3) == 0) != 0;
    if (!block) {
      if (!live) return;
#pragma unroll
      for (int q = 0; q < BN / 2; ++q) {
        const int w = (n0 >> 1) + q;
        if (w < W) {
          const float vre = -f * v[2 * q + 1], vim = f * v[2 * q];
          const size_t a = ((size_t)w * M + i) * ld + j, b = ((size_t)w * M + j) * ld + i;
          put(re_hi, re_lo, a, vre);
          put(im_hi, im_lo, a, vim);
          if (i != j) {
            put(re_hi, re_lo, b, vre);
            put(im_hi, im_lo, b, vim);
          }
        }
      }
      return;
    }
    __half* dpl = plane(c);
    __half* tpl = plane(r & 3);
    const size_t doff = (size_t)(i0 + r) * ld + j0;                  // row i0 + r, columns j0 ..
    const size_t toff = (size_t)(j0 + c) * ld + i0 + 4 * (r >> 2);  // row j0 + c, columns i0 + 4 (r / 4) ..
    const size_t wstride = (size_t)M * ld;
    const int dsrc = 4 * r, tsrc = 16 * (r >> 2) + c;
#pragma unroll
    for (int q = 0; q < BN / 2; ++q) {
      const int w = (n0 >> 1) + q;
      if (w >= W) break;  // the same for the whole warp
      const float vre = -f * v[2 * q + 1], vim = f * v[2 * q];
      const __half h0 = __float2half_rn(vre), h2 = __float2half_rn(vim);
      const __half h1 = __float2half_rn(vre - __half2float(h0)), h3 = __float2half_rn(vim - __half2float(h2));
      const uint32_t a = (uint32_t)__half_as_ushort(h0) | ((uint32_t)__half_as_ushort(h1) << 16);
      const uint32_t b = (uint32_t)__half_as_ushort(h2) | ((uint32_t)__half_as_ushort(h3) << 16);
      uint32_t d[4], e[4];
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        d[t] = pick(c, __shfl_sync(kFull, a, dsrc + t), __shfl_sync(kFull, b, dsrc + t));
        e[t] = pick(r & 3, __shfl_sync(kFull, a, tsrc + 4 * t), __shfl_sync(kFull, b, tsrc + 4 * t));
      }
      *reinterpret_cast<uint2*>(dpl + w * wstride + doff) = make_uint2(d[0] | (d[1] << 16), d[2] | (d[3] << 16));
      *reinterpret_cast<uint2*>(tpl + w * wstride + toff) = make_uint2(e[0] | (e[1] << 16), e[2] | (e[3] << 16));
    }
  }
};

// VHS for the FP16 orbital chain, block-tiled: the product runs transposed -- rows (w, c) of
// the fields (c = re/im), columns the Cholesky rows of one 16 x 16 block of orbital pairs
// (i, j) = (16 I + a, 16 J + b), I <= J, row-major in the block (a diagonal block carries all
// 256 pairs, both triangles) -- so that a thread holds one walker's re or im part of a whole
// block half (rows a = 8g .. 8g + 7 for column group g).  It writes them as 16-byte runs of
// 8 halves: its 8 rows i, columns 16 J .. 16 J + 15 (two runs), and for an off-diagonal block
// the transposed rows j = 16 J + b, columns 16 I + 8g .. + 7; every run starts on a multiple of
// 8 halves of a row of ld (a multiple of 8) halves, so each store is 16-byte aligned and whole
// 32-byte sectors are written by one or two neighbouring runs.  V = i sqrt(dt) S: the re part of
// S (c = 0) gives the imaginary planes, the im part (c = 1) the real planes.  Rows i >= M are
// skipped; columns in [M, ld) receive the zero products of the zero Cholesky rows.
// binary16 head and remainder of the pair (y0, y1), packed two per word (y0 in the low half)
__device__ __forceinline__ uint32_t split2_f16(float y0, float y1, uint32_t& lo) {
  const __half2 h = __floats2half2_rn(y0, y1);
  const float2 hf = __half22float2(h);
  const __half2 l = __floats2half2_rn(y0 - hf.x, y1 - hf.y);
  lo = *reinterpret_cast<const uint32_t*>(&l);
  return *reinterpret_cast<const uint32_t*>(&h);
}

// The epilogue goes through shared memory and TMA tensor stores: one 32 KB staging box of 64
// walkers x 16 rows x 16 halves (the {16, 16, 64} box of the plane maps maps->out: re_hi, re_lo,
// im_hi, im_lo), filled and stored eight times per tile -- real then imaginary plane, the
// transposed block (J, I) then the block (I, J), head then remainder -- by the threads of the
// rows (c) that feed that plane.  A thread's scattered 16-byte global stores (one 32-byte sector
// split between two of them, 16 walkers per warp instruction) took ~30k cycles per tile and
// stalled the next tile's products; the staged tensor stores leave the copy to the TMA engine.
// Rows i >= M and columns j >= ld of a box are clipped by the store.
//
// Bank spread: a walker's part of the box is 512 bytes, so the 16 walkers of a warp instruction
// would all write the same four banks if each wrote the same 16-byte chunk of its part.  Lane k
// (k = (lane / 2) mod 8) writes its chunks in an order rotated by k instead: its block chunks
// (8 rows x two 16-byte halves) rotated by k within each half of eight, which spreads the 16
// lanes over all 32 banks (two wavefronts per instruction), and the transposed rows b rotated by
// k mod 4 within each group of four (four wavefronts: a transposed row has one 16-byte half per
// column group).  The values are split into head and remainder once per tile.
struct EpiVHSBlock {
  int M, W, nb;  // nb: 16-orbital blocks per side
  float f;       // sqrt(dt) v_scale / (operand scales)
  static constexpr int kSmemBytes = 64 * 16 * 32;
  static constexpr bool kUsesMaps = true;
  static constexpr int kThreads = 256;  // the epilogue threads of the 128 x 256 tile (barrier 3)
  __device__ __forceinline__ static void sync() { asm volatile("bar.sync 3, %0;\n" ::"r"(kThreads) : "memory"); }
  // chunk q of 16 (row q / 2 of the block half, 16-byte half q % 2) moved to position q's
  // rotation: after the call, chunk i holds the original chunk (i & 8) | ((i + k) & 7)
  __device__ __forceinline__ static void rotate(uint32_t (&x)[64], int k) {
#pragma unroll
    for (int st = 1; st < 8; st <<= 1) {
      const bool r = (k & st) != 0;
      uint32_t t[64];
#pragma unroll
      for (int q = 0; q < 16; ++q)
#pragma unroll
        for (int u = 0; u < 4; ++u) t[4 * q + u] = r ? x[4 * ((q & 8) | ((q + st) & 7)) + u] : x[4 * q + u];
#pragma unroll
      for (int e = 0; e < 64; ++e) x[e] = t[e];
    }
  }
  // one round's 16 chunks of the thread's part of the box (x: head or remainder pairs)
  __device__ __forceinline__ static void put(const uint32_t (&x)[64], bool tr, int k, int g, uint8_t* mine) {
    if (tr) {
      // rows b (orbital 16 J + b), columns 8g .. 8g + 7 (orbitals 16 I + 8g ..): halves of the
      // thread's rows a = 0 .. 7 at column b, b = 4 j + ((i + k) & 3) at instruction i
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const int bb = (i + k) & 3, b = (i & ~3) | bb;
        const bool mh = bb >= 2;
        const uint32_t sel = (bb & 1) ? 0x7632u : 0x5410u;
        const int m0 = 2 * (i >> 2);
        uint32_t wd[4];
#pragma unroll
        for (int t = 0; t < 4; ++t) {
          const uint32_t x0 = mh ? x[8 * (2 * t) + m0 + 1] : x[8 * (2 * t) + m0];
          const uint32_t x1 = mh ? x[8 * (2 * t + 1) + m0 + 1] : x[8 * (2 * t + 1) + m0];
          wd[t] = __byte_perm(x0, x1, sel);
        }
        *reinterpret_cast<uint4*>(mine + b * 32 + 16 * g) = make_uint4(wd[0], wd[1], wd[2], wd[3]);
      }
    } else {
      // rows 8g + a of the box, columns 16 J .. 16 J + 15: chunk i (rotated) is the original chunk q
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const int q = (i & 8) | ((i + k) & 7);
        *reinterpret_cast<uint4*>(mine + 256 * g + 16 * q) = make_uint4(x[4 * i], x[4 * i + 1], x[4 * i + 2], x[4 * i + 3]);
      }
    }
  }
  __device__ __forceinline__ void operator()(int, int row, int col0, const float* v, uint8_t* smem,
                                             const GemmMaps* maps) const {
    const int w = row >> 1, c = row & 1;
    const int w0 = (row & ~127) >> 1, wl = w - w0;
    const bool live = w < W;
    int blk = col0 >> 8, I = 0;  // tile = block index, row-major over I <= J
    while (blk >= nb - I) {
      blk -= nb - I;
      ++I;
    }
    const int J = I + blk;
    const int g = (col0 >> 7) & 1;
    const float s = c ? -f : f;
    const int k = (threadIdx.x >> 1) & 7;
    uint8_t* mine = smem + wl * 512;
    // head / remainder pairs: word 8 a + m holds columns 2m, 2m + 1 of the thread's row a
    uint32_t ph[64], pl[64];
#pragma unroll
    for (int e = 0; e < 64; ++e) ph[e] = split2_f16(v[2 * e] * s, v[2 * e + 1] * s, pl[e]);
#pragma unroll
    for (int half = 0; half < 2; ++half) {
      const int pc = 1 - half;  // the rows feeding this plane: c = 1 real, c = 0 imaginary
      const bool act = live && c == pc;
#pragma unroll
      for (int rd = 0; rd < 4; ++rd) {
        const int tr = rd < 2, lo = rd & 1;
        if (tr && I == J) continue;  // the same for every thread of the tile
        if (rd == 2 && act) {
          rotate(ph, k);
          rotate(pl, k);
        }
        if (threadIdx.x == 0) bulk_wait_read_all();  // the previous box has left shared memory
        sync();
        if (act) {
          if (lo)
            put(pl, tr, k, g, mine);
          else
            put(ph, tr, k, g, mine);
          asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        }
        sync();
        if (threadIdx.x == 0) {
          tma_store_3d(&maps->out[(pc ? 0 : 2) + lo], tr ? 16 * I : 16 * J, tr ? 16 * J : 16 * I, w0, smem);
          bulk_commit();
        }
      }
    }
  }
};

// Rows of the block-tiled Cholesky operand gathered from the packed one: row r takes packed
// row rowmap[r] (or zeros for -1), scaled and split into binary16 head and remainder; (R, ldx).
__global__ void vhs_block_pack_kernel(const double* __restrict__ cp, const int* __restrict__ rowmap, long long R,
                                      int X, int ldx, double scale, __half* __restrict__ hi, __half* __restrict__ lo) {
  const long long n = R * ldx;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    const long long r = e / ldx;
    const int x = (int)(e - r * ldx);
    const int p = rowmap[r];
    const double val = (p >= 0 && x < X) ? cp[(long long)p * X + x] : 0.0;
    __half h, l;
    split_f16(val, scale, h, l);
    hi[e] = h;
    lo[e] = l;
  }
}

// One Taylor term / one-body factor on the orbitals of walker z (one spin):
// accumulators (columns c*N + n, c = re/im of the right operand):
//   one-body (NA = 1):  U = E . T
//   Taylor   (NA = 2):  U = (V_re T_re - V_im T_im) + i (V_re T_im + V_im T_re)
// then per mode
//   PRE   : phi_acc = U;                 next B = U
//   TERM  : T = U / n; phi_acc += T;     next B = T           (next B = phi_acc when last)
//   POST  : phi_out = U
enum OrbMode { ORB_PRE = 0, ORB_TERM = 1, ORB_TERM_LAST = 2, ORB_POST = 3 };

template <int NA, int BN>
struct EpiOrbital {
  const double2* phi_base;  // one-body modes: phi_out = phi_base + (E - I) phi (FP64 add)
  double2* phi_acc;         // (W, M, N) complex double
  float* nb_hi;             // next right operand (W, 2N, M) fp32 hi/lo
  float* nb_lo;
  int M, N;
  float inv_n;
  int mode;
  __device__ __forceinline__ void operator()(int w, int m, int, const float* v, uint8_t*) const {
    if (m >= M) return;
    for (int n = 0; n < N; ++n) {
      float ur, ui;
      if (NA == 2) {
        ur = v[n] - v[BN + N + n];
        ui = v[N + n] + v[BN + n];
      } else {
        ur = v[n];
        ui = v[N + n];
      }
      const size_t pi = ((size_t)w * M + m) * N + n;
      const size_t bre = ((size_t)w * 2 * N + n) * M + m, bim = ((size_t)w * 2 * N + N + n) * M + m;
      if (mode == ORB_PRE || mode == ORB_POST) {
        // the one-body factor is applied as phi + (E - I) phi: the identity part stays exact in
        // FP64 and the TF32 product only carries the small correction
        const double2 b = phi_base[pi];
        const double2 out = make_double2(b.x + (double)ur, b.y + (double)ui);
        phi_acc[pi] = out;
        if (mode == ORB_PRE) {
          store_split(nb_hi, nb_lo, bre, out.x);
          store_split(nb_hi, nb_lo, bim, out.y);
        }
      } else {
        const float tr = ur * inv_n, ti = ui * inv_n;
        double2 acc = phi_acc[pi];
        acc.x += tr;
        acc.y += ti;
        phi_acc[pi] = acc;
        if (mode == ORB_TERM) {
          store_split(nb_hi, nb_lo, bre, tr);
          store_split(nb_hi, nb_lo, bim, ti);
        } else {
          store_split(nb_hi, nb_lo, bre, acc.x);
          store_split(nb_hi, nb_lo, bim, acc.y);
        }
      }
    }
  }
};

// phi (W, M, N) complex double -> planar right operand (W, 2N, M) fp32 hi/lo.
__global__ void phi_to_planar_kernel(const double2* __restrict__ phi, int W, int M, int N, float* __restrict__ hi,
                                     float* __restrict__ lo) {
  const long long total = (long long)W * M * N;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
    // e enumerates the output order (w, c-less n, m) so stores are coalesced
    const int m = (int)(e % M);
    const long long t = e / M;
    const int n = (int)(t % N);
    const int w = (int)(t / N);
    const double2 z = phi[((size_t)w * M + m) * N + n];
    store_split(hi, lo, ((size_t)w * 2 * N + n) * M + m, z.x);
    store_split(hi, lo, ((size_t)w * 2 * N + N + n) * M + m, z.y);
  }
}

// Ghalf (W, N*M) complex double -> planar (W, 2, N*M) fp32 (TF32-rounded).
__global__ void ghalf_to_planar_kernel(const double2* __restrict__ g, long long W, long long K, float* __restrict__ out) {
  const long long total = W * K;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
    const long long w = e / K, k = e % K;
    const double2 z = g[e];
    out[(w * 2) * K + k] = (float)z.x;
    out[(w * 2 + 1) * K + k] = (float)z.y;
  }
}

static unsigned grid_for(long long n) {
  long long b = (n + 255) / 256;
  if (b > 148 * 32) b = 148 * 32;
  return (unsigned)(b < 1 ? 1 : b);
}

// Exchange in 3-pass TF32: rows (x, i) of the padded half-rotated Cholesky
// (X*NP, M), columns (w, c, j) of the padded planar Green's function
// (W*2*NP, M); the epilogue forms sum_{i,j<N} T_ij T_ji per (x, w) block, one
// partial per (x tile, w).  The NP rows of one x lie in one warp (32 % NP == 0),
// so each warp parks its own 32 rows in shared memory and walks its blocks
// without a CTA barrier: lane (g, j), g = lane / NP, j = lane % NP, runs over the
// rows i of x block g.  A lane's products and sum in FP32 (the operands carry the
// split products' errors already), the sums across lanes and blocks in FP64.
template <int NP, int BN>
struct EpiExchange {
  static constexpr int LD = BN + 1;  // odd stride: row and column walks are both conflict-free
  static constexpr int XB = kBM / NP, WB = BN / (2 * NP);
  static constexpr int kPartOffset = ((kBM * LD * 4 + 15) / 16) * 16;
  static constexpr int kSmemBytes = kPartOffset + XB * WB * 16;
  static_assert(32 % NP == 0, "an x block must not straddle warps");
  double2* part;
  int X, W, N;
  double inv_rscale2;          // 1 / (Cholesky operand scale)^2
  const double* walker_scale;  // per-walker scale of the Green's-function operand
  __device__ __forceinline__ void operator()(int, int row, int n0, const float* v, uint8_t* smem) const {
    const int mt = row / kBM;  // row tile
    float* sC = reinterpret_cast<float*>(smem);
    double2* wpart = reinterpret_cast<double2*>(smem + kPartOffset);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
#pragma unroll
    for (int c = 0; c < BN; ++c) sC[tid * LD + c] = v[c];
    __syncwarp();
    const int g = lane / NP, j = lane % NP;
    const int xl = warp * (32 / NP) + g;
    const bool xok = mt * XB + xl < X && j < N;
    for (int wl = 0; wl < WB; ++wl) {
      const float* blk = sC + (xl * NP) * LD + wl * 2 * NP;
      double sr = 0.0, si = 0.0;
      if (xok && (n0 / (2 * NP)) + wl < W) {
        // a lane's N products summed in FP32 (~2^-24 each, below the split products' own
        // errors in the operands), then FP64 across lanes and blocks
        float fr = 0.0f, fi = 0.0f;
#pragma unroll 4
        for (int i = 0; i < N; ++i) {
          const float ar = blk[i * LD + j], ai = blk[i * LD + NP + j];
          const float br = blk[j * LD + i], bi = blk[j * LD + NP + i];
          fr = fmaf(ar, br, fmaf(-ai, bi, fr));
          fi = fmaf(ar, bi, fmaf(ai, br, fi));
        }
        sr = fr;
        si = fi;
      }
#pragma unroll
      for (int o = NP / 2; o > 0; o >>= 1) {
        sr += __shfl_xor_sync(0xffffffffu, sr, o);
        si += __shfl_xor_sync(0xffffffffu, si, o);
      }
      if (j == 0) {
        // undo the operand scales: T = acc / (s_r s_w), the sum is quadratic in T
        const int w = (n0 / (2 * NP)) + wl;
        const double iw = w < W ? 1.0 / walker_scale[w] : 0.0;
        const double f = inv_rscale2 * iw * iw;
        wpart[xl * WB + wl] = make_double2(f * sr, f * si);
      }
    }
    epi_sync();
    if (tid < WB) {
      const int w = n0 / (2 * NP) + tid;
      if (w < W) {
        double2 s = make_double2(0.0, 0.0);
        for (int x = 0; x < XB; ++x) s = cadd(s, wpart[x * WB + tid]);
        part[(size_t)mt * W + w] = s;
      }
    }
    epi_sync();  // wpart is rewritten by the next tile
  }
};

// rchol (X, N*M) double -> rows (x, i) padded to NP, columns padded to Mp = f16_ld(M):
// (X*NP, Mp) binary16 hi/lo of rchol x scale, zeros for i >= N and m >= M.
__global__ void rchol_pad_f16_kernel(const double* __restrict__ r, int X, int N, int M, int NP, int Mp, double scale,
                                     __half* __restrict__ hi, __half* __restrict__ lo) {
  const long long total = (long long)X * NP * Mp;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
    const int m = (int)(e % Mp);
    const long long t = e / Mp;
    const int i = (int)(t % NP);
    const long long x = t / NP;
    const double val = (i < N && m < M) ? r[(x * N + i) * M + m] : 0.0;
    __half h, l;
    split_f16(val, scale, h, l);
    hi[e] = h;
    lo[e] = l;
  }
}

// Ghalf (W, N, M) complex double -> planar padded (W, 2, NP, Mp) binary16 hi/lo of Ghalf x s_w,
// zeros for j >= N and m >= M; s_w = 2^(14 - e) with max_w |Re, Im| = f 2^e, f in [0.5, 1), so
// the walker's largest entry lands in [2^13, 2^14).  With gref (N, M) given, the operand is
// Ghalf - gref (the deviation from the trial).  One CTA per walker: a max pass, then the split
// (the second read of the walker's block comes from cache).  scale[w] = s_w.
__global__ void __launch_bounds__(256) ghalf_pad_f16_kernel(const double2* __restrict__ g,
                                                            const double2* __restrict__ gref, int N, int M, int NP,
                                                            int Mp, __half* __restrict__ hi, __half* __restrict__ lo,
                                                            double* __restrict__ scale) {
  __shared__ double red[8];
  const int w = blockIdx.x, tid = threadIdx.x;
  const double2* gw = g + (size_t)w * N * M;
  double mx = 0.0;
  for (int e = tid; e < N * M; e += 256) {
    double2 z = gw[e];
    if (gref != nullptr) {
      const double2 r = gref[e];
      z.x -= r.x;
      z.y -= r.y;
    }
    mx = fmax(mx, fmax(fabs(z.x), fabs(z.y)));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if ((tid & 31) == 0) red[tid >> 5] = mx;
  __syncthreads();
  mx = red[0];
#pragma unroll
  for (int k = 1; k < 8; ++k) mx = fmax(mx, red[k]);
  int ex = 0;
  if (mx > 0.0 && isfinite(mx)) frexp(mx, &ex);
  const double sw = ldexp(1.0, 14 - ex);
  if (tid == 0) scale[w] = sw;
  const long long base = (long long)w * 2 * NP * Mp;
  // each entry read once, both planes written (real part at row j, imaginary at row NP + j), two
  // neighbouring columns per thread (Mp is even, so a pair never straddles a row)
  for (int e = 2 * tid; e < NP * Mp; e += 2 * 256) {
    const int m = e % Mp, j = e / Mp;
    double2 z[2];
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      z[q] = make_double2(0.0, 0.0);
      if (j < N && m + q < M) {
        z[q] = gw[(size_t)j * M + m + q];
        if (gref != nullptr) {
          const double2 r = gref[(size_t)j * M + m + q];
          z[q].x -= r.x;
          z[q].y -= r.y;
        }
      }
    }
    __half h0, l0, h1, l1;
    split_f16(z[0].x, sw, h0, l0);
    split_f16(z[1].x, sw, h1, l1);
    *reinterpret_cast<__half2*>(hi + base + e) = __halves2half2(h0, h1);
    *reinterpret_cast<__half2*>(lo + base + e) = __halves2half2(l0, l1);
    split_f16(z[0].y, sw, h0, l0);
    split_f16(z[1].y, sw, h1, l1);
    *reinterpret_cast<__half2*>(hi + base + NP * Mp + e) = __halves2half2(h0, h1);
    *reinterpret_cast<__half2*>(lo + base + NP * Mp + e) = __halves2half2(l0, l1);
  }
}

int exchange_np(int N) { return N <= 8 ? 8 : N <= 16 ? 16 : N <= 32 ? 32 : -1; }

cudaError_t mixed_rchol_pad(const double* rchol, int X, int N, int M, double scale, __half* hi, __half* lo,
                            cudaStream_t st) {
  const int NP = exchange_np(N);
  if (NP < 0) return cudaErrorInvalidValue;
  const int Mp = f16_ld(M);
  rchol_pad_f16_kernel<<<grid_for((long long)X * NP * Mp), 256, 0, st>>>(rchol, X, N, M, NP, Mp, scale, hi, lo);
  note_launch();
  return cudaGetLastError();
}

// The Green's-function operand of the FP16 products, carved from the caller's fp32 work array
// (2 W 2 32 M floats, more than the binary16 hi/lo of (W, 2, NP, Mp) plus W scales need).
struct GPad {
  __half* hi;
  __half* lo;
  double* scale;
};
static GPad carve_gpad(float* gwork, int W, int NP, int M) {
  const size_t n = (size_t)W * 2 * NP * f16_ld(M);
  GPad g;
  g.hi = reinterpret_cast<__half*>(gwork);
  g.lo = g.hi + n;
  g.scale = reinterpret_cast<double*>(reinterpret_cast<uintptr_t>(g.lo + n + 7) & ~uintptr_t(7));
  return g;
}

// Padded planar Green's function (FP16 head/remainder, per-walker scale) of one spin block.
static cudaError_t pad_ghalf(const double2* ghalf, int W, int M, int N, int NP, const GPad& gp, cudaStream_t st,
                             const double2* gref = nullptr) {
  ghalf_pad_f16_kernel<<<W, 256, 0, st>>>(ghalf, gref, N, M, NP, f16_ld(M), gp.hi, gp.lo, gp.scale);
  note_launch();
  return cudaGetLastError();
}

// Reference row of the exchange around the trial: with T linear in Ghalf,
//   raw(G) = sum_x tr(T_G T_G) = raw(G_T) + K.(G - G_T) + raw(G - G_T),
// K = d raw/dG at the trial.  out[w] = raw(G_T) + sum K (G_w - G_T) in FP64; the
// quadratic remainder raw(G - G_T) is the tensor-core part.  One CTA per walker.
__global__ void __launch_bounds__(256) exchange_ref_row_kernel(const double2* __restrict__ g,
                                                               const double2* __restrict__ gref,
                                                               const double2* __restrict__ kmat, int NM,
                                                               const double2* __restrict__ raw_ref,
                                                               double2* __restrict__ out) {
  __shared__ double2 red[32];
  const int w = blockIdx.x;
  double2 acc = make_double2(0.0, 0.0);
  for (int e = threadIdx.x; e < NM; e += blockDim.x) {
    const double2 a = g[(size_t)w * NM + e], r = gref[e];
    acc = cadd(acc, cmul(kmat[e], make_double2(a.x - r.x, a.y - r.y)));
  }
  acc = block_sum2(acc, red);
  if (threadIdx.x == 0) out[w] = cadd(acc, raw_ref[0]);
}

// The trial's Coulomb vector (one walker): xv[x] (+)= scale sum_k rchol[x][k] g[k], one warp per x
// (the FP64 force-bias GEMM with a single walker column left most SMs idle: 0.76 ms at c2).
__global__ void __launch_bounds__(256) coulomb_row_kernel(const double* __restrict__ rchol,
                                                          const double2* __restrict__ g, int X, int K,
                                                          double2* __restrict__ xv, int accumulate, double scale) {
  const int x = (int)((blockIdx.x * 256u + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (x >= X) return;
  const double* r = rchol + (size_t)x * K;
  double sx = 0.0, sy = 0.0;
  for (int k = lane; k < K; k += 32) {
    const double a = r[k];
    const double2 b = g[k];
    sx += a * b.x;
    sy += a * b.y;
  }
  sx = warp_sum(sx);
  sy = warp_sum(sy);
  if (lane == 0) {
    double2 v = make_double2(scale * sx, scale * sy);
    if (accumulate) v = cadd(v, xv[x]);
    xv[x] = v;
  }
}

static cudaError_t coulomb_row(const double* rchol, const double2* g, int X, int K, double2* xv, int accumulate,
                               double scale, cudaStream_t st) {
  coulomb_row_kernel<<<(unsigned)((X + 7) / 8), 256, 0, st>>>(rchol, g, X, K, xv, accumulate, scale);
  note_launch();
  return cudaGetLastError();
}

static cudaError_t exchange_ref_row(const double2* g, const double2* gref, const double2* kmat, int W, int NM,
                                    const double2* raw_ref, double2* out, cudaStream_t st) {
  exchange_ref_row_kernel<<<W, 256, 0, st>>>(g, gref, kmat, NM, raw_ref, out);
  note_launch();
  return cudaGetLastError();
}

// X[w][x] (scale, accumulate as the force bias) = sum_k rchol[x][k] Ghalf[w][k] as a 3-pass FP16
// product of the padded operands: rows (x) of (X, NP*Mp) x rscale, rows (w, c) of (2W, NP*Mp)
// with per-walker scales (the pads are zero in both, so K runs over them).
static cudaError_t coulomb3(const void* r_hi, const void* r_lo, double rscale, const GPad& gp, int W, int X, int M,
                            int NP, double2* xv, int accumulate, double scale, unsigned* status, cudaStream_t st) {
  // CTA pairs on 256 x 192 tiles, the Green's function's rows (w, c) as the 256-row side: each SM
  // stages 128 of them and 96 Cholesky rows per K step.  At c2 (4096 x 1600) that is 16 x 9 = 144
  // tiles, two full waves of 74 pairs (256 x 256 tiles the other way round: 112, 1.5 waves)
  constexpr int BN = 192, CG = 2;
  const long long K = (long long)NP * f16_ld(M);
  GemmMaps maps;
  memset(&maps, 0, sizeof(maps));
  cudaError_t e;
  if ((e = map_f16_pair(&maps.a_hi[0], &maps.a_lo[0], gp.hi, gp.lo, 2LL * W, K, K, kBM, false, &maps.a_planes)) !=
      cudaSuccess)
    return e;
  if ((e = map_f16_pair(&maps.b_hi, &maps.b_lo, r_hi, r_lo, X, K, K, BN / CG, false, &maps.b_planes)) !=
      cudaSuccess)
    return e;
  dim3 grid((X + BN - 1) / BN, (2 * W + CG * kBM - 1) / (CG * kBM), 1);
  // row tiles fastest: a Cholesky tile stays in L2 while the Green's function streams past it
  const EpiVbiasT<BN> epi{xv, X, W, scale / rscale, gp.scale, accumulate};
  return launch_umma<BN, 1, 3, 4, EpiVbiasT<BN>, KIND_F16, CG>(maps, (int)K, 0, 0, grid, epi, status, st, true);
}

// Exchange partials of one spin block as a 3-pass FP16 product: (X*NP, M) x (W*2*NP, M)^T, rows
// of both operands padded to Mp halves (TMA reads the pads as zeros).
template <int NP>
static cudaError_t exchange3_np(const void* r_hi, const void* r_lo, double rscale, const GPad& gp, int W, int X, int M,
                                int N, double2* part, unsigned* status, cudaStream_t st) {
  constexpr int BN = 128;
  const int Mp = f16_ld(M);
  GemmMaps maps;
  memset(&maps, 0, sizeof(maps));
  cudaError_t e;
  if ((e = map_f16_pair(&maps.a_hi[0], &maps.a_lo[0], r_hi, r_lo, (long long)X * NP, M, Mp, kBM, false,
                        &maps.a_planes)) != cudaSuccess)
    return e;
  if ((e = map_f16_pair(&maps.b_hi, &maps.b_lo, gp.hi, gp.lo, (long long)W * 2 * NP, M, Mp, BN, false,
                        &maps.b_planes)) != cudaSuccess)
    return e;
  dim3 grid((W * 2 * NP + BN - 1) / BN, (X * NP + kBM - 1) / kBM, 1);
  // row tiles fastest, in groups of 148 (~15 MB of the padded Cholesky operand at M = 200):
  // one wave of CTAs multiplies a group against one Green's-function tile, the group stays in
  // L2 for the whole sweep over the walkers and the Green's function streams once per group
  const EpiExchange<NP, BN> epi{part, X, W, N, 1.0 / (rscale * rscale), gp.scale};
  return launch_umma<BN, 1, 3, 2, EpiExchange<NP, BN>, KIND_F16>(maps, M, 0, 0, grid, epi, status, st, true, true,
                                                                 148);
}

static cudaError_t exchange3(const void* r_hi, const void* r_lo, double rscale, const GPad& gp, int W, int X, int M,
                             int N, double2* part, unsigned* status, cudaStream_t st) {
  switch (exchange_np(N)) {
    case 8: return exchange3_np<8>(r_hi, r_lo, rscale, gp, W, X, M, N, part, status, st);
    case 16: return exchange3_np<16>(r_hi, r_lo, rscale, gp, W, X, M, N, part, status, st);
    case 32: return exchange3_np<32>(r_hi, r_lo, rscale, gp, W, X, M, N, part, status, st);
    default: return cudaErrorInvalidValue;
  }
}

int exchange3_rows(int X, int N) { return (X * exchange_np(N) + kBM - 1) / kBM; }

cudaError_t mixed_vhs(const void* cp_hi, const void* cp_lo, const int* ii, const int* jj, int P, int X, int M,
                      const void* xs_hi, const void* xs_lo, int W, double sqrt_dt, double cp_scale, int f16_planes,
                      double v_scale, void* re_hi, void* re_lo, void* im_hi, void* im_lo, unsigned* status,
                      cudaStream_t st) {
  // FP16 operands (packed Cholesky x cp_scale, fields x kFieldScaleF16) on 128 x 256 tiles
  // (two column groups of 128: half the re-reads of the packed Cholesky).  One CTA per tile:
  // measured faster here than persistent CTAs.
  constexpr int BN = 256;
  const int ldx = f16_ld(X);
  GemmMaps maps;
  memset(&maps, 0, sizeof(maps));
  cudaError_t e;
  if ((e = make_map_f16(&maps.a_hi[0], cp_hi, P, X, ldx, kBM)) != cudaSuccess) return e;
  if ((e = make_map_f16(&maps.a_lo[0], cp_lo, P, X, ldx, kBM)) != cudaSuccess) return e;
  if ((e = make_map_f16(&maps.b_hi, xs_hi, 2LL * W, X, ldx, BN)) != cudaSuccess) return e;
  if ((e = make_map_f16(&maps.b_lo, xs_lo, 2LL * W, X, ldx, BN)) != cudaSuccess) return e;
  dim3 grid((2 * W + BN - 1) / BN, (P + kBM - 1) / kBM, 1);
  const double unscale = sqrt_dt / (cp_scale * kFieldScaleF16);  // powers of two: exact
  if (f16_planes) {
    using H = __half*;
    EpiVHSF16<128> epi{H(re_hi), H(re_lo), H(im_hi), H(im_lo), ii, jj, P, M, f16_ld(M), W, (float)(unscale * v_scale)};
    return launch_umma<BN, 1, 3, 2, EpiVHSF16<128>, KIND_F16>(maps, X, 0, 0, grid, epi, status, st, false, false);
  }
  using F = float*;
  EpiVHSSplit<128> epi{F(re_hi), F(re_lo), F(im_hi), F(im_lo), ii, jj, P, M, W, (float)unscale};
  return launch_umma<BN, 1, 3, 2, EpiVHSSplit<128>, KIND_F16>(maps, X, 0, 0, grid, epi, status, st, false, false);
}

int vhs_blocks(int M) {
  const int nb = (M + 15) / 16;
  return nb * (nb + 1) / 2;
}

// The block-tiled VHS (EpiVHSBlock): fields (2W, X) as the left operand, the block-tiled
// Cholesky (vhs_blocks(M) * 256, X) as the right one, 128 x 256 tiles with the walker tiles
// fastest so that each Cholesky block is read from DRAM once while the fields stay in L2.
cudaError_t mixed_vhs_blocks(const void* cb_hi, const void* cb_lo, int X, int M, const void* xs_hi, const void* xs_lo,
                             int W, double sqrt_dt, double cb_scale, double v_scale, void* re_hi, void* re_lo,
                             void* im_hi, void* im_lo, int persistent, unsigned* status, cudaStream_t st) {
  constexpr int BN = 256;
  const int ldx = f16_ld(X);
  const int nblk = vhs_blocks(M);
  GemmMaps maps;
  memset(&maps, 0, sizeof(maps));
  cudaError_t e;
  if ((e = map_f16_pair(&maps.a_hi[0], &maps.a_lo[0], xs_hi, xs_lo, 2LL * W, X, ldx, kBM, true, &maps.a_planes)) !=
      cudaSuccess)
    return e;
  if ((e = map_f16_pair(&maps.b_hi, &maps.b_lo, cb_hi, cb_lo, 256LL * nblk, X, ldx, BN, true, &maps.b_planes)) !=
      cudaSuccess)
    return e;
  dim3 grid(nblk, (2 * W + kBM - 1) / kBM, 1);
  using H = __half*;
  void* planes[4] = {re_hi, re_lo, im_hi, im_lo};
  for (int p = 0; p < 4; ++p)
    if ((e = make_map_f16_store(&maps.out[p], planes[p], W, M, f16_ld(M), 16, 16, 64)) != cudaSuccess) return e;
  const EpiVHSBlock epi{M, W, (M + 15) / 16, (float)(sqrt_dt / (cb_scale * kFieldScaleF16) * v_scale)};
  // 64-byte K rows: four 48 KB stages instead of two of 96 KB, so that three are in flight
  return launch_umma<BN, 1, 3, 4, EpiVHSBlock, KIND_F16_K32>(maps, X, 0, 0, grid, epi, status, st, true,
                                                            persistent != 0);
}

// Orbital update of one spin block: phi_out = E exp(V) E phi_in (Taylor order nmax),
// every product on the tensor cores as 3-pass TF32; phi accumulates in FP64.
// E enters as its difference from the identity: (E - I) hi/lo (M, Mp) fp32 with Mp % 4 == 0; V: planar (W, M, M) hi/lo;
// b0/b1: two (W, 2N, M) fp32 hi/lo ping-pong buffers (4 arrays).
cudaError_t mixed_orbitals(const float* e_hi, const float* e_lo, int Mp, const float* v_re_hi, const float* v_re_lo,
                           const float* v_im_hi, const float* v_im_lo, const double2* phi_in, double2* phi_out,
                           float* b0_hi, float* b0_lo, float* b1_hi, float* b1_lo, int W, int M, int N, int nmax,
                           unsigned* status, cudaStream_t st) {
  constexpr int BN = 64;
  if (2 * N > BN || M % 4) return cudaErrorInvalidValue;
  phi_to_planar_kernel<<<grid_for((long long)W * M * N), 256, 0, st>>>(phi_in, W, M, N, b0_hi, b0_lo);
  note_launch();
  float* bh[2] = {b0_hi, b1_hi};
  float* bl[2] = {b0_lo, b1_lo};
  int cur = 0;
  cudaError_t e;
  const dim3 grid(1, (M + kBM - 1) / kBM, W);
  const int brows = 2 * N;
  // one-body (pre, post): A = E shared by all walkers (rows per batch 0)
  auto one_body = [&](int mode) -> cudaError_t {
    GemmMaps maps;
    memset(&maps, 0, sizeof(maps));
    cudaError_t r;
    if ((r = make_map(&maps.a_hi[0], e_hi, M, M, Mp, kBM)) != cudaSuccess) return r;
    if ((r = make_map(&maps.a_lo[0], e_lo, M, M, Mp, kBM)) != cudaSuccess) return r;
    if ((r = make_map(&maps.b_hi, bh[cur], (long long)W * brows, M, M, BN)) != cudaSuccess) return r;
    if ((r = make_map(&maps.b_lo, bl[cur], (long long)W * brows, M, M, BN)) != cudaSuccess) return r;
    EpiOrbital<1, BN> epi{mode == ORB_PRE ? phi_in : phi_out, phi_out, bh[cur ^ 1], bl[cur ^ 1], M, N, 1.0f, mode};
    r = launch_umma<BN, 1, 3, 3>(maps, M, 0, brows, grid, epi, status, st);
    cur ^= 1;
    return r;
  };
  if ((e = one_body(ORB_PRE)) != cudaSuccess) return e;
  for (int n = 1; n <= nmax; ++n) {
    GemmMaps maps;
    memset(&maps, 0, sizeof(maps));
    if ((e = make_map(&maps.a_hi[0], v_re_hi, (long long)W * M, M, M, kBM)) != cudaSuccess) return e;
    if ((e = make_map(&maps.a_lo[0], v_re_lo, (long long)W * M, M, M, kBM)) != cudaSuccess) return e;
    if ((e = make_map(&maps.a_hi[1], v_im_hi, (long long)W * M, M, M, kBM)) != cudaSuccess) return e;
    if ((e = make_map(&maps.a_lo[1], v_im_lo, (long long)W * M, M, M, kBM)) != cudaSuccess) return e;
    if ((e = make_map(&maps.b_hi, bh[cur], (long long)W * brows, M, M, BN)) != cudaSuccess) return e;
    if ((e = make_map(&maps.b_lo, bl[cur], (long long)W * brows, M, M, BN)) != cudaSuccess) return e;
    EpiOrbital<2, BN> epi{nullptr, phi_out, bh[cur ^ 1], bl[cur ^ 1], M, N, 1.0f / n,
                          n == nmax ? ORB_TERM_LAST : ORB_TERM};
    if ((e = launch_umma<BN, 2, 3, 2>(maps, M, M, brows, grid, epi, status, st)) != cudaSuccess) return e;
    cur ^= 1;
  }
  return one_body(ORB_POST);
}

}  // namespace umma
}  // namespace ipie_b200

extern "C" int ipie_b200_construct_force_bias_mixed(const void* ra_hi, const void* ra_lo, double ra_scale,
                                                    const void* rb_hi, const void* rb_lo, double rb_scale,
                                                    const void* ghalfa, const void* ghalfb, float* gwork, int W, int X,
                                                    int M, int na, int nb, void* vbias, unsigned int* status,
                                                    void* stream) {
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  const bool alias = nb == na && nb > 0 && rb_hi == ra_hi && ghalfb == ghalfa;
  const int NPa = umma::exchange_np(na), NPb = nb > 0 ? umma::exchange_np(nb) : 8;
  if (NPa < 0 || NPb < 0 || M < 4 || !(ra_scale > 0.0) || (nb > 0 && !(rb_scale > 0.0))) return (int)cudaErrorInvalidValue;
  const umma::GPad gp = umma::carve_gpad(gwork, W, 32, M);
  double2* v = reinterpret_cast<double2*>(vbias);
  cudaError_t e = umma::pad_ghalf(reinterpret_cast<const double2*>(ghalfa), W, M, na, NPa, gp, st);
  if (e == cudaSuccess)
    e = umma::coulomb3(ra_hi, ra_lo, ra_scale, gp, W, X, M, NPa, v, 0, alias ? 2.0 : 1.0, status, st);
  if (e != cudaSuccess || nb == 0 || alias) return (int)e;
  e = umma::pad_ghalf(reinterpret_cast<const double2*>(ghalfb), W, M, nb, NPb, gp, st);
  if (e == cudaSuccess) e = umma::coulomb3(rb_hi, rb_lo, rb_scale, gp, W, X, M, NPb, v, 1, 1.0, status, st);
  return (int)e;
}

extern "C" int ipie_b200_field_shift_mixed(const void* vbias, const double* xi, const void* mf_shift, int W, int X,
                                           double sqrt_dt, double bound, void* xshifted, void* xs_hi, void* xs_lo,
                                           void* cmf, void* cfb, void* stream) {
  return (int)launch_field_shift(reinterpret_cast<const double2*>(vbias), xi, reinterpret_cast<const double2*>(mf_shift),
                                 W, X, sqrt_dt, bound, reinterpret_cast<double2*>(xshifted),
                                 reinterpret_cast<double2*>(cmf), reinterpret_cast<double2*>(cfb),
                                 reinterpret_cast<cudaStream_t>(stream), xs_hi, xs_lo);
}

extern "C" int ipie_b200_construct_vhs_mixed(const void* cp_hi, const void* cp_lo, const int* idx_i,
                                             const int* idx_j, int M, int X, const void* xs_hi, const void* xs_lo,
                                             int W, double sqrt_dt, double cp_scale, int f16_planes, double v_scale,
                                             void* v_re_hi, void* v_re_lo, void* v_im_hi, void* v_im_lo,
                                             unsigned int* status, void* stream) {
  if (!(cp_scale > 0.0) || (f16_planes && !(v_scale > 0.0))) return (int)cudaErrorInvalidValue;
  return (int)umma::mixed_vhs(cp_hi, cp_lo, idx_i, idx_j, M * (M + 1) / 2, X, M, xs_hi, xs_lo, W, sqrt_dt, cp_scale,
                              f16_planes, v_scale, v_re_hi, v_re_lo, v_im_hi, v_im_lo, status,
                              reinterpret_cast<cudaStream_t>(stream));
}

extern "C" int ipie_b200_vhs_blocks(int M) { return M > 0 ? umma::vhs_blocks(M) : 0; }

extern "C" int ipie_b200_vhs_block_pack(const double* chol_packed, const int* rowmap, int M, int X, double scale,
                                        void* cb_hi, void* cb_lo, void* stream) {
  if (M <= 0 || X <= 0 || !(scale > 0.0)) return (int)cudaErrorInvalidValue;
  const long long R = 256LL * umma::vhs_blocks(M);
  const long long n = R * f16_ld(X);
  long long blocks = (n + 255) / 256;
  if (blocks > 148 * 32) blocks = 148 * 32;
  umma::vhs_block_pack_kernel<<<(unsigned)blocks, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      chol_packed, rowmap, R, X, f16_ld(X), scale, reinterpret_cast<__half*>(cb_hi), reinterpret_cast<__half*>(cb_lo));
  note_launch();
  return (int)cudaGetLastError();
}

extern "C" int ipie_b200_construct_vhs_blocks(const void* cb_hi, const void* cb_lo, int M, int X, const void* xs_hi,
                                              const void* xs_lo, int W, double sqrt_dt, double cb_scale,
                                              double v_scale, void* v_re_hi, void* v_re_lo, void* v_im_hi,
                                              void* v_im_lo, int flags, unsigned int* status, void* stream) {
  if (M <= 0 || X <= 0 || W <= 0 || !(cb_scale > 0.0) || !(v_scale > 0.0)) return (int)cudaErrorInvalidValue;
  return (int)umma::mixed_vhs_blocks(cb_hi, cb_lo, X, M, xs_hi, xs_lo, W, sqrt_dt, cb_scale, v_scale, v_re_hi,
                                     v_re_lo, v_im_hi, v_im_lo, flags & 1, status,
                                     reinterpret_cast<cudaStream_t>(stream));
}

extern "C" int ipie_b200_orbital_chain16_fits(int M, int N) { return umma::orbital_chain16_fits(M, N) ? 1 : 0; }

extern "C" int ipie_b200_propagate_orbitals_mixed16(const void* e_hi, const void* e_lo, double e_scale,
                                                    const void* v_re_hi, const void* v_re_lo, const void* v_im_hi,
                                                    const void* v_im_lo, double v_scale, const void* phi_in,
                                                    void* phi_out, int W, int M, int N, int nmax,
                                                    unsigned int* status, void* stream) {
  return (int)umma::mixed_orbital_chain16(e_hi, e_lo, (float)e_scale, v_re_hi, v_re_lo, v_im_hi, v_im_lo,
                                          (float)v_scale, reinterpret_cast<const double2*>(phi_in),
                                          reinterpret_cast<double2*>(phi_out), W, M, N, nmax, status,
                                          reinterpret_cast<cudaStream_t>(stream));
}

extern "C" int ipie_b200_propagate_orbitals_mixed(const float* e_hi, const float* e_lo, int lde, const float* v_re_hi,
                                                  const float* v_re_lo, const float* v_im_hi, const float* v_im_lo,
                                                  const void* phi_in, void* phi_out, float* work, int W, int M, int N,
                                                  int nmax, unsigned int* status, void* stream) {
  if (phi_in == phi_out || lde % 4 || lde < M) return (int)cudaErrorInvalidValue;
  if (umma::orbital_chain_fits(M, N))
    return (int)umma::mixed_orbital_chain(e_hi, e_lo, lde, v_re_hi, v_re_lo, v_im_hi, v_im_lo,
                                          reinterpret_cast<const double2*>(phi_in), reinterpret_cast<double2*>(phi_out),
                                          W, M, N, nmax, status, reinterpret_cast<cudaStream_t>(stream));
  const size_t plane = (size_t)W * 2 * N * M;
  return (int)umma::mixed_orbitals(e_hi, e_lo, lde, v_re_hi, v_re_lo, v_im_hi, v_im_lo,
                                   reinterpret_cast<const double2*>(phi_in), reinterpret_cast<double2*>(phi_out), work,
                                   work + plane, work + 2 * plane, work + 3 * plane, W, M, N, nmax, status,
                                   reinterpret_cast<cudaStream_t>(stream));
}

extern "C" int ipie_b200_rchol_pad_split(const double* rchol, int X, int N, int M, double scale, void* hi, void* lo,
                                         void* stream) {
  if (!(scale > 0.0)) return (int)cudaErrorInvalidValue;
  return (int)umma::mixed_rchol_pad(rchol, X, N, M, scale, reinterpret_cast<__half*>(hi), reinterpret_cast<__half*>(lo),
                                    reinterpret_cast<cudaStream_t>(stream));
}

// Per-walker sum of the exchange partial rows: out[w] = sum_t part[t * W + w].
__global__ void row_sum_kernel(const double2* __restrict__ part, int rows, int W, double2* __restrict__ out) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= W) return;
  double2 acc = make_double2(0.0, 0.0);
  for (int t = 0; t < rows; ++t) acc = cadd(acc, part[(size_t)t * W + w]);
  out[w] = acc;
}

extern "C" int ipie_b200_exchange_mixed(const void* r_hi, const void* r_lo, double r_scale, const void* ghalf,
                                        const void* ghalf_trial, const void* kmat, const void* raw_trial, int W, int X,
                                        int M, int N, float* gwork, void* part, void* exx, unsigned int* status,
                                        void* stream) {
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  using CC = const double2*;
  const int NP = umma::exchange_np(N);
  if (NP < 0 || M < 4 || W <= 0 || X <= 0 || !(r_scale > 0.0)) return (int)cudaErrorInvalidValue;
  const bool delta = ghalf_trial != nullptr;
  if (delta && (kmat == nullptr || raw_trial == nullptr)) return (int)cudaErrorInvalidValue;
  const umma::GPad gp = umma::carve_gpad(gwork, W, 32, M);
  double2* p = reinterpret_cast<double2*>(part);
  cudaError_t e = umma::pad_ghalf((CC)ghalf, W, M, N, NP, gp, st, delta ? (CC)ghalf_trial : nullptr);
  if (e == cudaSuccess) e = umma::exchange3(r_hi, r_lo, r_scale, gp, W, X, M, N, p, status, st);
  if (e != cudaSuccess) return (int)e;
  int rows = umma::exchange3_rows(X, N);
  if (delta) {
    e = umma::exchange_ref_row((CC)ghalf, (CC)ghalf_trial, (CC)kmat, W, N * M, (CC)raw_trial, p + (size_t)rows * W, st);
    if (e != cudaSuccess) return (int)e;
    rows += 1;
  }
  row_sum_kernel<<<(W + 127) / 128, 128, 0, st>>>(p, rows, W, reinterpret_cast<double2*>(exx));
  note_launch();
  return (int)cudaGetLastError();
}

// rows 1..W-1 of xv (W, X) = row 0 (the trial's Coulomb vector, before the per-walker deviations)
__global__ void broadcast_row0_kernel(double2* __restrict__ xv, int W, int X) {
  const long long n = (long long)(W - 1) * X;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
    xv[X + e] = xv[e % X];
}

extern "C" int ipie_b200_local_energy_mixed(int rhf, const double* rchola, const double* rcholb, const void* ra_hi,
                                            const void* ra_lo, double ra_scale, const void* rb_hi, const void* rb_lo,
                                            double rb_scale, const void* rH1a, const void* rH1b, double ecore, const void* ghalfa,
                                            const void* ghalfb, const void* ghalf_trial_a,
                                            const void* ghalf_trial_b, const void* kmat_a, const void* kmat_b,
                                            const void* raw_trial, int W, int X, int M, int na, int nb, float* gwork,
                                            void* work, void* energy, unsigned int* status, void* stream) {
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  const bool alias = !rhf && nb == na && nb > 0 && rb_hi == ra_hi && ghalfb == ghalfa;
  const int use_b = (!rhf && nb > 0 && !alias);
  const bool delta = ghalf_trial_a != nullptr;
  if (delta && (kmat_a == nullptr || raw_trial == nullptr || (use_b && (ghalf_trial_b == nullptr || kmat_b == nullptr))))
    return (int)cudaErrorInvalidValue;
  using CC = const double2*;
  double2* xv = reinterpret_cast<double2*>(work);
  double2* part = xv + (size_t)W * X;
  const int NPa = umma::exchange_np(na), NPb = nb > 0 ? umma::exchange_np(nb) : 8;
  if (NPa < 0 || NPb < 0 || M < 4 || !(ra_scale > 0.0) || (use_b && !(rb_scale > 0.0))) return (int)cudaErrorInvalidValue;
  const umma::GPad gp = umma::carve_gpad(gwork, W, 32, M);
  cudaError_t e;
  if (delta) {
    // Coulomb vector around the trial: X_T = sum_s rchol_s . G_T,s in FP64 (one walker's product,
    // into row 0, then copied to every row), plus the 3-pass FP16 product of G - G_T added per
    // spin block below, so that only the deviation carries the tensor cores' rounding
    e = umma::coulomb_row(rchola, (CC)ghalf_trial_a, X, na * M, xv, 0, alias ? 2.0 : 1.0, st);
    if (e == cudaSuccess && use_b) e = umma::coulomb_row(rcholb, (CC)ghalf_trial_b, X, nb * M, xv, 1, 1.0, st);
    if (e != cudaSuccess) return (int)e;
    if (W > 1) {
      long long blocks = ((long long)(W - 1) * X + 255) / 256;
      if (blocks > 148 * 16) blocks = 148 * 16;
      broadcast_row0_kernel<<<(unsigned)blocks, 256, 0, st>>>(xv, W, X);
      note_launch();
      if ((e = cudaGetLastError()) != cudaSuccess) return (int)e;
    }
  } else {
    // Coulomb vector in FP64 (DMMA): the Coulomb energy is the large, cancellation-free term
    e = launch_force_bias(rchola, reinterpret_cast<const double2*>(ghalfa), W, X, na * M, xv, 0, st,
                          alias ? 2.0 : 1.0);
    if (e == cudaSuccess && use_b)
      e = launch_force_bias(rcholb, reinterpret_cast<const double2*>(ghalfb), W, X, nb * M, xv, 1, st);
    if (e != cudaSuccess) return (int)e;
  }
  // exchange: 3-pass FP16 tensor-core products (of G - G_T when the trial reference is given),
  // bilinear sums in FP64; the reference row adds raw(G_T) + K.(G - G_T) in FP64
  e = umma::pad_ghalf((CC)ghalfa, W, M, na, NPa, gp, st, delta ? (CC)ghalf_trial_a : nullptr);
  if (e == cudaSuccess && delta)
    e = umma::coulomb3(ra_hi, ra_lo, ra_scale, gp, W, X, M, NPa, xv, 1, alias ? 2.0 : 1.0, status, st);
  if (e == cudaSuccess) e = umma::exchange3(ra_hi, ra_lo, ra_scale, gp, W, X, M, na, part, status, st);
  if (e != cudaSuccess) return (int)e;
  int rows = umma::exchange3_rows(X, na);
  if (use_b) {
    e = umma::pad_ghalf((CC)ghalfb, W, M, nb, NPb, gp, st, delta ? (CC)ghalf_trial_b : nullptr);
    if (e == cudaSuccess && delta) e = umma::coulomb3(rb_hi, rb_lo, rb_scale, gp, W, X, M, NPb, xv, 1, 1.0, status, st);
    if (e == cudaSuccess)
      e = umma::exchange3(rb_hi, rb_lo, rb_scale, gp, W, X, M, nb, part + (size_t)rows * W, status, st);
    if (e != cudaSuccess) return (int)e;
    rows += umma::exchange3_rows(X, nb);
  }
  if (delta) {
    e = umma::exchange_ref_row((CC)ghalfa, (CC)ghalf_trial_a, (CC)kmat_a, W, na * M, (CC)raw_trial,
                               part + (size_t)rows * W, st);
    rows += 1;
    if (e == cudaSuccess && use_b) {
      e = umma::exchange_ref_row((CC)ghalfb, (CC)ghalf_trial_b, (CC)kmat_b, W, nb * M, (CC)raw_trial + 1,
                                 part + (size_t)rows * W, st);
      rows += 1;
    }
    if (e != cudaSuccess) return (int)e;
  }
  const double f1 = rhf ? 2.0 : 1.0, fc = rhf ? 2.0 : 0.5, fx = (rhf || alias) ? 1.0 : 0.5;
  const bool e1_b = !rhf && nb > 0;
  return (int)launch_energy_combine(W, X, na * M, nb * M, reinterpret_cast<const double2*>(ghalfa),
                                    e1_b ? reinterpret_cast<const double2*>(ghalfb) : nullptr,
                                    reinterpret_cast<const double2*>(rH1a), reinterpret_cast<const double2*>(rH1b),
                                    ecore, xv, part, rows, f1, fc, fx, reinterpret_cast<double2*>(energy), status, st);
}
