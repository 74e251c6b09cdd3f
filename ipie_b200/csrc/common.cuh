// Shared device helpers for the B200 phaseless-AFQMC walker step.
//
// Complex numbers are stored interleaved (re, im) as double2, the layout of
// numpy/torch complex128.  Nothing here traps: kernels report numerical
// trouble through a status word that the host reads.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace ipie_b200 {

// Host-side count of kernels this library has enqueued (instrumentation).
void note_launch();

// Status bits written (atomicOr) into the device status word.
enum StatusBits : unsigned int {
  STATUS_NONFINITE = 1u << 0,     // NaN/Inf met in a weight, overlap or energy
  STATUS_SINGULAR = 1u << 1,      // exactly singular pivot in an overlap LU
  STATUS_BAD_SHAPE = 1u << 2,     // a kernel was launched with sizes it does not support
  STATUS_ZERO_NORM = 1u << 3,     // a zero column met in Gram-Schmidt
  STATUS_ZERO_WEIGHT = 1u << 4,   // total walker weight below 1e-8 in population control
};

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cmulc(double2 a, double2 b) {  // conj(a) * b
  return make_double2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
__device__ __forceinline__ double cabs2(double2 a) { return a.x * a.x + a.y * a.y; }
__device__ __forceinline__ double cabs_(double2 a) { return hypot(a.x, a.y); }
__device__ __forceinline__ double2 cdiv(double2 a, double2 b) {
  // Smith's algorithm for a / b.
  if (fabs(b.x) >= fabs(b.y)) {
    double r = b.y / b.x, d = b.x + b.y * r;
    return make_double2((a.x + a.y * r) / d, (a.y - a.x * r) / d);
  }
  double r = b.x / b.y, d = b.y + b.x * r;
  return make_double2((a.x * r + a.y) / d, (a.y * r - a.x) / d);
}
__device__ __forceinline__ double2 cexp_(double2 z) {
  double e = exp(z.x), s, c;
  sincos(z.y, &s, &c);
  return make_double2(e * c, e * s);
}
__device__ __forceinline__ bool finite2(double2 z) { return isfinite(z.x) && isfinite(z.y); }

// Warp-level f64 tensor-core MMA, m8n8k4: D(8x8) += A(8x4, row) * B(4x8, col).
// Fragment layout (PTX ISA, mma.m8n8k4 .f64): lane = 4*g + t;
//   a = A[g][t], b = B[t][g], d[i] = D[g][2t + i].
__device__ __forceinline__ void dmma884(double (&d)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

// 16-byte asynchronous copy global -> shared (cp.async, L2 only); src_bytes < 16 zero-fills the
// rest (0: all zeros, nothing read)
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, int src_bytes) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
// wait until at most N of this thread's committed groups are still in flight
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ double2 warp_sum2(double2 v) {
  v.x = warp_sum(v.x);
  v.y = warp_sum(v.y);
  return v;
}

// Block-wide sum of a double2 (blockDim.x a multiple of 32, <= 1024).
__device__ __forceinline__ double2 block_sum2(double2 v, double2* scratch32) {
  v = warp_sum2(v);
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  __syncthreads();
  if (lane == 0) scratch32[wid] = v;
  __syncthreads();
  double2 r = make_double2(0.0, 0.0);
  if (wid == 0) {
    if (lane < nw) r = scratch32[lane];
    r = warp_sum2(r);
    if (lane == 0) scratch32[0] = r;
  }
  __syncthreads();
  r = scratch32[0];
  __syncthreads();
  return r;
}

__device__ __forceinline__ void flag(unsigned int* status, unsigned int bits) {
  if (status) atomicOr(status, bits);
}

}  // namespace ipie_b200
