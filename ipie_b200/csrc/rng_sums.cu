// Device normal draws (Philox4x32-10 + Box-Muller) for the throughput mode and
// deterministic per-walker block sums for the estimators and accumulators.
#include "common.cuh"
#include "kernels.h"
#include "philox.cuh"

namespace ipie_b200 {

__global__ void normal_fill_kernel(double* __restrict__ out, long long n, unsigned long long seed,
                                   unsigned long long offset) {
  const long long pairs = (n + 1) / 2;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < pairs; i += (long long)gridDim.x * blockDim.x) {
    U4 c{(unsigned)i, (unsigned)(i >> 32), (unsigned)offset, (unsigned)(offset >> 32)};
    U4 r = philox10(c, (unsigned)seed, (unsigned)(seed >> 32));
    const double u1 = u53(r.x, r.y), u2 = u53(r.z, r.w);
    const double rad = sqrt(-2.0 * log(u1));
    double s, co;
    sincospi(2.0 * u2, &s, &co);
    out[2 * i] = rad * co;
    if (2 * i + 1 < n) out[2 * i + 1] = rad * s;
  }
}

cudaError_t launch_normal_fill(double* out, long long n, unsigned long long seed, unsigned long long offset,
                               cudaStream_t st) {
  const long long pairs = (n + 1) / 2;
  long long blocks = (pairs + 255) / 256;
  if (blocks > 148 * 16) blocks = 148 * 16;
  if (blocks < 1) blocks = 1;
  normal_fill_kernel<<<(unsigned)blocks, 256, 0, st>>>(out, n, seed, offset);
  note_launch();
  return cudaGetLastError();
}

// Same draws with the counter block read from device memory and advanced by one
// afterwards (two launches): a captured CUDA graph then draws a new block per replay.
__global__ void normal_fill_dev_kernel(double* __restrict__ out, long long n, unsigned long long seed,
                                       const unsigned long long* __restrict__ counter) {
  const unsigned long long offset = *counter;
  const long long pairs = (n + 1) / 2;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < pairs; i += (long long)gridDim.x * blockDim.x) {
    U4 c{(unsigned)i, (unsigned)(i >> 32), (unsigned)offset, (unsigned)(offset >> 32)};
    U4 r = philox10(c, (unsigned)seed, (unsigned)(seed >> 32));
    const double u1 = u53(r.x, r.y), u2 = u53(r.z, r.w);
    const double rad = sqrt(-2.0 * log(u1));
    double s, co;
    sincospi(2.0 * u2, &s, &co);
    out[2 * i] = rad * co;
    if (2 * i + 1 < n) out[2 * i + 1] = rad * s;
  }
}

__global__ void counter_add_kernel(unsigned long long* counter, unsigned long long inc) { *counter += inc; }

cudaError_t launch_normal_fill_dev(double* out, long long n, unsigned long long seed, unsigned long long* counter,
                                   cudaStream_t st) {
  const long long pairs = (n + 1) / 2;
  long long blocks = (pairs + 255) / 256;
  if (blocks > 148 * 16) blocks = 148 * 16;
  if (blocks < 1) blocks = 1;
  normal_fill_dev_kernel<<<(unsigned)blocks, 256, 0, st>>>(out, n, seed, counter);
  note_launch();
  counter_add_kernel<<<1, 1, 0, st>>>(counter, 1ull);
  note_launch();
  return cudaGetLastError();
}

// Uniform (0, 1] doubles from the same generator (pair-branch draws on device).
__device__ double philox_uniform(unsigned long long seed, unsigned long long offset, unsigned long long i) {
  U4 c{(unsigned)i, (unsigned)(i >> 32), (unsigned)offset, (unsigned)(offset >> 32) ^ 0x5bd1e995u};
  U4 r = philox10(c, (unsigned)seed, (unsigned)(seed >> 32));
  return u53(r.x, r.y);
}

// out[0..6] = [sum w, sum w_unscaled, sum w*E_hyb, sum w*Re E0, sum w, sum w*Re E1, sum w*Re E2]
// (complex).  One CTA, fixed reduction order (deterministic).
__global__ void __launch_bounds__(1024) walker_sums_kernel(int W, const double* __restrict__ weight,
                                                           const double* __restrict__ unscaled,
                                                           const double2* __restrict__ ehyb,
                                                           const double2* __restrict__ energy, double2* __restrict__ out,
                                                           int accumulate) {
  __shared__ double2 red[32];
  double2 a[7];
#pragma unroll
  for (int q = 0; q < 7; ++q) a[q] = make_double2(0.0, 0.0);
  for (int w = threadIdx.x; w < W; w += blockDim.x) {
    const double wt = weight[w];
    a[0].x += wt;
    if (unscaled) a[1].x += unscaled[w];
    if (ehyb) {
      a[2].x += wt * ehyb[w].x;
      a[2].y += wt * ehyb[w].y;
    }
    if (energy) {
      a[3].x += wt * energy[3 * w].x;
      a[4].x += wt;
      a[5].x += wt * energy[3 * w + 1].x;
      a[6].x += wt * energy[3 * w + 2].x;
    }
  }
#pragma unroll
  for (int q = 0; q < 7; ++q) {
    double2 r = block_sum2(a[q], red);
    if (threadIdx.x == 0) out[q] = accumulate ? cadd(out[q], r) : r;
  }
}

cudaError_t launch_walker_sums(int W, const double* weight, const double* unscaled, const double2* ehyb,
                               const double2* energy, double2* out, int accumulate, cudaStream_t st) {
  walker_sums_kernel<<<1, 1024, 0, st>>>(W, weight, unscaled, ehyb, energy, out, accumulate);
  note_launch();
  return cudaGetLastError();
}

}  // namespace ipie_b200
