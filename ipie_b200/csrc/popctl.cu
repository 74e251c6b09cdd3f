// Pair-branch population control decided on the device (throughput mode).
//
// ipie decides pair branching on the host: it gathers |w|, rescales the
// weights by total |w| / target (walkers/pop_controller.py:78-125), sorts |w|
// (stable mergesort), walks pairs inward from both ends while the lightest
// walker is below min_weight or the heaviest above max_weight, draws one
// uniform per pair to choose the survivor, and sends the survivor's buffer
// to the killed walker (:304-429).  This kernel does the same in one CTA so
// that the step needs no device-to-host round trip and can sit in a CUDA
// graph:
//
//   * the total is a fixed-order reduction (deterministic run to run);
//   * the sort is a bitonic network on (|w|, walker index) pairs, which
//     orders equal weights by index exactly as a stable sort does;
//   * the uniforms come from Philox4x32-10 keyed by the seed, with the
//     counter block read from device memory and advanced by one per call,
//     one uniform per pair in pair order;
//   * the pairing walk itself is serial (one thread; it visits only the
//     pairs formed, a few percent of the walkers);
//   * the result is a source index per walker for ipie_b200_walker_copy:
//     the survivor of a pair gets half the pair's weight, the killed walker
//     receives either the highest-index survivor's buffer (ipie's
//     single-process semantics, where every send carries the same tag and
//     the last one wins) or its own pair's survivor (ipie's semantics when
//     the pairs live on different ranks).
//
// A total weight below 1e-8 (ipie raises ValueError there) leaves every
// weight untouched and raises status bit 16.
#include <limits.h>

#include "../../include/ipie_b200.h"
#include "common.cuh"
#include "kernels.h"
#include "philox.cuh"

namespace ipie_b200 {

constexpr int kPairMaxW = 8192;
constexpr int kPairThreads = 1024;

__device__ __forceinline__ bool key_less(double ka, int ia, double kb, int ib) {
  return ka < kb || (ka == kb && ia < ib);
}

size_t pair_branch_smem(int n2) { return (size_t)n2 * 8 + (size_t)(n2 / 2) * 8 + (size_t)n2 * 4 + (size_t)(n2 / 2); }

__global__ void __launch_bounds__(kPairThreads)
    pair_branch_kernel(int W, int n2, double* __restrict__ weight, double* __restrict__ unscaled, double target,
                       double wmin, double wmax, unsigned long long seed, unsigned long long* counter, int paired,
                       int* __restrict__ src, double* total_out, double* wbound_out, double* u_out, unsigned* status) {
  extern __shared__ __align__(16) unsigned char sm[];
  double* key = reinterpret_cast<double*>(sm);  // n2 sorted |w| / scale, then the walk's new weights
  double* uni = key + n2;                       // n2 / 2 uniforms, one per possible pair
  int* idx = reinterpret_cast<int*>(uni + n2 / 2);
  unsigned char* keep_e = reinterpret_cast<unsigned char*>(idx + n2);  // pair j: 1 if its heavier walker survives
  __shared__ double red[kPairThreads / 32];
  __shared__ unsigned long long ctr;
  __shared__ double s_total;
  __shared__ int s_ok, s_npairs, s_maxclone;
  const int t = threadIdx.x;

  double acc = 0.0;
  for (int i = t; i < W; i += blockDim.x) acc += fabs(weight[i]);
  acc = warp_sum(acc);
  if ((t & 31) == 0) red[t >> 5] = acc;
  if (t == 0) ctr = *counter;
  __syncthreads();
  if (t < 32) {
    double v = t < (int)(blockDim.x >> 5) ? red[t] : 0.0;
    v = warp_sum(v);
    if (t == 0) {
      s_total = v;
      s_ok = (v >= 1e-8 && isfinite(v)) ? 1 : 0;
    }
  }
  __syncthreads();
  const double total = s_total;
  if (!s_ok) {
    for (int i = t; i < W; i += blockDim.x) src[i] = -1;
    if (t == 0) {
      flag(status, (unsigned)STATUS_ZERO_WEIGHT | (isfinite(total) ? 0u : (unsigned)STATUS_NONFINITE));
      *counter = ctr + 1ull;
    }
    return;
  }
  const double scale = total / target;
  const double inf = __longlong_as_double(0x7ff0000000000000LL);
  for (int i = t; i < n2; i += blockDim.x) {
    if (i < W) {
      const double w = weight[i];
      const double ws = w / scale;
      unscaled[i] = w;
      weight[i] = ws;
      key[i] = fabs(ws);
      idx[i] = i;
    } else {
      key[i] = inf;
      idx[i] = INT_MAX;
    }
  }
  for (int k = t; k < n2 / 2; k += blockDim.x) {
    const U4 c{(unsigned)k, 0u, (unsigned)ctr, (unsigned)(ctr >> 32)};
    const U4 r = philox10(c, (unsigned)seed, (unsigned)(seed >> 32));
    uni[k] = u53(r.x, r.y);
  }
  __syncthreads();
  // bitonic sort, ascending in (|w|, index)
  for (int size = 2; size <= n2; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int i = t; i < n2 / 2; i += blockDim.x) {
        const int lo = 2 * i - (i & (stride - 1));
        const int hi = lo + stride;
        const double ka = key[lo], kb = key[hi];
        const int ia = idx[lo], ib = idx[hi];
        const bool up = (lo & size) == 0;
        if (up ? key_less(kb, ib, ka, ia) : key_less(ka, ia, kb, ib)) {
          key[lo] = kb;
          key[hi] = ka;
          idx[lo] = ib;
          idx[hi] = ia;
        }
      }
      __syncthreads();
    }
  }
  // the pairing walk: pair j joins sorted positions j and W - 1 - j
  if (t == 0) {
    int s = 0, e = W - 1, maxclone = -1;
    while (s < e) {
      const double ws = key[s], we = key[e];
      if (!(ws < wmin || we > wmax)) break;
      const double wab = ws + we;
      const double r = uni[s];
      if (u_out) u_out[s] = r;
      const bool ke = r < we / wab;
      keep_e[s] = ke ? 1 : 0;
      const int keep = ke ? e : s, drop = ke ? s : e;
      key[keep] = 0.5 * wab;
      key[drop] = 0.0;
      maxclone = max(maxclone, idx[keep]);
      ++s;
      --e;
    }
    s_npairs = s;
    s_maxclone = maxclone;
    total_out[0] = total;
    if (wbound_out) wbound_out[0] = 0.10 * total;
    *counter = ctr + 1ull;
  }
  __syncthreads();
  const int npairs = s_npairs, maxclone = s_maxclone;
  for (int p = t; p < W; p += blockDim.x) {
    const int i = idx[p];
    const int j = p < npairs ? p : (p >= W - npairs ? W - 1 - p : -1);
    int from = -1;
    if (j >= 0) {
      const int survivor = keep_e[j] ? W - 1 - j : j;
      if (p == survivor) {
        weight[i] = key[p];
      } else {
        from = paired ? idx[survivor] : maxclone;
      }
    }
    src[i] = from;
  }
}

cudaError_t launch_pair_branch(int W, double* weight, double* unscaled, double target, double wmin, double wmax,
                               unsigned long long seed, unsigned long long* counter, int paired, int* src,
                               double* total_out, double* wbound_out, double* u_out, unsigned* status,
                               cudaStream_t st) {
  if (W < 2 || W > kPairMaxW || !(target > 0.0)) return cudaErrorInvalidValue;
  int n2 = 2;
  while (n2 < W) n2 <<= 1;
  const size_t smem = pair_branch_smem(n2);
  cudaError_t e = cudaFuncSetAttribute(pair_branch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  pair_branch_kernel<<<1, kPairThreads, smem, st>>>(W, n2, weight, unscaled, target, wmin, wmax, seed, counter,
                                                    paired, src, total_out, wbound_out, u_out, status);
  note_launch();
  return cudaGetLastError();
}

}  // namespace ipie_b200

using namespace ipie_b200;

extern "C" int ipie_b200_pair_branch(int W, double* weight, double* unscaled_weight, double target_weight,
                                     double min_weight, double max_weight, unsigned long long seed,
                                     unsigned long long* counter, int paired, int* src, double* total_weight,
                                     double* wbound, double* uniforms, unsigned int* status, void* stream) {
  if (weight == nullptr || unscaled_weight == nullptr || counter == nullptr || src == nullptr ||
      total_weight == nullptr)
    return (int)cudaErrorInvalidValue;
  return (int)launch_pair_branch(W, weight, unscaled_weight, target_weight, min_weight, max_weight, seed, counter,
                                 paired, src, total_weight, wbound, uniforms, status,
                                 reinterpret_cast<cudaStream_t>(stream));
}
