// Kernels of the response of an AFQMC block energy to a one-body coupling,
// differentiated through the walk (forward mode: every walker carries the
// derivative of its orbitals and weight along the coupling lambda).
//
// The walk is ipie's AD-AFQMC propagator (addons/adafqmc/propagation/
// propagator.py:190-249, an RHF walk with the (det ratio)^2 importance
// function, the 1/2 (|cos| + cos) projection and the 0.1 total-weight cap);
// the derivative is the pathwise one ipie takes with torch autograd
// (addons/adafqmc/qmc/adafqmc.py:300-344), with the auxiliary fields and the
// population-control choices held fixed.  The orbital propagation reuses the
// library's fused one-body . Taylor . one-body kernel on the block operators
// [[E, 0], [dE, E]] and [[V, 0], [dV, V]] acting on the stacked [phi; dphi]
// (the derivative of a polynomial in a matrix is the off-diagonal block of the
// same polynomial in the block matrix); these kernels do the rest:
//
//   ad_gf_kernel       O = phi^T psi*, Ghalf = O^-1 phi^T, log det O, and their
//                      derivatives dGhalf = O^-1 dphi^T - (O^-1 dO) Ghalf,
//                      d log det O = tr(O^-1 dO)
//   ad_field_kernel    bounded force bias xbar, shifted fields x - xbar (X, W)
//                      and sum_x x xbar - xbar^2 / 2, -sqrt(dt) sum_x xs mf,
//                      with derivatives
//   ad_weight_kernel   the weight factor, its derivative and the weight cap
//   ad_reortho_kernel  modified Gram-Schmidt of phi; the same triangular map
//                      applied to dphi (every observable is invariant under
//                      phi -> phi T, so the derivative may follow the gauge)
//   ad_block_vhs_kernel the block operator [[V, 0], [dV, V]]
#include "../../include/ipie_b200.h"
#include "common.cuh"
#include "kernels.h"

namespace ipie_b200 {

constexpr int kAdMaxN = 32;

__device__ __forceinline__ double2 clog_(double2 z) {
  return make_double2(log(hypot(z.x, z.y)), atan2(z.y, z.x));
}

// One CTA per walker.  phi and dphi: (M, N) row-major blocks at phi + w * ld_w and
// dphi + w * ld_w.  psi_c = conj(trial) (M, N).  Out: g, dg (W, N, M); logdet, dlogdet (W).
__global__ void ad_gf_kernel(const double2* __restrict__ phi, const double2* __restrict__ dphi, long long ld_w, int M,
                             int N, const double2* __restrict__ psi_c, double2* __restrict__ g, double2* __restrict__ dg,
                             double2* __restrict__ logdet, double2* __restrict__ dlogdet, unsigned* status) {
  // N x N matrices with rows padded to N + 1 (dynamic shared memory)
  extern __shared__ double2 ad_sm[];
  const int ld = N + 1;
  double2* o = ad_sm;              // O, reduced to I by Gauss-Jordan; then P = O^-1 dO
  double2* oi = o + N * ld;        // O^-1
  double2* od = oi + N * ld;       // dO
  double2* fcol = od + N * ld;     // column k of O before each elimination step
  __shared__ double2 piv_ld;                    // running log det
  __shared__ int piv_row;
  const int w = blockIdx.x, t = threadIdx.x, nt = blockDim.x;
  const double2* p = phi + w * ld_w;
  const double2* dp = dphi + w * ld_w;
  for (int e = t; e < N * N; e += nt) {
    const int i = e / N, j = e % N;
    double2 a = make_double2(0.0, 0.0), b = make_double2(0.0, 0.0);
    for (int m = 0; m < M; ++m) {
      const double2 c = psi_c[(size_t)m * N + j];
      a = cadd(a, cmul(p[(size_t)m * N + i], c));
      b = cadd(b, cmul(dp[(size_t)m * N + i], c));
    }
    o[(i) * ld + (j)] = a;
    od[(i) * ld + (j)] = b;
    oi[(i) * ld + (j)] = make_double2(i == j ? 1.0 : 0.0, 0.0);
  }
  if (t == 0) piv_ld = make_double2(0.0, 0.0);
  __syncthreads();
  // Gauss-Jordan with partial pivoting on [O | I]
  for (int k = 0; k < N; ++k) {
    if (t == 0) {
      int r = k;
      double best = cabs2(o[(k) * ld + (k)]);
      for (int i = k + 1; i < N; ++i)
        if (cabs2(o[(i) * ld + (k)]) > best) {
          best = cabs2(o[(i) * ld + (k)]);
          r = i;
        }
      piv_row = r;
      if (best == 0.0) flag(status, STATUS_SINGULAR);
    }
    __syncthreads();
    const int r = piv_row;
    if (r != k)
      for (int j = t; j < N; j += nt) {
        double2 a = o[(k) * ld + (j)];
        o[(k) * ld + (j)] = o[(r) * ld + (j)];
        o[(r) * ld + (j)] = a;
        a = oi[(k) * ld + (j)];
        oi[(k) * ld + (j)] = oi[(r) * ld + (j)];
        oi[(r) * ld + (j)] = a;
      }
    __syncthreads();
    const double2 pv = o[(k) * ld + (k)];
    if (t == 0) {
      double2 l = clog_(pv);
      if (r != k) l.y += 3.141592653589793238462643383279502884;  // a row swap flips the sign
      piv_ld = cadd(piv_ld, l);
    }
    __syncthreads();
    const double2 inv = cdiv(make_double2(1.0, 0.0), pv);
    for (int j = t; j < N; j += nt) {
      o[(k) * ld + (j)] = cmul(o[(k) * ld + (j)], inv);
      oi[(k) * ld + (j)] = cmul(oi[(k) * ld + (j)], inv);
    }
    for (int i = t; i < N; i += nt) fcol[i] = o[(i) * ld + (k)];
    __syncthreads();
    for (int e = t; e < N * N; e += nt) {
      const int i = e / N, j = e % N;
      if (i == k) continue;
      const double2 f = fcol[i];
      o[(i) * ld + (j)] = csub(o[(i) * ld + (j)], cmul(f, o[(k) * ld + (j)]));
      oi[(i) * ld + (j)] = csub(oi[(i) * ld + (j)], cmul(f, oi[(k) * ld + (j)]));
    }
    __syncthreads();
  }
  // P = O^-1 dO (into o, which is no longer needed)
  for (int e = t; e < N * N; e += nt) {
    const int i = e / N, j = e % N;
    double2 s = make_double2(0.0, 0.0);
    for (int k = 0; k < N; ++k) s = cadd(s, cmul(oi[(i) * ld + (k)], od[(k) * ld + (j)]));
    o[(i) * ld + (j)] = s;
  }
  __syncthreads();
  if (t == 0) {
    double2 tr = make_double2(0.0, 0.0);
    for (int i = 0; i < N; ++i) tr = cadd(tr, o[(i) * ld + (i)]);
    logdet[w] = piv_ld;
    dlogdet[w] = tr;
  }
  // Ghalf = O^-1 phi^T and dGhalf = O^-1 dphi^T - P Ghalf, column by column (m)
  double2* gw = g + (size_t)w * N * M;
  double2* dgw = dg + (size_t)w * N * M;
  for (int m = t; m < M; m += nt) {
    double2 gc[kAdMaxN];
    for (int i = 0; i < N; ++i) {
      double2 s = make_double2(0.0, 0.0), d = make_double2(0.0, 0.0);
      for (int j = 0; j < N; ++j) {
        s = cadd(s, cmul(oi[(i) * ld + (j)], p[(size_t)m * N + j]));
        d = cadd(d, cmul(oi[(i) * ld + (j)], dp[(size_t)m * N + j]));
      }
      gc[i] = s;
      gw[(size_t)i * M + m] = s;
      dgw[(size_t)i * M + m] = d;
    }
    for (int i = 0; i < N; ++i) {
      double2 s = dgw[(size_t)i * M + m];
      for (int j = 0; j < N; ++j) s = csub(s, cmul(o[(i) * ld + (j)], gc[j]));
      dgw[(size_t)i * M + m] = s;
    }
  }
}

// One CTA per walker.  vbias, dvbias, x: (W, X); mf (X).  Out: xs, dxs (X, W) (transposed for the
// VHS product); fb = sum x xbar - xbar^2/2, mfs = -sqrt(dt) sum xs mf and their derivatives (W).
__global__ void ad_field_kernel(const double2* __restrict__ vbias, const double2* __restrict__ dvbias,
                                const double* __restrict__ x, const double2* __restrict__ mf, int W, int X,
                                double sqrt_dt, double bound, double2* __restrict__ xs, double2* __restrict__ dxs,
                                double2* __restrict__ fb, double2* __restrict__ dfb, double2* __restrict__ mfs,
                                double2* __restrict__ dmfs) {
  __shared__ double2 red[32];
  const int w = blockIdx.x;
  double2 s_fb = make_double2(0.0, 0.0), s_dfb = s_fb, s_mf = s_fb, s_dmf = s_fb;
  for (int k = threadIdx.x; k < X; k += blockDim.x) {
    const double2 vb = vbias[(size_t)w * X + k], dvb = dvbias[(size_t)w * X + k], f = mf[k];
    // xbar = -sqrt(dt) (i vbias - mf), dxbar = -sqrt(dt) i dvbias
    double2 xb = make_double2(sqrt_dt * (vb.y + f.x), sqrt_dt * (-vb.x + f.y));
    double2 dxb = make_double2(sqrt_dt * dvb.y, -sqrt_dt * dvb.x);
    const double a = hypot(xb.x, xb.y);
    if (a > bound) {
      // xbar / |xbar|: d = dxbar / a - xbar Re(conj(xbar) dxbar) / a^3
      const double re = (xb.x * dxb.x + xb.y * dxb.y) / (a * a * a);
      dxb = make_double2(dxb.x / a - xb.x * re, dxb.y / a - xb.y * re);
      xb = make_double2(xb.x / a, xb.y / a);
    }
    const double xv = x[(size_t)w * X + k];
    const double2 sh = make_double2(xv - xb.x, -xb.y);
    const double2 dsh = make_double2(-dxb.x, -dxb.y);
    xs[(size_t)k * W + w] = sh;
    dxs[(size_t)k * W + w] = dsh;
    s_fb = cadd(s_fb, csub(cscale(xb, xv), cscale(cmul(xb, xb), 0.5)));
    s_dfb = cadd(s_dfb, csub(cscale(dxb, xv), cmul(xb, dxb)));
    s_mf = cadd(s_mf, cmul(sh, f));
    s_dmf = cadd(s_dmf, cmul(dsh, f));
  }
  s_fb = block_sum2(s_fb, red);
  s_dfb = block_sum2(s_dfb, red);
  s_mf = block_sum2(s_mf, red);
  s_dmf = block_sum2(s_dmf, red);
  if (threadIdx.x == 0) {
    fb[w] = s_fb;
    dfb[w] = s_dfb;
    mfs[w] = cscale(s_mf, -sqrt_dt);
    dmfs[w] = cscale(s_dmf, -sqrt_dt);
  }
}

// One CTA for all walkers: w <- w |ratio expfb expmf exp(c)| max(cos theta, 0), theta =
// arg(ratio expmf), ratio = (det O_new / det O)^2, then w <- min(w, 0.1 sum w); the same for the
// derivatives.  c = dt (E_est - h0) and dc its derivative.
__global__ void ad_weight_kernel(int W, const double2* __restrict__ ld_old, const double2* __restrict__ dld_old,
                                 const double2* __restrict__ ld_new, const double2* __restrict__ dld_new,
                                 const double2* __restrict__ fb, const double2* __restrict__ dfb,
                                 const double2* __restrict__ mfs, const double2* __restrict__ dmfs, double c,
                                 double dc, double* __restrict__ weight, double* __restrict__ dweight,
                                 unsigned* status) {
  __shared__ double2 red[32];
  double2 acc = make_double2(0.0, 0.0);
  for (int w = threadIdx.x; w < W; w += blockDim.x) {
    const double2 lr = cscale(csub(ld_new[w], ld_old[w]), 2.0);
    const double2 dlr = cscale(csub(dld_new[w], dld_old[w]), 2.0);
    const double mod_log = lr.x + fb[w].x + mfs[w].x + c;
    const double theta = lr.y + mfs[w].y;
    const double dmod = dlr.x + dfb[w].x + dmfs[w].x + dc;
    const double dtheta = dlr.y + dmfs[w].y;
    double st, ct;
    sincos(theta, &st, &ct);
    const double mod = exp(mod_log);
    const double proj = 0.5 * (fabs(ct) + ct);
    const double factor = mod * proj;
    const double dfactor = mod * dmod * proj + (ct > 0.0 ? -mod * st * dtheta : 0.0);
    const double w0 = weight[w], dw0 = dweight[w];
    const double w1 = w0 * factor, dw1 = dw0 * factor + w0 * dfactor;
    if (!isfinite(w1) || !isfinite(dw1)) flag(status, STATUS_NONFINITE);
    weight[w] = w1;
    dweight[w] = dw1;
    acc = cadd(acc, make_double2(w1, dw1));
  }
  acc = block_sum2(acc, red);
  const double bound = 0.10 * acc.x, dbound = 0.10 * acc.y;
  for (int w = threadIdx.x; w < W; w += blockDim.x)
    if (!(weight[w] < bound)) {
      weight[w] = bound;
      dweight[w] = dbound;
    }
}

// One CTA per walker: modified Gram-Schmidt of the columns of phi (M, N) in place, the same
// column operations on dphi.
__global__ void ad_reortho_kernel(double2* __restrict__ phi, double2* __restrict__ dphi, long long ld_w, int M,
                                  int N, unsigned* status) {
  __shared__ double2 red[32];
  double2* p = phi + blockIdx.x * ld_w;
  double2* dp = dphi + blockIdx.x * ld_w;
  for (int j = 0; j < N; ++j) {
    for (int k = 0; k < j; ++k) {
      double2 r = make_double2(0.0, 0.0);
      for (int m = threadIdx.x; m < M; m += blockDim.x) r = cadd(r, cmulc(p[(size_t)m * N + k], p[(size_t)m * N + j]));
      r = block_sum2(r, red);
      for (int m = threadIdx.x; m < M; m += blockDim.x) {
        p[(size_t)m * N + j] = csub(p[(size_t)m * N + j], cmul(r, p[(size_t)m * N + k]));
        dp[(size_t)m * N + j] = csub(dp[(size_t)m * N + j], cmul(r, dp[(size_t)m * N + k]));
      }
      __syncthreads();
    }
    double2 nn = make_double2(0.0, 0.0);
    for (int m = threadIdx.x; m < M; m += blockDim.x) nn.x += cabs2(p[(size_t)m * N + j]);
    nn = block_sum2(nn, red);
    if (!(nn.x > 0.0)) {
      if (threadIdx.x == 0) flag(status, STATUS_ZERO_NORM);
      continue;
    }
    const double inv = 1.0 / sqrt(nn.x);
    for (int m = threadIdx.x; m < M; m += blockDim.x) {
      p[(size_t)m * N + j] = cscale(p[(size_t)m * N + j], inv);
      dp[(size_t)m * N + j] = cscale(dp[(size_t)m * N + j], inv);
    }
    __syncthreads();
  }
}

// out (W, 2M, 2M) = [[V, 0], [dV, V]] from V, dV (W, M, M).
__global__ void ad_block_vhs_kernel(const double2* __restrict__ v, const double2* __restrict__ dv, int W, int M,
                                    double2* __restrict__ out) {
  const long long M2 = 2LL * M;
  const long long n = (long long)W * M2 * M2;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    const long long w = e / (M2 * M2), r = (e / M2) % M2, c = e % M2;
    double2 val = make_double2(0.0, 0.0);
    if (r < M && c < M)
      val = v[(w * M + r) * M + c];
    else if (r >= M && c >= M)
      val = v[(w * M + (r - M)) * M + (c - M)];
    else if (r >= M && c < M)
      val = dv[(w * M + (r - M)) * M + c];
    out[e] = val;
  }
}

// out = a + s b (complex arrays of n entries).
__global__ void ad_axpy_kernel(const double2* __restrict__ a, const double2* __restrict__ b, double s, long long n,
                               double2* __restrict__ out) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
    out[e] = cadd(a[e], cscale(b[e], s));
}

// out[d] = in[src[d]] for blocks of len complex entries (stochastic reconfiguration of [phi; dphi]).
__global__ void ad_gather_kernel(const int* __restrict__ src, long long len, const double2* __restrict__ in,
                                 double2* __restrict__ out) {
  const long long d = blockIdx.x, s = src[d];
  for (long long e = threadIdx.x; e < len; e += blockDim.x) out[d * len + e] = in[s * len + e];
}

}  // namespace ipie_b200

using namespace ipie_b200;

extern "C" int ipie_b200_ad_axpy(const void* a, const void* b, double s, long long n, void* out, void* stream) {
  if (n <= 0) return (int)cudaErrorInvalidValue;
  long long blocks = (n + 255) / 256;
  if (blocks > 148 * 16) blocks = 148 * 16;
  ad_axpy_kernel<<<(unsigned)blocks, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      reinterpret_cast<const double2*>(a), reinterpret_cast<const double2*>(b), s, n, reinterpret_cast<double2*>(out));
  note_launch();
  return (int)cudaGetLastError();
}

extern "C" int ipie_b200_ad_gather(const int* src, int W, long long len, const void* in, void* out, void* stream) {
  if (W <= 0 || len <= 0 || in == out) return (int)cudaErrorInvalidValue;
  ad_gather_kernel<<<W, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      src, len, reinterpret_cast<const double2*>(in), reinterpret_cast<double2*>(out));
  note_launch();
  return (int)cudaGetLastError();
}

extern "C" int ipie_b200_ad_greens_function(const void* phi, const void* dphi, long long walker_stride, int W, int M,
                                            int N, const void* psi_conj, void* ghalf, void* dghalf, void* logdet,
                                            void* dlogdet, unsigned int* status, void* stream) {
  if (W <= 0 || M <= 0 || N <= 0 || N > kAdMaxN || walker_stride < (long long)M * N) return (int)cudaErrorInvalidValue;
  const size_t smem = (size_t)(3 * N * (N + 1) + N) * sizeof(double2);
  cudaError_t e = cudaFuncSetAttribute(ad_gf_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return (int)e;
  ad_gf_kernel<<<W, 128, smem, reinterpret_cast<cudaStream_t>(stream)>>>(
      reinterpret_cast<const double2*>(phi), reinterpret_cast<const double2*>(dphi), walker_stride, M, N,
      reinterpret_cast<const double2*>(psi_conj), reinterpret_cast<double2*>(ghalf),
      reinterpret_cast<double2*>(dghalf), reinterpret_cast<double2*>(logdet), reinterpret_cast<double2*>(dlogdet),
      status);
  note_launch();
  return (int)cudaGetLastError();
}

extern "C" int ipie_b200_ad_field_shift(const void* vbias, const void* dvbias, const double* x, const void* mf, int W,
                                        int X, double sqrt_dt, double bound, void* xshifted, void* dxshifted, void* fb,
                                        void* dfb, void* mfs, void* dmfs, void* stream) {
  if (W <= 0 || X <= 0) return (int)cudaErrorInvalidValue;
  ad_field_kernel<<<W, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      reinterpret_cast<const double2*>(vbias), reinterpret_cast<const double2*>(dvbias), x,
      reinterpret_cast<const double2*>(mf), W, X, sqrt_dt, bound, reinterpret_cast<double2*>(xshifted),
      reinterpret_cast<double2*>(dxshifted), reinterpret_cast<double2*>(fb), reinterpret_cast<double2*>(dfb),
      reinterpret_cast<double2*>(mfs), reinterpret_cast<double2*>(dmfs));
  note_launch();
  return (int)cudaGetLastError();
}

extern "C" int ipie_b200_ad_update_weight(int W, const void* logdet_old, const void* dlogdet_old, const void* logdet_new,
                                          const void* dlogdet_new, const void* fb, const void* dfb, const void* mfs,
                                          const void* dmfs, double c, double dc, double* weight, double* dweight,
                                          unsigned int* status, void* stream) {
  if (W <= 0) return (int)cudaErrorInvalidValue;
  ad_weight_kernel<<<1, 1024, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      W, reinterpret_cast<const double2*>(logdet_old), reinterpret_cast<const double2*>(dlogdet_old),
      reinterpret_cast<const double2*>(logdet_new), reinterpret_cast<const double2*>(dlogdet_new),
      reinterpret_cast<const double2*>(fb), reinterpret_cast<const double2*>(dfb),
      reinterpret_cast<const double2*>(mfs), reinterpret_cast<const double2*>(dmfs), c, dc, weight, dweight, status);
  note_launch();
  return (int)cudaGetLastError();
}

extern "C" int ipie_b200_ad_reortho(void* phi, void* dphi, long long walker_stride, int W, int M, int N,
                                    unsigned int* status, void* stream) {
  if (W <= 0 || M <= 0 || N <= 0 || walker_stride < (long long)M * N) return (int)cudaErrorInvalidValue;
  ad_reortho_kernel<<<W, 128, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      reinterpret_cast<double2*>(phi), reinterpret_cast<double2*>(dphi), walker_stride, M, N, status);
  note_launch();
  return (int)cudaGetLastError();
}

extern "C" int ipie_b200_ad_block_vhs(const void* vhs, const void* dvhs, int W, int M, void* out, void* stream) {
  if (W <= 0 || M <= 0) return (int)cudaErrorInvalidValue;
  const long long n = (long long)W * 4 * M * M;
  long long blocks = (n + 255) / 256;
  if (blocks > 148 * 16) blocks = 148 * 16;
  ad_block_vhs_kernel<<<(unsigned)blocks, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      reinterpret_cast<const double2*>(vhs), reinterpret_cast<const double2*>(dvhs), W, M,
      reinterpret_cast<double2*>(out));
  note_launch();
  return (int)cudaGetLastError();
}
