// Learned control variate for the exchange energy: a small MLP
// (16 -> 256 -> 256 -> 1, SiLU) with bf16 weights and FP32 accumulation,
// trained on the GPU by these forward/backward/Adam kernels; plus the
// per-walker feature kernel and the subsampled unbiased correction.
//
// Layer convention: Y[b][n] = act(sum_k X[b][k] W[k][n] + bias[n]), W row-major (K, N).
#include <cuda_bf16.h>

#include "../../include/ipie_b200.h"
#include "common.cuh"
#include "kernels.h"

namespace ipie_b200 {

namespace {

constexpr int TS = 32;  // output tile edge

__device__ __forceinline__ float silu(float a) { return a / (1.0f + __expf(-a)); }
__device__ __forceinline__ float silu_grad(float a) {
  const float s = 1.0f / (1.0f + __expf(-a));
  return s * (1.0f + a * (1.0f - s));
}

template <class T>
__device__ __forceinline__ float ld(const T* p, size_t i);
template <>
__device__ __forceinline__ float ld<float>(const float* p, size_t i) { return p[i]; }
template <>
__device__ __forceinline__ float ld<__nv_bfloat16>(const __nv_bfloat16* p, size_t i) { return __bfloat162float(p[i]); }

// C[r][c] (+)= sum_k A(r, k) B(k, c) where A(r,k) = TA ? A[k*lda + r] : A[r*lda + k]
// and B(k,c) = TB ? B[c*ldb + k] : B[k*ldb + c]; 32x32 output tile per 256 threads (4 each).
template <bool TA, bool TB, class TAe, class TBe>
__global__ void __launch_bounds__(256) small_gemm_kernel(int R, int Cn, int K, const TAe* __restrict__ A, int lda,
                                                         const TBe* __restrict__ B, int ldb, float* __restrict__ C,
                                                         int ldc, int accumulate) {
  __shared__ float sA[TS][TS + 1];
  __shared__ float sB[TS][TS + 1];
  const int r0 = blockIdx.y * TS, c0 = blockIdx.x * TS;
  const int tx = threadIdx.x % TS, ty = threadIdx.x / TS;  // ty 0..7
  float acc[4] = {0.f, 0.f, 0.f, 0.f};
  for (int k0 = 0; k0 < K; k0 += TS) {
    for (int e = threadIdx.x; e < TS * TS; e += 256) {
      const int i = e / TS, j = e % TS;
      // sA[i][j] = A(r0+i, k0+j); sB[i][j] = B(k0+i, c0+j)
      const int r = r0 + i, k = k0 + j;
      sA[i][j] = (r < R && k < K) ? ld(A, TA ? (size_t)k * lda + r : (size_t)r * lda + k) : 0.f;
      const int kk = k0 + i, c = c0 + j;
      sB[i][j] = (kk < K && c < Cn) ? ld(B, TB ? (size_t)c * ldb + kk : (size_t)kk * ldb + c) : 0.f;
    }
    __syncthreads();
#pragma unroll 8
    for (int k = 0; k < TS; ++k) {
      const float b = sB[k][tx];
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[q] += sA[ty + 8 * q][k] * b;
    }
    __syncthreads();
  }
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int r = r0 + ty + 8 * q, c = c0 + tx;
    if (r < R && c < Cn) {
      float v = acc[q];
      if (accumulate) v += C[(size_t)r * ldc + c];
      C[(size_t)r * ldc + c] = v;
    }
  }
}

template <bool TA, bool TB, class TAe, class TBe>
cudaError_t small_gemm(int R, int Cn, int K, const TAe* A, int lda, const TBe* B, int ldb, float* C, int ldc,
                       int accumulate, cudaStream_t st) {
  dim3 grid((Cn + TS - 1) / TS, (R + TS - 1) / TS);
  small_gemm_kernel<TA, TB, TAe, TBe><<<grid, 256, 0, st>>>(R, Cn, K, A, lda, B, ldb, C, ldc, accumulate);
  note_launch();
  return cudaGetLastError();
}

// pre = Y + bias (in place), post = act(pre)
__global__ void bias_act_kernel(float* __restrict__ pre, float* __restrict__ post, const float* __restrict__ bias,
                                long long n, int N, int act) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float a = pre[i] + bias[i % N];
    pre[i] = a;
    post[i] = act ? silu(a) : a;
  }
}

// dA = dH * silu'(A)  (in place on dH)
__global__ void silu_bwd_kernel(float* __restrict__ dh, const float* __restrict__ pre, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    dh[i] *= silu_grad(pre[i]);
}

// column sums: db[n] (+)= sum_b dY[b][n]
__global__ void colsum_kernel(const float* __restrict__ dy, int B, int N, float* __restrict__ db, int accumulate) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  float s = 0.f;
  for (int b = 0; b < B; ++b) s += dy[(size_t)b * N + n];
  db[n] = accumulate ? db[n] + s : s;
}

// MSE on (pred - target): grad = 2 (pred - target) / B; loss partial sums in loss[0] (atomic)
__global__ void mse_grad_kernel(const float* __restrict__ pred, const float* __restrict__ target, int B,
                                float* __restrict__ grad, float* __restrict__ loss) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  float d = 0.f;
  if (b < B) {
    d = pred[b] - target[b];
    grad[b] = 2.0f * d / B;
  }
  float l = warp_sum(d * d);
  if ((threadIdx.x & 31) == 0 && loss) atomicAdd(loss, l / B);
}

// Adam on fp32 master weights, refreshed bf16 copy for the forward kernels.
__global__ void adam_kernel(float* __restrict__ master, __nv_bfloat16* __restrict__ wbf, const float* __restrict__ g,
                            float* __restrict__ m, float* __restrict__ v, long long n, float lr, float b1, float b2,
                            float eps, float bc1, float bc2) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float w = master[i] - lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
    master[i] = w;
    if (wbf) wbf[i] = __float2bfloat16(w);
  }
}

unsigned grid1(long long n) {
  long long b = (n + 255) / 256;
  if (b > 148 * 16) b = 148 * 16;
  return (unsigned)(b < 1 ? 1 : b);
}

}  // namespace

// Parameter block layout (fp32 master, bf16 copy, grads, Adam moments share it):
//   W1 (F, H), b1 (H), W2 (H, H), b2 (H), W3 (H, 1), b3 (1)
struct MlpDims {
  int F, H;
  size_t w1() const { return 0; }
  size_t b1() const { return (size_t)F * H; }
  size_t w2() const { return b1() + H; }
  size_t b2() const { return w2() + (size_t)H * H; }
  size_t w3() const { return b2() + H; }
  size_t b3() const { return w3() + H; }
  size_t total() const { return b3() + 1; }
};

// Forward pass; act buffers (may be null when not training): a1, h1, a2, h2 each (B, H).
cudaError_t mlp_forward(const float* x, int B, MlpDims d, const __nv_bfloat16* wbf, const float* master, float* a1,
                        float* h1, float* a2, float* h2, float* out, cudaStream_t st) {
  const int F = d.F, H = d.H;
  cudaError_t e;
  if ((e = small_gemm<false, false>(B, H, F, x, F, wbf + d.w1(), H, a1, H, 0, st)) != cudaSuccess) return e;
  bias_act_kernel<<<grid1((long long)B * H), 256, 0, st>>>(a1, h1, master + d.b1(), (long long)B * H, H, 1);
  note_launch();
  if ((e = small_gemm<false, false>(B, H, H, h1, H, wbf + d.w2(), H, a2, H, 0, st)) != cudaSuccess) return e;
  bias_act_kernel<<<grid1((long long)B * H), 256, 0, st>>>(a2, h2, master + d.b2(), (long long)B * H, H, 1);
  note_launch();
  if ((e = small_gemm<false, false>(B, 1, H, h2, H, wbf + d.w3(), 1, out, 1, 0, st)) != cudaSuccess) return e;
  bias_act_kernel<<<grid1(B), 256, 0, st>>>(out, out, master + d.b3(), B, 1, 0);
  note_launch();
  return cudaGetLastError();
}

// Backward of MSE(out, target) into grad (same layout as the parameters); dtmp (B, H) x 2 scratch.
cudaError_t mlp_backward(const float* x, const float* target, int B, MlpDims d, const __nv_bfloat16* wbf,
                         const float* a1, const float* h1, const float* a2, const float* h2, const float* out,
                         float* grad, float* dout, float* dh1, float* dh2, float* loss, cudaStream_t st) {
  const int F = d.F, H = d.H;
  cudaError_t e;
  mse_grad_kernel<<<(B + 255) / 256, 256, 0, st>>>(out, target, B, dout, loss);
  note_launch();
  // layer 3: dW3 = h2^T dout (H x 1), db3 = sum dout, dh2 = dout W3^T
  if ((e = small_gemm<true, false>(H, 1, B, h2, H, dout, 1, grad + d.w3(), 1, 0, st)) != cudaSuccess) return e;
  colsum_kernel<<<1, 32, 0, st>>>(dout, B, 1, grad + d.b3(), 0);
  note_launch();
  if ((e = small_gemm<false, true>(B, H, 1, dout, 1, wbf + d.w3(), 1, dh2, H, 0, st)) != cudaSuccess) return e;
  silu_bwd_kernel<<<grid1((long long)B * H), 256, 0, st>>>(dh2, a2, (long long)B * H);
  note_launch();
  // layer 2
  if ((e = small_gemm<true, false>(H, H, B, h1, H, dh2, H, grad + d.w2(), H, 0, st)) != cudaSuccess) return e;
  colsum_kernel<<<(H + 127) / 128, 128, 0, st>>>(dh2, B, H, grad + d.b2(), 0);
  note_launch();
  if ((e = small_gemm<false, true>(B, H, H, dh2, H, wbf + d.w2(), H, dh1, H, 0, st)) != cudaSuccess) return e;
  silu_bwd_kernel<<<grid1((long long)B * H), 256, 0, st>>>(dh1, a1, (long long)B * H);
  note_launch();
  // layer 1
  if ((e = small_gemm<true, false>(F, H, B, x, F, dh1, H, grad + d.w1(), H, 0, st)) != cudaSuccess) return e;
  colsum_kernel<<<(H + 127) / 128, 128, 0, st>>>(dh1, B, H, grad + d.b1(), 0);
  note_launch();
  return cudaGetLastError();
}

cudaError_t mlp_adam(float* master, __nv_bfloat16* wbf, const float* g, float* m, float* v, long long n, float lr,
                     int t, cudaStream_t st) {
  const float b1 = 0.9f, b2 = 0.999f;
  adam_kernel<<<grid1(n), 256, 0, st>>>(master, wbf, g, m, v, n, lr, b1, b2, 1e-8f, 1.f - powf(b1, (float)t),
                                        1.f - powf(b2, (float)t));
  note_launch();
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Per-walker features for the exchange control variate (16 per walker, fp32):
//  0,1  Re/Im e1b          2,3  Re/Im ecoul       4  sum_x |X|^2   5  sum_x (Re X)^2
//  6,7  cos/sin arg(ovlp)  8    log|ovlp|          9,10 Re/Im hybrid energy
// 11    sum |Ghalf|^2     12,13 Re/Im sum_i Ghalf[i, :] . psi*[:, i] (trial projection)
// 14    sum |Ghalf - Ghalf_T|^2 (distance from the trial density)   15  weight
// ---------------------------------------------------------------------------
// Per-spin sums of one walker's half-rotated Green's function G against the
// trial's G_T and the exchange gradient K at the trial:
//   (|G|^2, |G - G_T|^2) and lin = sum K (G - G_T)  (complex, no conjugation).
__device__ __forceinline__ void cv_spin_sums(const double2* __restrict__ g, const double2* __restrict__ gt,
                                             const double2* __restrict__ kmat, int NM, double2& g2, double2& lin) {
  for (int e = threadIdx.x; e < NM; e += blockDim.x) {
    const double2 a = g[e], t = gt[e];
    const double dx = a.x - t.x, dy = a.y - t.y;
    g2.x += a.x * a.x + a.y * a.y;
    g2.y += dx * dx + dy * dy;
    lin = cadd(lin, cmul(kmat[e], make_double2(dx, dy)));
  }
}

// One CTA per walker.  base[w] = Re(lin): the first-order change of the
// exchange term y = 1/2 Re(raw_a + raw_b) away from its trial value.
__global__ void __launch_bounds__(256) cv_features_kernel(int W, int X, int na, int nb, int M, bool alias,
                                                          const double2* __restrict__ energy,
                                                          const double2* __restrict__ xv,
                                                          const double2* __restrict__ ovlp,
                                                          const double2* __restrict__ ehyb,
                                                          const double2* __restrict__ ghalfa,
                                                          const double2* __restrict__ ghalfb,
                                                          const double2* __restrict__ gta,
                                                          const double2* __restrict__ gtb,
                                                          const double2* __restrict__ ka,
                                                          const double2* __restrict__ kb,
                                                          const double* __restrict__ weight,
                                                          const double* __restrict__ lead, float* __restrict__ feat,
                                                          double* __restrict__ base) {
  __shared__ double2 red[32];
  const int w = blockIdx.x;
  double2 sx = make_double2(0.0, 0.0);  // (sum |X|^2, sum (Re X)^2)
  for (int x = threadIdx.x; x < X; x += blockDim.x) {
    const double2 v = xv[(size_t)w * X + x];
    sx.x += v.x * v.x + v.y * v.y;
    sx.y += v.x * v.x;
  }
  double2 g2a = make_double2(0.0, 0.0), lina = make_double2(0.0, 0.0);
  double2 g2b = make_double2(0.0, 0.0), linb = make_double2(0.0, 0.0);
  cv_spin_sums(ghalfa + (size_t)w * na * M, gta, ka, na * M, g2a, lina);
  if (nb > 0 && !alias) cv_spin_sums(ghalfb + (size_t)w * nb * M, gtb, kb, nb * M, g2b, linb);
  sx = block_sum2(sx, red);
  g2a = block_sum2(g2a, red);
  lina = block_sum2(lina, red);
  g2b = block_sum2(g2b, red);
  linb = block_sum2(linb, red);
  if (threadIdx.x == 0) {
    // alias: both blocks are spin a (y = raw_a); otherwise y = (raw_a + raw_b) / 2
    const double fa = alias ? 1.0 : 0.5;
    const double2 lin = make_double2(fa * lina.x + 0.5 * linb.x, fa * lina.y + 0.5 * linb.y);
    const double g2 = alias ? 2.0 * g2a.x : g2a.x + g2b.x;
    const double d2 = alias ? 2.0 * g2a.y : g2a.y + g2b.y;
    float* f = feat + (size_t)w * 16;
    const double2 e1 = energy[(size_t)w * 3 + 1], e2 = energy[(size_t)w * 3 + 2];
    const double2 o = ovlp[w], h = ehyb[w];
    const double ao = hypot(o.x, o.y);
    f[0] = (float)e1.x;
    f[1] = (float)e1.y;
    f[2] = (float)e2.x;
    f[3] = (float)e2.y;
    f[4] = (float)sx.x;
    f[5] = (float)sx.y;
    f[6] = ao > 0 ? (float)(o.x / ao) : 1.f;
    f[7] = ao > 0 ? (float)(o.y / ao) : 0.f;
    f[8] = ao > 0 ? (float)log(ao) : 0.f;
    f[9] = (float)h.x;
    f[10] = (float)h.y;
    f[11] = (float)g2;
    f[12] = (float)lin.x;
    f[13] = (float)lin.y;
    f[14] = (float)d2;
    f[15] = lead != nullptr ? (float)lead[w] : (float)weight[w];
    base[w] = lin.x;
  }
}

// (x - mu) / sigma per feature column, in place
__global__ void normalize_kernel(float* __restrict__ x, long long rows, int F, const float* __restrict__ mu,
                                 const float* __restrict__ sigma) {
  const long long n = rows * F;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int f = (int)(i % F);
    x[i] = (x[i] - mu[f]) / sigma[f];
  }
}

// dst[s] = src[idx[s]] for rows of `row` complex elements
__global__ void gather_rows_kernel(const double2* __restrict__ src, const int* __restrict__ idx, int S, long long row,
                                   double2* __restrict__ dst) {
  const int s = blockIdx.x;
  if (s >= S) return;
  const double2* a = src + (size_t)idx[s] * row;
  double2* b = dst + (size_t)s * row;
  for (long long e = threadIdx.x; e < row; e += blockDim.x) b[e] = a[e];
}

// Control-variate energy sums (one CTA, fixed order):
//   out[0] = sum_w w (A_w - c_w),  out[1] = (W/S) sum_s w_s (y_s - c_s),  out[2] = sum_w w,
//   out[3] = sum_w w A_w (no exchange), out[4] = (W/S) sum_s w_s y_s (plain subsample estimate)
// with A_w = Re E_w of the exchange-free energy, c = prediction of the exchange term, y_s exact.
__global__ void __launch_bounds__(1024) cv_sums_kernel(int W, const double* __restrict__ weight,
                                                       const double2* __restrict__ energy_noexx,
                                                       const float* __restrict__ pred, int S, const int* __restrict__ idx,
                                                       const double* __restrict__ y_s, double* __restrict__ out) {
  __shared__ double2 red[32];
  double2 a = make_double2(0.0, 0.0), b = make_double2(0.0, 0.0), c = make_double2(0.0, 0.0);
  for (int w = threadIdx.x; w < W; w += blockDim.x) {
    const double wt = weight[w], A = energy_noexx[(size_t)w * 3].x;
    a.x += wt * (A - (double)pred[w]);
    a.y += wt;
    c.x += wt * A;
  }
  for (int s = threadIdx.x; s < S; s += blockDim.x) {
    const int w = idx[s];
    b.x += weight[w] * (y_s[s] - (double)pred[w]);
    b.y += weight[w] * y_s[s];
  }
  a = block_sum2(a, red);
  b = block_sum2(b, red);
  c = block_sum2(c, red);
  if (threadIdx.x == 0) {
    const double f = (double)W / S;
    out[0] = a.x;
    out[1] = f * b.x;
    out[2] = a.y;
    out[3] = c.x;
    out[4] = f * b.y;
  }
}

}  // namespace ipie_b200

using namespace ipie_b200;

extern "C" {

int ipie_b200_normalize_features(float* x, long long rows, int F, const float* mu, const float* sigma, void* stream) {
  normalize_kernel<<<grid1(rows * F), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(x, rows, F, mu, sigma);
  note_launch();
  return (int)cudaGetLastError();
}

int ipie_b200_gather_walkers(const void* src, const int* idx, int S, long long row, void* dst, void* stream) {
  if (S <= 0) return 0;
  gather_rows_kernel<<<S, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      reinterpret_cast<const double2*>(src), idx, S, row, reinterpret_cast<double2*>(dst));
  note_launch();
  return (int)cudaGetLastError();
}

int ipie_b200_cv_sums(int W, const double* weight, const void* energy_noexx, const float* pred, int S, const int* idx,
                      const double* y_s, double* out, void* stream) {
  cv_sums_kernel<<<1, 1024, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      W, weight, reinterpret_cast<const double2*>(energy_noexx), pred, S, idx, y_s, out);
  note_launch();
  return (int)cudaGetLastError();
}

int ipie_b200_mlp_forward(const float* x, int B, int F, int H, const void* wbf, const float* master, float* acts,
                          float* out, void* stream) {
  MlpDims d{F, H};
  const size_t bh = (size_t)B * H;
  return (int)mlp_forward(x, B, d, reinterpret_cast<const __nv_bfloat16*>(wbf), master, acts, acts + bh,
                          acts + 2 * bh, acts + 3 * bh, out, reinterpret_cast<cudaStream_t>(stream));
}

int ipie_b200_mlp_backward(const float* x, const float* target, int B, int F, int H, const void* wbf,
                           const float* acts, const float* out, float* grad, float* work, float* loss, void* stream) {
  MlpDims d{F, H};
  const size_t bh = (size_t)B * H;
  return (int)mlp_backward(x, target, B, d, reinterpret_cast<const __nv_bfloat16*>(wbf), acts, acts + bh, acts + 2 * bh,
                           acts + 3 * bh, out, grad, work, work + B, work + B + bh, loss,
                           reinterpret_cast<cudaStream_t>(stream));
}

int ipie_b200_mlp_adam(float* master, void* wbf, const float* grad, float* m, float* v, long long n, float lr, int t,
                       void* stream) {
  return (int)mlp_adam(master, reinterpret_cast<__nv_bfloat16*>(wbf), grad, m, v, n, lr, t,
                       reinterpret_cast<cudaStream_t>(stream));
}

int ipie_b200_cv_features(int W, int X, int na, int nb, int M, const void* energy, const void* xv, const void* ovlp,
                          const void* hybrid_energy, const void* ghalfa, const void* ghalfb, const void* ghalf_trial_a,
                          const void* ghalf_trial_b, const void* kmat_a, const void* kmat_b, const double* weight,
                          const double* lead, float* feat, double* base, void* stream) {
  const bool alias = nb == na && nb > 0 && ghalfb == ghalfa;
  if (nb > 0 && !alias && (ghalfb == nullptr || ghalf_trial_b == nullptr || kmat_b == nullptr))
    return (int)cudaErrorInvalidValue;
  using C = const double2*;
  cv_features_kernel<<<W, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      W, X, na, nb, M, alias, reinterpret_cast<C>(energy), reinterpret_cast<C>(xv), reinterpret_cast<C>(ovlp),
      reinterpret_cast<C>(hybrid_energy), reinterpret_cast<C>(ghalfa), reinterpret_cast<C>(ghalfb),
      reinterpret_cast<C>(ghalf_trial_a), reinterpret_cast<C>(ghalf_trial_b), reinterpret_cast<C>(kmat_a),
      reinterpret_cast<C>(kmat_b), weight, lead, feat, base);
  note_launch();
  return (int)cudaGetLastError();
}

}  // extern "C"
