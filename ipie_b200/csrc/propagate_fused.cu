// Fused orbital propagation for one walker-spin per CTA:
//
//   phi <- expH1 . phi                       (one-body, optional)
//   T_0 = phi;  T_n = VHS T_{n-1} / n;  phi <- phi + sum_{n=1..nmax} T_n
//   phi <- expH1 . phi                       (one-body, optional)
//
// the arithmetic of ipie's propagate_one_body (propagation/operations.py:26-55)
// and apply_exponential (operations.py:58-82), in one launch.  The running
// term T lives in shared memory for the whole chain and serves as the right
// operand of every GEMM pass; the left operand (this walker's VHS, or the
// shared expH1) streams through a two-stage cp.async pipeline in 16-wide k
// chunks, so VHS leaves HBM once per walker and its 6 re-reads hit L2.  The
// accumulated phi is kept in the output array (L2 resident), as the
// recurrence phi += T_n needs it once per term.
//
// MMA: f64 tensor cores (mma.sync m8n8k4).  The complex product V T is the
// real GEMM [V as M x 2M interleaved] . [T embedded 2x2], the embedding done
// at fragment-load time from the complex T in shared memory.  16 warps: 4 row
// groups of FM m8 tiles x 4 column groups of FN n8 tiles.
#include "common.cuh"
#include "kernels.h"

namespace ipie_b200 {

namespace {

constexpr int kBK = 16;       // k chunk (doubles) of the streamed left operand
constexpr int kLDA = kBK + 4;  // smem row stride of an A chunk (conflict-free fragment reads)

// Rows of the running term kept in shared memory: every k chunk of either pass
// kind (K = M real or K = 2M complex-interleaved) reads rows < KROWS, and rows
// >= M are zero.  kTSlack extra entries absorb the column overrun of the last
// row (output columns >= 2N are computed and discarded).
__host__ __device__ inline int fused_krows(int M) { return ((M + kBK - 1) / kBK) * kBK + 1; }
constexpr int kTSlack = 32;

struct PassDesc {
  const double* a;  // left operand, row-major real view
  int lda;          // doubles per row
  int K;            // real k extent of this pass
  int cplx;         // 1: right operand is complex T embedded 2x2 (K = 2M); 0: real A times T's real view (K = M)
};

constexpr int kThreads = 512;  // 16 warps: 4 row groups x 4 column groups

template <int FM>
struct Geometry {
  static constexpr int MPAD = 4 * FM * 8;
};

// Issue the cp.async copies of k chunk `c` of pass `p` into stage buffer sA.
template <int FM>
__device__ __forceinline__ void load_chunk(double* sA, const PassDesc& pd, int c, int M) {
  constexpr int MPAD = Geometry<FM>::MPAD;
  const int k0 = c * kBK;
  // MPAD rows x 4 segments of 16 bytes (2 doubles) ... kBK = 16 doubles = 8 segments
  for (int e = threadIdx.x; e < MPAD * 8; e += blockDim.x) {
    const int r = e >> 3, seg = e & 7;
    const int k = k0 + seg * 2;
    double* dst = sA + r * kLDA + seg * 2;
    int bytes = 0;
    const double* src = pd.a;
    if (r < M && k < pd.K) {
      bytes = (pd.K - k >= 2) ? 16 : 8;
      src = pd.a + (size_t)r * pd.lda + k;
    }
    cp_async16(dst, src, bytes);
  }
}

}  // namespace

// sT: complex running term, rows padded to KROWS (zeros beyond M), row stride TS (complex)
template <int FM, int FN>
__global__ void __launch_bounds__(kThreads, 1)
    propagate_fused_kernel(const double2* __restrict__ vhs, const double* __restrict__ expH1, int lda_e,
                           const double2* __restrict__ phi_in, double2* __restrict__ phi_out, int M, int N, int nmax,
                           int pre_one_body, int post_one_body) {
  extern __shared__ double smem_d[];
  constexpr int MPAD = Geometry<FM>::MPAD;
  const int TS = N + 1;
  const int KROWS = fused_krows(M);
  double* const sA0 = smem_d;  // stage s at sA0 + s * MPAD * kLDA
  double2* sT = reinterpret_cast<double2*>(smem_d + 2 * MPAD * kLDA);

  const int w = blockIdx.x;
  const double2* vw = vhs + (size_t)w * M * M;
  const double2* pin = phi_in + (size_t)w * M * N;
  double2* pout = phi_out + (size_t)w * M * N;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  const int wr = warp >> 2, wc = warp & 3;  // 4 row groups x 4 column groups
  const int row0 = wr * FM * 8, col0 = wc * FN * 8;

  // load phi_in into sT, zero the padding rows/cols and the slack past the last row
  for (int e = threadIdx.x; e < KROWS * TS + kTSlack; e += blockDim.x) {
    const int r = e / TS, cidx = e % TS;
    sT[e] = (r < M && cidx < N) ? pin[(size_t)r * N + cidx] : make_double2(0.0, 0.0);
  }
  // pass list
  const int npass = nmax + (pre_one_body ? 1 : 0) + (post_one_body ? 1 : 0);
  auto pass_desc = [&](int p) {
    PassDesc pd;
    const bool is_pre = pre_one_body && p == 0;
    const bool is_post = post_one_body && p == npass - 1;
    if (is_pre || is_post) {
      pd.a = expH1;
      pd.lda = lda_e;
      pd.K = M;
      pd.cplx = 0;
    } else {
      pd.a = reinterpret_cast<const double*>(vw);
      pd.lda = 2 * M;
      pd.K = 2 * M;
      pd.cplx = 1;
    }
    return pd;
  };
  // flattened (pass, chunk) stream for the pipeline
  int total_chunks = 0;
  for (int p = 0; p < npass; ++p) total_chunks += (pass_desc(p).K + kBK - 1) / kBK;

  int cur_p = 0, cur_c = 0;
  PassDesc pd = pass_desc(0);
  int nch = (pd.K + kBK - 1) / kBK;
  // prefetch chunk 0
  load_chunk<FM>(sA0, pd, 0, M);
  cp_async_commit();
  int pf_p = 0, pf_c = 0;  // position of the last issued chunk
  auto advance = [&](int& p, int& c) {
    ++c;
    if (c >= (pass_desc(p).K + kBK - 1) / kBK) {
      c = 0;
      ++p;
    }
  };

  double acc[FM][FN][2];
#pragma unroll
  for (int i = 0; i < FM; ++i)
#pragma unroll
    for (int j = 0; j < FN; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

  int taylor_n = 0;  // index of the Taylor term the current pass computes (1..nmax), 0 for one-body
  auto term_of = [&](int p) { return (pre_one_body && p == 0) || (post_one_body && p == npass - 1) ? 0 : p + 1 - (pre_one_body ? 1 : 0); };
  taylor_n = term_of(0);

  __syncthreads();
  for (int q = 0; q < total_chunks; ++q) {
    // issue the next chunk into the other stage
    int np_ = pf_p, nc_ = pf_c;
    advance(np_, nc_);
    if (q + 1 < total_chunks) {
      load_chunk<FM>(sA0 + ((q + 1) & 1) * MPAD * kLDA, pass_desc(np_), nc_, M);
      pf_p = np_;
      pf_c = nc_;
    }
    cp_async_commit();
    cp_async_wait<1>();
    __syncthreads();
    const double* a_s = sA0 + (q & 1) * MPAD * kLDA;
    const int k0 = cur_c * kBK;
#pragma unroll 1
    for (int kk = 0; kk < kBK; kk += 4) {
      double af[FM], bf[FN];
#pragma unroll
      for (int i = 0; i < FM; ++i) af[i] = a_s[(row0 + 8 * i + g) * kLDA + kk + t];
      const int kr = k0 + kk + t;  // real k index
#pragma unroll
      for (int j = 0; j < FN; ++j) {
        const int nr = col0 + 8 * j + g;  // real column index (n, c)
        if (pd.cplx) {
          const double2 v = sT[(kr >> 1) * TS + (nr >> 1)];
          // B''[2k+c'][2n+c]: (c',c) = (0,0) re, (0,1) im, (1,0) -im, (1,1) re
          const int cp = kr & 1, cc = nr & 1;
          bf[j] = cp == cc ? v.x : (cp == 0 ? v.y : -v.y);
        } else {
          const double* sTr = reinterpret_cast<const double*>(sT);
          bf[j] = sTr[kr * 2 * TS + nr];
        }
      }
#pragma unroll
      for (int i = 0; i < FM; ++i)
#pragma unroll
        for (int j = 0; j < FN; ++j) dmma884(acc[i][j], af[i], bf[j]);
    }
    __syncthreads();  // stage q&1 free for reuse; all reads of sT for this chunk done
    // end of a pass: epilogue
    if (cur_c == nch - 1) {
      const bool last = (cur_p == npass - 1);
      const double sc = taylor_n > 0 ? 1.0 / taylor_n : 1.0;
#pragma unroll
      for (int i = 0; i < FM; ++i)
#pragma unroll
        for (int j = 0; j < FN; ++j) {
          const int r = row0 + 8 * i + g, cr = col0 + 8 * j + 2 * t;
          if (r < M && cr < 2 * N) {
            const int n = cr >> 1;
            const double2 v = make_double2(acc[i][j][0] * sc, acc[i][j][1] * sc);
            const size_t gi = (size_t)r * N + n;
            if (taylor_n == 0) {
              // one-body result: new phi (pre: start of the Taylor chain; post: final output)
              pout[gi] = v;
              if (!last) sT[r * TS + n] = v;
            } else {
              const double2 base = (taylor_n == 1) ? (pre_one_body ? pout[gi] : pin[gi]) : pout[gi];
              pout[gi] = cadd(base, v);
              sT[r * TS + n] = v;
            }
          }
          acc[i][j][0] = acc[i][j][1] = 0.0;
        }
      __syncthreads();
      // the post one-body multiplies the accumulated phi, not the last term
      if (!last && post_one_body && cur_p + 1 == npass - 1) {
        for (int e = threadIdx.x; e < M * N; e += blockDim.x) sT[(e / N) * TS + e % N] = pout[e];
        __syncthreads();
      }
      if (!last) {
        cur_p += 1;
        cur_c = 0;
        pd = pass_desc(cur_p);
        nch = (pd.K + kBK - 1) / kBK;
        taylor_n = term_of(cur_p);
      }
    } else {
      cur_c += 1;
    }
  }
  cp_async_wait<0>();
}

template <int FM, int FN>
static cudaError_t launch_fused_fm_fn(const double2* vhs, const double* expH1, int lda_e, const double2* phi_in,
                                      double2* phi_out, int W, int M, int N, int nmax, int pre, int post, cudaStream_t st) {
  constexpr int MPAD = Geometry<FM>::MPAD;
  size_t smem = sizeof(double) * 2 * MPAD * kLDA + sizeof(double2) * ((size_t)fused_krows(M) * (N + 1) + kTSlack);
  if (smem > 227 * 1024) return cudaErrorInvalidValue;
  auto k = propagate_fused_kernel<FM, FN>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  k<<<W, kThreads, smem, st>>>(vhs, expH1, lda_e, phi_in, phi_out, M, N, nmax, pre, post);
  note_launch();
  return cudaGetLastError();
}

template <int FM>
static cudaError_t launch_fused_fm(const double2* vhs, const double* expH1, int lda_e, const double2* phi_in,
                                   double2* phi_out, int W, int M, int N, int nmax, int pre, int post, cudaStream_t st) {
  const int fn = (2 * N + 31) / 32;  // n8 tiles per column group (4 groups cover 2N real columns)
  switch (fn) {
    case 1: return launch_fused_fm_fn<FM, 1>(vhs, expH1, lda_e, phi_in, phi_out, W, M, N, nmax, pre, post, st);
    case 2: return launch_fused_fm_fn<FM, 2>(vhs, expH1, lda_e, phi_in, phi_out, W, M, N, nmax, pre, post, st);
    default: return cudaErrorInvalidValue;
  }
}

// Returns cudaErrorInvalidValue for shapes it does not cover (M > 256, N > 32,
// shared memory over the limit); callers then use the per-term GEMM path.
// expH1: real (M x lda_e) row-major with lda_e even (16-byte aligned rows for
// the cp.async staging); may be null when pre = post = 0.
cudaError_t launch_propagate_fused(const double2* vhs, const double* expH1, int lda_e, const double2* phi_in,
                                   double2* phi_out, int W, int M, int N, int nmax, int pre, int post, cudaStream_t st) {
  if (M <= 0 || N <= 0 || N > 32 || nmax < 1 || phi_in == phi_out) return cudaErrorInvalidValue;
  if ((pre || post) && (expH1 == nullptr || (lda_e & 1) || lda_e < M)) return cudaErrorInvalidValue;
  const int fm = (M + 31) / 32;
  switch (fm) {
    case 1: return launch_fused_fm<1>(vhs, expH1, lda_e, phi_in, phi_out, W, M, N, nmax, pre, post, st);
    case 2: return launch_fused_fm<2>(vhs, expH1, lda_e, phi_in, phi_out, W, M, N, nmax, pre, post, st);
    case 3: return launch_fused_fm<3>(vhs, expH1, lda_e, phi_in, phi_out, W, M, N, nmax, pre, post, st);
    case 4: return launch_fused_fm<4>(vhs, expH1, lda_e, phi_in, phi_out, W, M, N, nmax, pre, post, st);
    case 5: return launch_fused_fm<5>(vhs, expH1, lda_e, phi_in, phi_out, W, M, N, nmax, pre, post, st);
    case 6: return launch_fused_fm<6>(vhs, expH1, lda_e, phi_in, phi_out, W, M, N, nmax, pre, post, st);
    case 7: return launch_fused_fm<7>(vhs, expH1, lda_e, phi_in, phi_out, W, M, N, nmax, pre, post, st);
    case 8: return launch_fused_fm<8>(vhs, expH1, lda_e, phi_in, phi_out, W, M, N, nmax, pre, post, st);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace ipie_b200
