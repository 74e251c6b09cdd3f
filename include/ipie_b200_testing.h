/*
 * ipie_b200 testing entry points -- not part of the product ABI.
 *
 * These expose the tcgen05 GEMM core alone, so that the tests can hold it
 * against a plain product before the fused kernels built on it are trusted.
 * They follow the conventions of ipie_b200.h (device pointers, a CUDA stream
 * as void*, 0 or a cudaError_t back) and have no counterpart in ipie.
 */
#ifndef IPIE_B200_TESTING_H
#define IPIE_B200_TESTING_H

#ifdef __cplusplus
extern "C" {
#endif

/* Validation entry of the tcgen05 TF32 GEMM core: c[row][a][col] =
 * sum_k A_a[row][k] B[col][k] for a < na (na = 1 or 2), A_a (M,K) and B (N,K)
 * row-major fp32 with K % 4 == 0; nsplit = 1 (TF32) or 3 (hi/lo split, the
 * *_lo operands used).  No counterpart in ipie. */
int ipie_b200_umma_gemm_test(const float* a0_hi, const float* a0_lo, const float* a1_hi, const float* a1_lo,
                             const float* b_hi, const float* b_lo, float* c, int M, int N, int K, int na, int nsplit,
                             unsigned int* status, void* stream);

/* Validation entry of the tcgen05 GEMM core on FP16 operands (kind::f16, FP32
 * accumulation): c[row][col] = sum_k A[row][k] B[col][k], A (M,K) and B (N,K)
 * row-major binary16 with K % 8 == 0; nsplit = 1 or 3 (hi/lo, the *_lo operands
 * used).  No counterpart in ipie. */
int ipie_b200_umma_gemm_f16_test(const void* a_hi, const void* a_lo, const void* b_hi, const void* b_lo, float* c,
                                 int M, int N, int K, int nsplit, unsigned int* status, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* IPIE_B200_TESTING_H */
