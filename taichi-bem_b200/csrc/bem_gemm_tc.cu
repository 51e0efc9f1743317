// Tensor-core (tcgen05, TF32) trailing update for the FP32 LU factor.
#include "bem_gemm.cuh"

int bem_gemm_tc_update(bem_ctx* ctx, float* C, const float* A, const float* B, int64_t m, int64_t n, int64_t k,
                       int64_t lda, bool cplx, cudaStream_t s) {
    (void)ctx; (void)C; (void)A; (void)B; (void)m; (void)n; (void)k; (void)lda; (void)cplx; (void)s;
    return 1;  // not handled: the SIMT kernel runs
}
