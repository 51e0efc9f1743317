// Trailing update of the blocked LU: C -= A * B (row-major, shared lda),
// C: m x n, A: m x k, B: k x n, k <= 64.
#pragma once

#include <cuda_runtime.h>

#include "bem_internal.cuh"

// FP32 real/complex updates go to the tcgen05 TF32 path when it is enabled
// (bem_gemm_tc.cu); it returns BEM_OK when it handled the call, 1 when the
// shape is not supported and the SIMT kernel below should run.
int bem_gemm_tc_update(bem_ctx* ctx, float* C, const float* A, const float* B, int64_t m, int64_t n, int64_t k,
                       int64_t lda, bool cplx, cudaStream_t s);

namespace bem_gemm_detail {

constexpr int BM = 64, BN = 64, BK = 16;

template <typename T, bool CPLX>
__global__ void __launch_bounds__(256) gemm_sub_kernel(T* __restrict__ Cm, const T* __restrict__ Am,
                                                        const T* __restrict__ Bm, int64_t m, int64_t n, int k,
                                                        int64_t lda) {
    constexpr int W = CPLX ? 2 : 1;
    __shared__ T As[BK][BM * W];
    __shared__ T Bs[BK][BN * W];
    const int tid = threadIdx.x;
    const int tx = tid & 15, ty = tid >> 4;
    const int64_t m0 = (int64_t)blockIdx.y * BM, n0 = (int64_t)blockIdx.x * BN;
    T acc_re[4][4], acc_im[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc_re[i][j] = acc_im[i][j] = T(0);

    for (int k0 = 0; k0 < k; k0 += BK) {
        // A tile: BM rows x BK cols -> As[kk][row]
        for (int e = tid; e < BM * BK; e += 256) {
            int r = e / BK, kk = e - r * BK;
            int64_t gr = m0 + r;
            int gk = k0 + kk;
            T vr = T(0), vi = T(0);
            if (gr < m && gk < k) {
                vr = Am[W * (gr * lda + gk)];
                if (CPLX) vi = Am[W * (gr * lda + gk) + 1];
            }
            As[kk][W * r] = vr;
            if (CPLX) As[kk][W * r + 1] = vi;
        }
        // B tile: BK rows x BN cols -> Bs[kk][col]
        for (int e = tid; e < BK * BN; e += 256) {
            int kk = e / BN, c = e - kk * BN;
            int gk = k0 + kk;
            int64_t gc = n0 + c;
            T vr = T(0), vi = T(0);
            if (gk < k && gc < n) {
                vr = Bm[W * ((int64_t)gk * lda + gc)];
                if (CPLX) vi = Bm[W * ((int64_t)gk * lda + gc) + 1];
            }
            Bs[kk][W * c] = vr;
            if (CPLX) Bs[kk][W * c + 1] = vi;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < BK; ++kk) {
            T ar[4], ai[4], br[4], bi[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                ar[i] = As[kk][W * (ty * 4 + i)];
                ai[i] = CPLX ? As[kk][W * (ty * 4 + i) + 1] : T(0);
                br[i] = Bs[kk][W * (tx * 4 + i)];
                bi[i] = CPLX ? Bs[kk][W * (tx * 4 + i) + 1] : T(0);
            }
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    acc_re[i][j] += ar[i] * br[j];
                    if (CPLX) {
                        acc_re[i][j] -= ai[i] * bi[j];
                        acc_im[i][j] += ar[i] * bi[j] + ai[i] * br[j];
                    }
                }
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        int64_t gr = m0 + ty * 4 + i;
        if (gr >= m) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            int64_t gc = n0 + tx * 4 + j;
            if (gc >= n) continue;
            Cm[W * (gr * lda + gc)] -= acc_re[i][j];
            if (CPLX) Cm[W * (gr * lda + gc) + 1] -= acc_im[i][j];
        }
    }
}

}  // namespace bem_gemm_detail

template <typename T, bool CPLX>
int bem_gemm_update(bem_ctx* ctx, T* Cm, const T* Am, const T* Bm, int64_t m, int64_t n, int64_t k, int64_t lda,
                    cudaStream_t s) {
    if (m <= 0 || n <= 0 || k <= 0) return BEM_OK;
    if constexpr (sizeof(T) == 4) {
        int rc = bem_gemm_tc_update(ctx, (float*)Cm, (const float*)Am, (const float*)Bm, m, n, k, lda, CPLX, s);
        if (rc <= 0) return rc;
    }
    dim3 grid((unsigned)((n + bem_gemm_detail::BN - 1) / bem_gemm_detail::BN),
              (unsigned)((m + bem_gemm_detail::BM - 1) / bem_gemm_detail::BM));
    bem_gemm_detail::gemm_sub_kernel<T, CPLX><<<grid, 256, 0, s>>>(Cm, Am, Bm, m, n, (int)k, lda);
    ctx->launches++;
    return bem_check_cuda(ctx, cudaGetLastError(), "gemm_sub_kernel");
}
