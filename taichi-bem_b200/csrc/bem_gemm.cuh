// Trailing update of the blocked LU: C -= A * B (row-major, shared lda),
// C: m x n, A: m x k, B: k x n.  FP32: tcgen05 (bem_gemm_tc.cu) or SIMT;
// FP64: DMMA.
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

// FP64 trailing update on the FP64 tensor cores (DMMA, mma.sync m8n8k4 f64):
// C -= A B for a 64 x 64 tile of C per CTA (complex: 64 x 64 complex entries,
// four real products per complex one), K staged in chunks of 8 through
// shared memory as separate real and imaginary planes, the next chunk read
// into registers while the current one is multiplied.  Eight warps, each a
// 32 x 16 block of C: 4 x 2 fragments of 8 x 8.  The fragment layouts of
// m8n8k4: A[row = lane / 4][k = lane % 4], B[k = lane % 4][col = lane / 4],
// C[row = lane / 4][col = 2 (lane % 4) + {0, 1}].
constexpr int DM_BM = 64, DM_BK = 8, DM_LDS = DM_BM + 4;

__device__ __forceinline__ void dmma_acc(double& d0, double& d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

template <bool CPLX>
__global__ void __launch_bounds__(256) dmma_update_kernel(double* __restrict__ Cm, const double* __restrict__ Am,
                                                           const double* __restrict__ Bm, int64_t m, int64_t n, int k,
                                                           int64_t lda) {
    constexpr int W = CPLX ? 2 : 1;
    constexpr int NP = CPLX ? 2 : 1;  // planes (re, im)
    __shared__ double sA[NP][DM_BK][DM_LDS];
    __shared__ double sB[NP][DM_BK][DM_LDS];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int64_t m0 = (int64_t)blockIdx.y * DM_BM, n0 = (int64_t)blockIdx.x * DM_BM;
    const int wr = warp & 1, wc = warp >> 1;
    double acc[4][2][NP][2];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b)
#pragma unroll
            for (int p = 0; p < NP; ++p) acc[a][b][p][0] = acc[a][b][p][1] = 0.0;
    // staging assignment: A row tid/4, k pair 2 (tid%4); B k row tid/32, column pair 2 (tid%32)
    const int ar_ = tid >> 2, ak_ = (tid & 3) * 2;
    const int bk_ = tid >> 5, bc_ = (tid & 31) * 2;
    double ra[2][NP], rb[2][NP];
    auto fetch = [&](int k0) {
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            const int64_t gr = m0 + ar_;
            const int gk = k0 + ak_ + e;
            const bool ok = gr < m && gk < k;
            const int64_t ia = W * (gr * lda + gk);
            ra[e][0] = ok ? Am[ia] : 0.0;
            if (CPLX) ra[e][NP - 1] = ok ? Am[ia + 1] : 0.0;
            const int gkb = k0 + bk_;
            const int64_t gc = n0 + bc_ + e;
            const bool okb = gkb < k && gc < n;
            const int64_t ib = W * ((int64_t)gkb * lda + gc);
            rb[e][0] = okb ? Bm[ib] : 0.0;
            if (CPLX) rb[e][NP - 1] = okb ? Bm[ib + 1] : 0.0;
        }
    };
    fetch(0);
    for (int k0 = 0; k0 < k; k0 += DM_BK) {
#pragma unroll
        for (int e = 0; e < 2; ++e)
#pragma unroll
            for (int p = 0; p < NP; ++p) {
                sA[p][ak_ + e][ar_] = ra[e][p];
                sB[p][bk_][bc_ + e] = rb[e][p];
            }
        __syncthreads();
        if (k0 + DM_BK < k) fetch(k0 + DM_BK);
#pragma unroll
        for (int k4 = 0; k4 < DM_BK; k4 += 4) {
            const int kr = k4 + (lane & 3);
            double fa[4][NP], fb[2][NP];
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int p = 0; p < NP; ++p) fa[a][p] = sA[p][kr][32 * wr + 8 * a + (lane >> 2)];
#pragma unroll
            for (int b = 0; b < 2; ++b)
#pragma unroll
                for (int p = 0; p < NP; ++p) fb[b][p] = sB[p][kr][16 * wc + 8 * b + (lane >> 2)];
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 2; ++b) {
                    dmma_acc(acc[a][b][0][0], acc[a][b][0][1], fa[a][0], fb[b][0]);
                    if (CPLX) {
                        dmma_acc(acc[a][b][0][0], acc[a][b][0][1], -fa[a][1], fb[b][1]);
                        dmma_acc(acc[a][b][1][0], acc[a][b][1][1], fa[a][0], fb[b][1]);
                        dmma_acc(acc[a][b][1][0], acc[a][b][1][1], fa[a][1], fb[b][0]);
                    }
                }
        }
        __syncthreads();
    }
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b) {
            const int64_t gr = m0 + 32 * wr + 8 * a + (lane >> 2);
            if (gr >= m) continue;
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int64_t gc = n0 + 16 * wc + 8 * b + 2 * (lane & 3) + e;
                if (gc >= n) continue;
                Cm[W * (gr * lda + gc)] -= acc[a][b][0][e];
                if (CPLX) Cm[W * (gr * lda + gc) + 1] -= acc[a][b][NP - 1][e];
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
    if constexpr (sizeof(T) == 8) {
        dim3 grid((unsigned)((n + bem_gemm_detail::DM_BM - 1) / bem_gemm_detail::DM_BM),
                  (unsigned)((m + bem_gemm_detail::DM_BM - 1) / bem_gemm_detail::DM_BM));
        if (grid.y > 65535) return bem_fail(ctx, BEM_ERR_INVALID, "dmma_update_kernel: m too large");
        bem_gemm_detail::dmma_update_kernel<CPLX><<<grid, 256, 0, s>>>((double*)Cm, (const double*)Am,
                                                                      (const double*)Bm, m, n, (int)k, lda);
        ctx->launches++;
        return bem_check_cuda(ctx, cudaGetLastError(), "dmma_update_kernel");
    }
    dim3 grid((unsigned)((n + bem_gemm_detail::BN - 1) / bem_gemm_detail::BN),
              (unsigned)((m + bem_gemm_detail::BM - 1) / bem_gemm_detail::BM));
    bem_gemm_detail::gemm_sub_kernel<T, CPLX><<<grid, 256, 0, s>>>(Cm, Am, Bm, m, n, (int)k, lda);
    ctx->launches++;
    return bem_check_cuda(ctx, cudaGetLastError(), "gemm_sub_kernel");
}
