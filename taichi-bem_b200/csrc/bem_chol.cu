// Blocked Cholesky factorisation N = L L^H of a Hermitian positive definite
// matrix (the column-equilibrated normal matrix of the transmission least
// squares), left in the tile-LU format of bem_lu_factor_tiled so that the
// persistent triangular solve (bem_lu_solve_tiled) and the refinement calls
// take it unchanged.
//
// Right-looking, panels of 1024 columns by default (BEM_TUNE_CHOL_NB), each
// factored in sub-blocks of 64 in FP64:
//   chol64_kernel     the 64 x 64 diagonal block in shared memory, and the
//                     inverse of its factor;
//   dmma_gemm_kernel  L21 = A21 L11^{-H} (a product with that inverse) and the
//                     update of the panel's remaining columns, on the FP64
//                     tensor cores (DMMA);
// then the trailing Hermitian rank-1024 update A22 -= L21 L21^H of the lower
// triangle, the step that carries the O(n^3) work:
//   BEM_PREC_FP64   DMMA products (dmma_gemm_kernel, lower tiles only);
//   BEM_PREC_MIXED  tcgen05 products of FP16 hi/lo splits of the panel (the
//                   normal-matrix kernel of bem_lstsq.cu in its update mode),
//                   summed in FP64 and subtracted from the FP64 Schur
//                   complement.  The panels and the Schur complement stay in
//                   FP64; only the products are split, so the factor's error
//                   is that of the ~22-bit products (about 4e-7 of the
//                   update, measured on the normal matrix), not an FP32
//                   accumulation over the n / 256 updates.
// The reference solves this system with torch.linalg.lstsq
// (BEM_manager.py:1049); the factor here preconditions the FP64 iteration of
// bem_lstsq_refine.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "bem_internal.cuh"

namespace {

constexpr int CH_IB = 64;   // diagonal sub-block
constexpr int CH_SP = 256;  // sub-panel width of the panel factorisation
constexpr int CH_NB_DEFAULT = 1024;  // panel width (columns per trailing update; measured 510 / 410 / 384 ms for 256 / 512 / 1024 on the 30722-unknown normal matrix)
constexpr int CH_LD = CH_IB + 1;

struct cd {
    double re, im;
};

template <bool C>
__device__ __forceinline__ cd ld_c(const double* A, int64_t idx) {
    return C ? cd{A[2 * idx], A[2 * idx + 1]} : cd{A[idx], 0.0};
}
template <bool C>
__device__ __forceinline__ void st_c(double* A, int64_t idx, cd v) {
    if (C) {
        A[2 * idx] = v.re;
        A[2 * idx + 1] = v.im;
    } else {
        A[idx] = v.re;
    }
}

// Cholesky of the nb x nb (nb <= 64) diagonal block at A (lower triangle
// read and written), and Linv = L^{-1} (64 x 64, identity beyond nb) into
// inv.  A non-positive or non-finite pivot sets *info to 1 + its global
// column (the first one wins) and is replaced by 1 so the kernel finishes.
template <bool C>
__global__ void __launch_bounds__(256) chol64_kernel(double* A, int64_t lda, int nb, double* inv, int32_t* info,
                                                     int col0) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cd* M = reinterpret_cast<cd*>(smem_raw);  // [64][CH_LD]
    cd* X = M + CH_IB * CH_LD;                // [64][64] inverse being built
    __shared__ double s_d;
    const int tid = threadIdx.x;
    for (int e = tid; e < CH_IB * CH_IB; e += blockDim.x) {
        const int r = e / CH_IB, c = e - r * CH_IB;
        cd v{r == c ? 1.0 : 0.0, 0.0};
        if (r < nb && c < nb && c <= r) v = ld_c<C>(A, (int64_t)r * lda + c);
        M[r * CH_LD + c] = v;
    }
    __syncthreads();
    for (int j = 0; j < nb; ++j) {
        if (tid == 0) {
            double d = M[j * CH_LD + j].re;
            if (!(d > 0.0) || !isfinite(d)) {
                atomicCAS(info, 0, col0 + j + 1);
                d = 1.0;
            }
            d = sqrt(d);
            M[j * CH_LD + j] = cd{d, 0.0};
            s_d = 1.0 / d;
        }
        __syncthreads();
        const double rd = s_d;
        for (int i = j + 1 + tid; i < nb; i += blockDim.x) {
            cd v = M[i * CH_LD + j];
            M[i * CH_LD + j] = cd{v.re * rd, v.im * rd};
        }
        __syncthreads();
        // rank-1 update of the trailing lower triangle: row i = j + 1 + tid % 64,
        // columns j + 1 + tid / 64, + 4, ... up to i
        {
            const int i = j + 1 + (tid & 63);
            if (i < nb) {
                const cd a = M[i * CH_LD + j];
                for (int c = j + 1 + (tid >> 6); c <= i; c += 4) {
                    const cd b = M[c * CH_LD + j];
                    // M[i][c] -= a conj(b)
                    cd v = M[i * CH_LD + c];
                    v.re -= a.re * b.re + a.im * b.im;
                    v.im -= a.im * b.re - a.re * b.im;
                    M[i * CH_LD + c] = v;
                }
            }
        }
        __syncthreads();
    }
    for (int e = tid; e < nb * nb; e += blockDim.x) {
        const int r = e / nb, c = e - r * nb;
        if (c <= r) st_c<C>(A, (int64_t)r * lda + c, M[r * CH_LD + c]);
    }
    // X = L^{-1} (lower), row by row: X[r][c] = (delta_rc - sum_{c<=q<r} L[r][q] X[q][c]) / L[r][r];
    // four threads per column split the sum over q and combine by shuffles
    {
        const int c = tid >> 2, part = tid & 3;
        for (int r = 0; r < CH_IB; ++r) {
            cd v{0.0, 0.0};
            if (r > c)
                for (int q = c + part; q < r; q += 4) {
                    const cd l = M[r * CH_LD + q], x = X[q * CH_IB + c];
                    v.re -= l.re * x.re - l.im * x.im;
                    v.im -= l.re * x.im + l.im * x.re;
                }
            v.re += __shfl_xor_sync(0xffffffffu, v.re, 1);
            v.im += __shfl_xor_sync(0xffffffffu, v.im, 1);
            v.re += __shfl_xor_sync(0xffffffffu, v.re, 2);
            v.im += __shfl_xor_sync(0xffffffffu, v.im, 2);
            if (part == 0) {
                if (r == c) v = cd{1.0, 0.0};
                if (r < c) v = cd{0.0, 0.0};
                const double d = M[r * CH_LD + r].re;  // real positive (identity padding beyond nb)
                X[r * CH_IB + c] = cd{v.re / d, v.im / d};
            }
            __syncthreads();
        }
    }
    for (int e = tid; e < CH_IB * CH_IB; e += blockDim.x) st_c<C>(inv, e, X[e]);
}

// General FP64 tensor-core product  C += alpha A op(B)  (m x n, K = k),
// op(B) = B (k x n, row-major, ldb) or, with CONJT, B^H for B stored n x k;
// LOWER skips 64 x 64 tiles of C entirely above the line c = r + diag.
// Same CTA shape, staging and fragment layout as the LU's DMMA update.
constexpr int DG_BM = 64, DG_BK = 8, DG_LDS = DG_BM + 4;

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// C (m x n, ldc) += alpha op(A) op(B) on the FP64 tensor cores (DMMA,
// m8n8k4), 64 x 64 tiles per CTA, 8-wide K stages.  op(A) = A (m x k) or
// A^H (A stored k x m, CONJA); op(B) = B (k x n) or B^H (B stored n x k,
// CONJT).  LOWER skips the tiles strictly above the diagonal shifted by
// `diag`.  blockIdx.z takes the K range [z kchunk, (z + 1) kchunk); with more
// than one range the tiles are added with FP64 atomics (split K for thin
// products).  tri & 1: op(A) is lower triangular, tri & 2: op(B) is upper
// triangular; the K range of a tile then ends at its diagonal.
template <bool CPLX, bool CONJA, bool CONJT, bool LOWER>
__global__ void __launch_bounds__(256) dmma_gemm_kernel(double* __restrict__ Cm, int64_t ldc,
                                                         const double* __restrict__ Am, int64_t lda,
                                                         const double* __restrict__ Bm, int64_t ldb, int64_t m,
                                                         int64_t n, int k, double alpha, int64_t diag, int kchunk,
                                                         int tri = 0) {
    constexpr int W = CPLX ? 2 : 1;
    constexpr int NP = CPLX ? 2 : 1;
    __shared__ double sA[NP][DG_BK][DG_LDS];
    __shared__ double sB[NP][DG_BK][DG_LDS];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int64_t m0 = (int64_t)blockIdx.y * DG_BM, n0 = (int64_t)blockIdx.x * DG_BM;
    if (LOWER && n0 > m0 + DG_BM - 1 + diag) return;
    const int wr = warp & 1, wc = warp >> 1;
    double acc[4][2][NP][2];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b)
#pragma unroll
            for (int p = 0; p < NP; ++p) acc[a][b][p][0] = acc[a][b][p][1] = 0.0;
    // staging: A (and B^H) row tid/4, k pair 2 (tid%4); B k row tid/32, column pair 2 (tid%32)
    const int ar_ = tid >> 2, ak_ = (tid & 3) * 2;
    const int bk_ = tid >> 5, bc_ = (tid & 31) * 2;
    double ra[2][NP], rb[2][NP];
    const int kbeg = (int)blockIdx.z * kchunk;
    int kend = min(k, kbeg + kchunk);
    if (tri & 1) kend = (int)min((int64_t)kend, m0 + DG_BM);
    if (tri & 2) kend = (int)min((int64_t)kend, n0 + DG_BM);
    auto fetch = [&](int k0) {
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            if (CONJA) {
                // A^H: k row tid/32, row pair 2 (tid%32), read along A's rows (coalesced)
                const int gka = k0 + bk_;
                const int64_t gr = m0 + bc_ + e;
                const bool ok = gr < m && gka < kend;
                const int64_t ia = W * ((int64_t)gka * lda + gr);
                ra[e][0] = ok ? Am[ia] : 0.0;
                if (CPLX) ra[e][NP - 1] = ok ? -Am[ia + 1] : 0.0;
            } else {
                const int64_t gr = m0 + ar_;
                const int gk = k0 + ak_ + e;
                const bool ok = gr < m && gk < kend;
                const int64_t ia = W * (gr * lda + gk);
                ra[e][0] = ok ? Am[ia] : 0.0;
                if (CPLX) ra[e][NP - 1] = ok ? Am[ia + 1] : 0.0;
            }
            const int gk = k0 + ak_ + e;
            if (CONJT) {
                const int64_t gc = n0 + ar_;
                const bool okb = gc < n && gk < kend;
                const int64_t ib = W * (gc * ldb + gk);
                rb[e][0] = okb ? Bm[ib] : 0.0;
                if (CPLX) rb[e][NP - 1] = okb ? -Bm[ib + 1] : 0.0;
            } else {
                const int gkb = k0 + bk_;
                const int64_t gc = n0 + bc_ + e;
                const bool okb = gkb < kend && gc < n;
                const int64_t ib = W * ((int64_t)gkb * ldb + gc);
                rb[e][0] = okb ? Bm[ib] : 0.0;
                if (CPLX) rb[e][NP - 1] = okb ? Bm[ib + 1] : 0.0;
            }
        }
    };
    fetch(kbeg);
    for (int k0 = kbeg; k0 < kend; k0 += DG_BK) {
#pragma unroll
        for (int e = 0; e < 2; ++e)
#pragma unroll
            for (int p = 0; p < NP; ++p) {
                if (CONJA)
                    sA[p][bk_][bc_ + e] = ra[e][p];
                else
                    sA[p][ak_ + e][ar_] = ra[e][p];
                if (CONJT)
                    sB[p][ak_ + e][ar_] = rb[e][p];
                else
                    sB[p][bk_][bc_ + e] = rb[e][p];
            }
        __syncthreads();
        if (k0 + DG_BK < kend) fetch(k0 + DG_BK);
#pragma unroll
        for (int k4 = 0; k4 < DG_BK; k4 += 4) {
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
                    dmma(acc[a][b][0][0], acc[a][b][0][1], fa[a][0], fb[b][0]);
                    if (CPLX) {
                        dmma(acc[a][b][0][0], acc[a][b][0][1], -fa[a][1], fb[b][1]);
                        dmma(acc[a][b][1][0], acc[a][b][1][1], fa[a][0], fb[b][1]);
                        dmma(acc[a][b][1][0], acc[a][b][1][1], fa[a][1], fb[b][0]);
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
                double* c = Cm + W * (gr * ldc + gc);
                if (gridDim.z > 1) {
                    atomicAdd(c, alpha * acc[a][b][0][e]);
                    if (CPLX) atomicAdd(c + 1, alpha * acc[a][b][NP - 1][e]);
                } else {
                    c[0] += alpha * acc[a][b][0][e];
                    if (CPLX) c[1] += alpha * acc[a][b][NP - 1][e];
                }
            }
        }
}

// Tile-LU form of L L^H: with D = diag(L) (real, positive),
//   L' = L D^{-1} (unit lower, strictly lower part stored),  U = D L^H,
// so L' U = L L^H.  The diagonal of L is read from dg (copied beforehand);
// each thread takes one strictly lower entry (i, j) and writes both (i, j)
// and (j, i); the diagonal becomes U[j][j] = D_j^2.
template <bool C>
__global__ void chol_to_lu_kernel(double* A, int64_t lda, int n, const double* dg) {
    const int j = blockIdx.y * 16 + (threadIdx.x >> 4);
    const int64_t i0 = (int64_t)blockIdx.x * 16 + (threadIdx.x & 15);
    if (j >= n || i0 >= n) return;
    const int i = (int)i0;
    if (i == j) {
        st_c<C>(A, (int64_t)j * lda + j, cd{dg[j] * dg[j], 0.0});
        return;
    }
    if (i < j) return;
    const cd l = ld_c<C>(A, (int64_t)i * lda + j);
    const double dj = dg[j];
    st_c<C>(A, (int64_t)i * lda + j, cd{l.re / dj, l.im / dj});
    st_c<C>(A, (int64_t)j * lda + i, cd{dj * l.re, -dj * l.im});
}

template <bool C>
__global__ void diag_copy_kernel(const double* A, int64_t lda, int n, double* dg) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < n) dg[j] = C ? A[2 * ((int64_t)j * lda + j)] : A[(int64_t)j * lda + j];
}

__global__ void iota_kernel(int32_t* piv, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) piv[i] = i;
}

// C += alpha op(A) op(B) (see dmma_gemm_kernel); products with fewer tiles
// than two waves of CTAs split K into ranges of at least 512.
template <bool C, bool CONJA, bool CONJT, bool LOWER>
int gemm64x(bem_ctx* ctx, double* Cm, int64_t ldc, const double* A, int64_t lda, const double* B, int64_t ldb,
            int64_t m, int64_t n, int k, double alpha, int64_t diag, cudaStream_t s, int tri = 0) {
    if (m <= 0 || n <= 0 || k <= 0) return BEM_OK;
    dim3 grid((unsigned)((n + DG_BM - 1) / DG_BM), (unsigned)((m + DG_BM - 1) / DG_BM));
    if (grid.y > 65535) return bem_fail(ctx, BEM_ERR_INVALID, "dmma_gemm_kernel: m too large");
    const int64_t tiles = (int64_t)grid.x * grid.y;
    int splits = 1;
    if (!LOWER && tiles < 2 * (int64_t)ctx->num_sms)
        splits = (int)std::max<int64_t>(1, std::min<int64_t>((2 * ctx->num_sms) / tiles, k / 512));
    const int kchunk = (int)(((int64_t)k + splits - 1) / splits + DG_BK - 1) / DG_BK * DG_BK;
    grid.z = (unsigned)(((int64_t)k + kchunk - 1) / kchunk);
    dmma_gemm_kernel<C, CONJA, CONJT, LOWER><<<grid, 256, 0, s>>>(Cm, ldc, A, lda, B, ldb, m, n, k, alpha, diag,
                                                                    kchunk, tri);
    ctx->launches++;
    return bem_check_cuda(ctx, cudaGetLastError(), "dmma_gemm_kernel");
}

template <bool C, bool CONJT, bool LOWER>
int gemm64(bem_ctx* ctx, double* Cm, int64_t ldc, const double* A, int64_t lda, const double* B, int64_t ldb,
           int64_t m, int64_t n, int k, double alpha, int64_t diag, cudaStream_t s) {
    return gemm64x<C, false, CONJT, LOWER>(ctx, Cm, ldc, A, lda, B, ldb, m, n, k, alpha, diag, s);
}

// The blocked Cholesky.  With X == nullptr the factor is left in tile-LU
// form (piv, dinv); otherwise L stays in the lower triangle and each diagonal
// tile's inverse L_jj^{-1} is written into X's diagonal tile (X, ldx: the
// start of bem_chol_inverse's triangular inverse).
template <bool C>
int chol_t(bem_ctx* ctx, double* A, int64_t n, int64_t lda, bool tensor_cores, int32_t* piv, double* dinv,
           int32_t* info, cudaStream_t s, double* X = nullptr, int64_t ldx = 0) {
    const int W = C ? 2 : 1;
    const int ni = (int)n;
    // workspace: the inverse of the current 64 x 64 factor, the L21 product, the diagonal
    const size_t inv_d = (size_t)W * CH_IB * CH_IB;
    const size_t tmp_d = (size_t)W * n * CH_IB;
    if (int rc = bem_ws_reserve(ctx, sizeof(double) * (inv_d + tmp_d + n))) return rc;
    double* inv = static_cast<double*>(ctx->ws);
    double* tmp = inv + inv_d;
    double* dg = tmp + tmp_d;
    if (int rc = bem_check_cuda(ctx, cudaMemsetAsync(info, 0, sizeof(int32_t), s), "chol info")) return rc;
    const size_t smem = sizeof(cd) * (CH_IB * CH_LD + CH_IB * CH_IB);
    if (int rc = bem_check_cuda(ctx, cudaFuncSetAttribute(chol64_kernel<C>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                          (int)smem),
                                "chol64 smem"))
        return rc;
    auto at = [&](int64_t r, int64_t c) { return A + W * (r * lda + c); };
    const int nbw = ctx->tune[BEM_TUNE_CHOL_NB] > 0 ? ctx->tune[BEM_TUNE_CHOL_NB] : CH_NB_DEFAULT;
    for (int64_t k0 = 0; k0 < n; k0 += nbw) {
        const int64_t kb = std::min<int64_t>(nbw, n - k0);
        // the panel in sub-panels of CH_SP columns: 64-wide steps update only
        // their sub-panel's remaining columns (K = 64); the sub-panel then
        // updates the rest of the panel in one product (K = CH_SP)
        for (int64_t s0 = k0; s0 < k0 + kb; s0 += CH_SP) {
        const int64_t sb = std::min<int64_t>(CH_SP, k0 + kb - s0);
        for (int64_t j0 = s0; j0 < s0 + sb; j0 += CH_IB) {
            const int jb = (int)std::min<int64_t>(CH_IB, s0 + sb - j0);
            chol64_kernel<C><<<1, 256, smem, s>>>(at(j0, j0), lda, jb, inv, info, (int)j0);
            ctx->launches++;
            if (int rc = bem_check_cuda(ctx, cudaGetLastError(), "chol64_kernel")) return rc;
            if (X)
                if (int rc = bem_check_cuda(ctx, cudaMemcpy2DAsync(X + W * (j0 * ldx + j0), sizeof(double) * W * ldx,
                                                                   inv, sizeof(double) * W * CH_IB,
                                                                   sizeof(double) * W * jb, jb,
                                                                   cudaMemcpyDeviceToDevice, s),
                                            "diagonal inverse copy"))
                    return rc;
            const int64_t r1 = j0 + jb, m1 = n - r1;
            if (m1 <= 0) continue;
            // L21 = A21 L11^{-H}: into tmp, then back into A21
            if (int rc = bem_check_cuda(ctx, cudaMemsetAsync(tmp, 0, sizeof(double) * W * m1 * CH_IB, s), "tmp"))
                return rc;
            if (int rc = gemm64<C, true, false>(ctx, tmp, CH_IB, at(r1, j0), lda, inv, CH_IB, m1, jb, jb, 1.0, 0, s))
                return rc;
            if (int rc = bem_check_cuda(ctx, cudaMemcpy2DAsync(at(r1, j0), sizeof(double) * W * lda, tmp,
                                                               sizeof(double) * W * CH_IB, sizeof(double) * W * jb, m1,
                                                               cudaMemcpyDeviceToDevice, s),
                                        "L21 copy"))
                return rc;
            // the sub-panel's remaining columns: A[r1:, r1:s0+sb] -= L21 L21[0:w]^H (lower part)
            const int64_t w = s0 + sb - r1;
            if (w > 0)
                if (int rc = gemm64<C, true, true>(ctx, at(r1, r1), lda, at(r1, j0), lda, at(r1, j0), lda, m1, w, jb,
                                                   -1.0, 0, s))
                    return rc;
        }
        // the rest of the panel: A[r3:, r3:k0+kb] -= L_sub L_sub[0:w3]^H (lower part, K = sb)
        const int64_t r3 = s0 + sb, w3 = k0 + kb - r3, m3 = n - r3;
        if (w3 > 0 && m3 > 0)
            if (int rc = gemm64<C, true, true>(ctx, at(r3, r3), lda, at(r3, s0), lda, at(r3, s0), lda, m3, w3,
                                               (int)sb, -1.0, 0, s))
                return rc;
        }
        // trailing Hermitian update of the lower triangle
        const int64_t r2 = k0 + kb, m2 = n - r2;
        if (m2 <= 0) continue;
        if (tensor_cores) {
            if (int rc = bem_herk_tc_update(ctx, C, at(r2, k0), lda, (int)m2, (int)kb, at(r2, r2), lda, s)) return rc;
        } else {
            if (int rc = gemm64<C, true, true>(ctx, at(r2, r2), lda, at(r2, k0), lda, at(r2, k0), lda, m2, m2, (int)kb,
                                               -1.0, 0, s))
                return rc;
        }
    }
    if (X) return BEM_OK;
    // the factor in tile-LU form, identity tile pivots, inverses of the diagonal tiles
    diag_copy_kernel<C><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(A, lda, ni, dg);
    const unsigned nb16 = (unsigned)((n + 15) / 16);
    chol_to_lu_kernel<C><<<dim3(nb16, nb16), 256, 0, s>>>(A, lda, ni, dg);
    iota_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(piv, ni);
    ctx->launches += 3;
    if (int rc = bem_check_cuda(ctx, cudaGetLastError(), "chol_to_lu")) return rc;
    return bem_tile_inverses(ctx, C ? BEM_C128 : BEM_F64, A, n, lda, dinv, s);
}

// X = L^{-1} for the lower triangle of L (n x n, lda) whose diagonal tiles'
// inverses are already in X's diagonal tiles (the rest of X zero), by the
// recursion on halves (rounded to 64 rows)
//   L = [L11 0; L21 L22],  L^{-1} = [X11 0; -X22 L21 X11  X22],
// the two products on the FP64 tensor cores; ws holds L21 X11.
template <bool C>
int tri_inv_rec(bem_ctx* ctx, const double* L, int64_t lda, double* X, int64_t ldx, int64_t lo, int64_t hi,
                double* ws, cudaStream_t s) {
    const int W = C ? 2 : 1;
    if (hi - lo <= CH_IB) return BEM_OK;
    const int64_t mid = lo + ((hi - lo) / 2 + CH_IB - 1) / CH_IB * CH_IB;
    if (int rc = tri_inv_rec<C>(ctx, L, lda, X, ldx, lo, mid, ws, s)) return rc;
    if (int rc = tri_inv_rec<C>(ctx, L, lda, X, ldx, mid, hi, ws, s)) return rc;
    const int64_t m1 = mid - lo, m2 = hi - mid;
    if (int rc = bem_check_cuda(ctx, cudaMemsetAsync(ws, 0, sizeof(double) * W * m2 * m1, s), "tri_inv ws")) return rc;
    // ws = L21 X11 (X11 lower triangular: the product's K range is all of it)
    if (int rc = gemm64x<C, false, false, false>(ctx, ws, m1, L + W * (mid * lda + lo), lda, X + W * (lo * ldx + lo),
                                                 ldx, m2, m1, (int)m1, 1.0, 0, s))
        return rc;
    // X21 = -X22 ws
    return gemm64x<C, false, false, false>(ctx, X + W * (mid * ldx + lo), ldx, X + W * (mid * ldx + mid), ldx, ws,
                                           m1, m2, m1, (int)m2, -1.0, 0, s);
}

}  // namespace

extern "C" int bem_gemm(bem_ctx* ctx, int dtype, int conj_a, int conj_b, int tri, int64_t m, int64_t n, int64_t k,
                        double alpha, const void* A, int64_t lda, const void* B, int64_t ldb, void* Cm, int64_t ldc,
                        void* stream) {
    if (!ctx) return BEM_ERR_INVALID;
    if (m < 0 || n < 0 || k < 0 || k > (1 << 30) || !Cm || ldc < n || (m > 0 && n > 0 && k > 0 && (!A || !B)))
        return bem_fail(ctx, BEM_ERR_INVALID, "gemm: bad arguments");
    if (lda < (conj_a ? m : k) || ldb < (conj_b ? k : n)) return bem_fail(ctx, BEM_ERR_INVALID, "gemm: bad leading dimension");
    if (dtype != BEM_C128 && dtype != BEM_F64) return bem_fail(ctx, BEM_ERR_INVALID, "gemm: dtype must be F64 or C128");
    cudaStream_t s = (cudaStream_t)stream;
    const double* a = (const double*)A;
    const double* b = (const double*)B;
    double* c = (double*)Cm;
    const int kk = (int)k;
    if (tri < 0 || tri > 3) return bem_fail(ctx, BEM_ERR_INVALID, "gemm: tri must be 0..3");
#define BEM_GEMM_CASE(CX, CA, CB) \
    return gemm64x<CX, CA, CB, false>(ctx, c, ldc, a, lda, b, ldb, m, n, kk, alpha, 0, s, tri)
    if (dtype == BEM_C128) {
        if (conj_a) {
            if (conj_b) BEM_GEMM_CASE(true, true, true);
            BEM_GEMM_CASE(true, true, false);
        }
        if (conj_b) BEM_GEMM_CASE(true, false, true);
        BEM_GEMM_CASE(true, false, false);
    }
    if (conj_a) {
        if (conj_b) BEM_GEMM_CASE(false, true, true);
        BEM_GEMM_CASE(false, true, false);
    }
    if (conj_b) BEM_GEMM_CASE(false, false, true);
    BEM_GEMM_CASE(false, false, false);
#undef BEM_GEMM_CASE
}

extern "C" int bem_chol_inverse(bem_ctx* ctx, int dtype, void* A, int64_t n, int64_t lda, void* X, int64_t ldx,
                                int32_t* info, void* stream) {
    if (!ctx) return BEM_ERR_INVALID;
    if (!A || !X || !info || n <= 0 || lda < n || ldx < n || n > (1 << 28))
        return bem_fail(ctx, BEM_ERR_INVALID, "chol_inverse: bad arguments");
    if (dtype != BEM_C128 && dtype != BEM_F64)
        return bem_fail(ctx, BEM_ERR_INVALID, "chol_inverse: A must be F64 or C128");
    cudaStream_t s = (cudaStream_t)stream;
    const bool C = dtype == BEM_C128;
    const int W = C ? 2 : 1;
    if (int rc = bem_check_cuda(ctx, cudaMemset2DAsync(X, sizeof(double) * W * ldx, 0, sizeof(double) * W * n, n, s),
                                "chol_inverse zero"))
        return rc;
    double* a = (double*)A;
    double* x = (double*)X;
    int rc = C ? chol_t<true>(ctx, a, n, lda, false, nullptr, nullptr, info, s, x, ldx)
               : chol_t<false>(ctx, a, n, lda, false, nullptr, nullptr, info, s, x, ldx);
    if (rc) return rc;
    // the recursion's scratch: L21 X11 of the top level, at most (n/2 + 64)^2
    const int64_t h = n / 2 + CH_IB;
    void* ws = nullptr;
    if (int e = bem_big_ws(ctx, sizeof(double) * W * h * h, &ws)) return e;
    return C ? tri_inv_rec<true>(ctx, a, lda, x, ldx, 0, n, (double*)ws, s)
             : tri_inv_rec<false>(ctx, a, lda, x, ldx, 0, n, (double*)ws, s);
}

extern "C" int bem_chol_factor(bem_ctx* ctx, int dtype, void* A, int64_t n, int64_t lda, int method, int32_t* piv,
                               void* dinv, int32_t* info, void* stream) {
    if (!ctx) return BEM_ERR_INVALID;
    if (!A || !piv || !dinv || !info || n <= 0 || lda < n || n > (1 << 28))
        return bem_fail(ctx, BEM_ERR_INVALID, "chol_factor: bad arguments");
    if (dtype != BEM_C128 && dtype != BEM_F64) return bem_fail(ctx, BEM_ERR_INVALID, "chol_factor: A must be F64 or C128");
    if (method != BEM_PREC_MIXED && method != BEM_PREC_FP64)
        return bem_fail(ctx, BEM_ERR_INVALID, "chol_factor: method must be BEM_PREC_MIXED or BEM_PREC_FP64");
    cudaStream_t s = (cudaStream_t)stream;
    const bool tc = method == BEM_PREC_MIXED;
    return dtype == BEM_C128 ? chol_t<true>(ctx, (double*)A, n, lda, tc, piv, (double*)dinv, info, s)
                             : chol_t<false>(ctx, (double*)A, n, lda, tc, piv, (double*)dinv, info, s);
}
