// Tile-pivoted LU and barrier-free triangular solves (the low-precision factor
// of the mixed path).
//
// Factorisation, per diagonal block k (LU_T = 64 columns):
//   diag   : one CTA factors the 64x64 diagonal block with partial pivoting
//            restricted to the block's rows, and forms the explicit inverses
//            Linv_k (unit lower) and Uinv_k (upper), stored in `dinv`;
//   laswp  : the block's row swaps applied to the other columns;
//   U12 = Linv_k A12 and L21 = A21 Uinv_k: one CTA per 64-wide tile, products
//            out of shared memory (no sequential substitution);
//   update : A22 -= L21 U12 (the trailing GEMM of bem_gemm.cuh).
// No grid-wide synchronisation is needed.  Pivoting within the diagonal tile
// is weaker than full partial pivoting; the FP64 iterative refinement that
// consumes this factor corrects the difference (and reports non-convergence).
//
// Solve: a persistent kernel in which CTA b owns block rows b, b+P, b+2P...;
// block row k accumulates L_kj x_j for every finished j < k (ready flags,
// acquire/release, bounded waits), applies Linv_k, publishes x_k and its flag.
// Each CTA handles its block rows in increasing order and all CTAs are
// co-resident (cooperative launch), so every wait ends.
#include <cuda_runtime.h>

#include <algorithm>

#include "bem_gemm.cuh"
#include "bem_internal.cuh"

namespace {

constexpr int LU_T = 64;
constexpr unsigned FLAG_SPIN_CAP = 1u << 22;

template <typename T>
struct CE {
    T re, im;
};

template <typename T, bool C>
__device__ __forceinline__ CE<T> ldE(const T* A, int64_t i) {
    CE<T> e;
    e.re = C ? A[2 * i] : A[i];
    e.im = C ? A[2 * i + 1] : T(0);
    return e;
}
template <typename T, bool C>
__device__ __forceinline__ void stE(T* A, int64_t i, CE<T> e) {
    if (C) {
        A[2 * i] = e.re;
        A[2 * i + 1] = e.im;
    } else {
        A[i] = e.re;
    }
}
template <typename T>
__device__ __forceinline__ CE<T> cmul(CE<T> a, CE<T> b) {
    return CE<T>{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
template <typename T>
__device__ __forceinline__ CE<T> cinv(CE<T> a) {
    T d = a.re * a.re + a.im * a.im;
    return d > T(0) ? CE<T>{a.re / d, -a.im / d} : CE<T>{T(0), T(0)};
}

// --------------------------------------------------------------------------
// diagonal tile: GEPP inside the tile + explicit inverses
// --------------------------------------------------------------------------
template <typename T, bool C>
__global__ void __launch_bounds__(256) tile_diag_kernel(T* A, int64_t lda, int n, int k0, int32_t* piv,
                                                        CE<T>* dinv, int32_t* info) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    CE<T>* S = reinterpret_cast<CE<T>*>(smem_raw);  // [LU_T][LU_T]
    CE<T>* Li = S + LU_T * LU_T;
    CE<T>* Ui = Li + LU_T * LU_T;
    __shared__ int s_p;
    __shared__ int s_zero_pivot;  // first zero pivot of this tile (1-based), 0 = none
    const int m = min(LU_T, n - k0);
    if (threadIdx.x == 0) s_zero_pivot = 0;
    for (int e = threadIdx.x; e < LU_T * LU_T; e += blockDim.x) {
        int r = e / LU_T, c = e - r * LU_T;
        S[e] = (r < m && c < m) ? ldE<T, C>(A, (int64_t)(k0 + r) * lda + k0 + c) : CE<T>{T(0), T(0)};
    }
    __syncthreads();
    for (int j = 0; j < m; ++j) {
        // pivot search in column j (warp 0), then swap rows j and p
        if (threadIdx.x < 32) {
            double best = -1.0;
            int bi = j;
            for (int r = j + threadIdx.x; r < m; r += 32) {
                CE<T> v = S[r * LU_T + j];
                double a = fabs((double)v.re) + fabs((double)v.im);
                if (a > best || (a == best && r < bi)) {
                    best = a;
                    bi = r;
                }
            }
            for (int o = 16; o > 0; o >>= 1) {
                double ob = __shfl_xor_sync(0xffffffffu, best, o);
                int oi = __shfl_xor_sync(0xffffffffu, bi, o);
                if (ob > best || (ob == best && oi < bi)) {
                    best = ob;
                    bi = oi;
                }
            }
            if (threadIdx.x == 0) {
                s_p = bi;
                piv[k0 + j] = k0 + bi;
                if (!(best > 0.0) && s_zero_pivot == 0) s_zero_pivot = k0 + j + 1;
            }
            const int p = __shfl_sync(0xffffffffu, bi, 0);
            if (p != j)
                for (int c = threadIdx.x; c < LU_T; c += 32) {
                    CE<T> t = S[j * LU_T + c];
                    S[j * LU_T + c] = S[p * LU_T + c];
                    S[p * LU_T + c] = t;
                }
        }
        __syncthreads();
        // multipliers and rank-1 update in one pass: element (r, c), c > j,
        // uses l_r = S[r][j] / S[j][j]; column j itself is scaled by the
        // threads of c == j after everyone has read it (second sync)
        const CE<T> inv = cinv(S[j * LU_T + j]);
        // thread t owns columns c = j + (t % 64) ... of rows j+1+(t/64), +4, ...:
        // fixed (row, column) ownership keeps the buffered values in registers
        const int cc = j + (threadIdx.x & 63);
        const int r0 = j + 1 + (threadIdx.x >> 6);
        constexpr int RPT = LU_T / 4;  // rows per thread
        CE<T> upd[RPT];
#pragma unroll
        for (int it = 0; it < RPT; ++it) {
            const int r = r0 + 4 * it;
            upd[it] = CE<T>{T(0), T(0)};
            if (r < m && cc < m) {
                const CE<T> l = cmul(S[r * LU_T + j], inv);
                if (cc == j) {
                    upd[it] = l;
                } else {
                    const CE<T> lu = cmul(l, S[j * LU_T + cc]), v = S[r * LU_T + cc];
                    upd[it] = CE<T>{v.re - lu.re, v.im - lu.im};
                }
            }
        }
        __syncthreads();
#pragma unroll
        for (int it = 0; it < RPT; ++it) {
            const int r = r0 + 4 * it;
            if (r < m && cc < m) S[r * LU_T + cc] = upd[it];
        }
        __syncthreads();
    }
    // explicit inverses, rows in sequence, all columns of a row in parallel:
    // threads 0..127 build Linv (two threads per column, partial sums combined
    // with a shuffle), threads 128..255 build Uinv the same way from the
    // bottom row up.  Named barriers keep the two halves independent.
    {
        const int half = threadIdx.x >> 7;  // 0: Linv, 1: Uinv
        const int t = threadIdx.x & 127;
        const int c = t >> 1, part = t & 1;
        CE<T>* X = half == 0 ? Li : Ui;
        for (int e = t; e < LU_T * LU_T; e += 128) X[e] = CE<T>{T(0), T(0)};
        if (half == 0)
            asm volatile("bar.sync 1, 128;" ::: "memory");
        else
            asm volatile("bar.sync 2, 128;" ::: "memory");
        for (int step = 0; step < LU_T; ++step) {
            const int r = half == 0 ? step : LU_T - 1 - step;
            CE<T> sum = CE<T>{T(0), T(0)};
            if (r < m) {
                if (half == 0) {
                    // Linv[r][c] = delta_rc - sum_{c <= q < r} L[r][q] Linv[q][c]   (c <= r)
                    if (c < r)
                        for (int q = c + part; q < r; q += 2) {
                            CE<T> tt = cmul(S[r * LU_T + q], X[q * LU_T + c]);
                            sum.re += tt.re;
                            sum.im += tt.im;
                        }
                } else {
                    // Uinv[r][c] = (delta_rc - sum_{r < q <= c} U[r][q] Uinv[q][c]) / U[r][r]   (r <= c)
                    if (c > r)
                        for (int q = r + 1 + part; q <= c && q < m; q += 2) {
                            CE<T> tt = cmul(S[r * LU_T + q], X[q * LU_T + c]);
                            sum.re += tt.re;
                            sum.im += tt.im;
                        }
                }
            }
            sum.re += __shfl_xor_sync(0xffffffffu, sum.re, 1);
            sum.im += __shfl_xor_sync(0xffffffffu, sum.im, 1);
            if (part == 0) {
                CE<T> val;
                if (r >= m) {
                    val = CE<T>{r == c ? T(1) : T(0), T(0)};  // identity padding of a short last tile
                } else if (half == 0) {
                    val = c < r ? CE<T>{-sum.re, -sum.im} : CE<T>{r == c ? T(1) : T(0), T(0)};
                } else if (c < r) {
                    val = CE<T>{T(0), T(0)};
                } else if (c >= m) {
                    val = CE<T>{T(0), T(0)};
                } else {
                    CE<T> d = CE<T>{(r == c ? T(1) : T(0)) - sum.re, -sum.im};
                    val = cmul(d, cinv(S[r * LU_T + r]));
                }
                X[r * LU_T + c] = val;
            }
            if (half == 0)
                asm volatile("bar.sync 1, 128;" ::: "memory");
            else
                asm volatile("bar.sync 2, 128;" ::: "memory");
        }
    }
    __syncthreads();
    if (threadIdx.x == 0 && s_zero_pivot != 0 && *info == 0) *info = s_zero_pivot;
    CE<T>* D = dinv + (size_t)(k0 / LU_T) * 2 * LU_T * LU_T;
    for (int e = threadIdx.x; e < LU_T * LU_T; e += blockDim.x) {
        D[e] = Li[e];
        D[LU_T * LU_T + e] = Ui[e];
        int r = e / LU_T, c = e - r * LU_T;
        if (r < m && c < m) stE<T, C>(A, (int64_t)(k0 + r) * lda + k0 + c, S[e]);
    }
}

template <typename T, bool C>
__global__ void tile_laswp_kernel(T* A, int64_t lda, int n, int k0, int m, const int32_t* piv) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n || (c >= k0 && c < k0 + m)) return;
    for (int j = 0; j < m; ++j) {
        int r1 = k0 + j, r2 = piv[k0 + j];
        if (r1 == r2) continue;
        CE<T> a = ldE<T, C>(A, (int64_t)r1 * lda + c);
        CE<T> b = ldE<T, C>(A, (int64_t)r2 * lda + c);
        stE<T, C>(A, (int64_t)r1 * lda + c, b);
        stE<T, C>(A, (int64_t)r2 * lda + c, a);
    }
}

// mode 0: U12 tile (rows k0.., 64 columns) <- Linv * tile
// mode 1: L21 tile (64 rows, columns k0..) <- tile * Uinv
template <typename T, bool C>
__global__ void __launch_bounds__(256) tile_apply_kernel(T* A, int64_t lda, int n, int k0, int m, const CE<T>* dinv,
                                                         int mode) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    CE<T>* M = reinterpret_cast<CE<T>*>(smem_raw);  // [LU_T][LU_T] inverse
    CE<T>* X = M + LU_T * LU_T;                     // [LU_T][LU_T] tile
    const CE<T>* D = dinv + (size_t)(k0 / LU_T) * 2 * LU_T * LU_T + (mode == 0 ? 0 : LU_T * LU_T);
    const int base = k0 + m + blockIdx.x * LU_T;  // first column (mode 0) / row (mode 1) of the tile
    const int cnt = min(LU_T, n - base);
    for (int e = threadIdx.x; e < LU_T * LU_T; e += blockDim.x) {
        M[e] = D[e];
        int r = e / LU_T, c = e - r * LU_T;
        CE<T> v = CE<T>{T(0), T(0)};
        if (mode == 0) {
            if (r < m && c < cnt) v = ldE<T, C>(A, (int64_t)(k0 + r) * lda + base + c);
        } else {
            if (r < cnt && c < m) v = ldE<T, C>(A, (int64_t)(base + r) * lda + k0 + c);
        }
        X[e] = v;
    }
    __syncthreads();
    // each thread: 16 outputs (4 rows x 4 columns)
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    CE<T> acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = CE<T>{T(0), T(0)};
    for (int q = 0; q < m; ++q) {
        CE<T> a[4], b[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            a[i] = mode == 0 ? M[(ty * 4 + i) * LU_T + q] : X[(ty * 4 + i) * LU_T + q];
            b[i] = mode == 0 ? X[q * LU_T + tx * 4 + i] : M[q * LU_T + tx * 4 + i];
        }
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                acc[i][j].re += a[i].re * b[j].re - (C ? a[i].im * b[j].im : T(0));
                if (C) acc[i][j].im += a[i].re * b[j].im + a[i].im * b[j].re;
            }
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            int r = ty * 4 + i, c = tx * 4 + j;
            if (mode == 0) {
                if (r < m && c < cnt) stE<T, C>(A, (int64_t)(k0 + r) * lda + base + c, acc[i][j]);
            } else {
                if (r < cnt && c < m) stE<T, C>(A, (int64_t)(base + r) * lda + k0 + c, acc[i][j]);
            }
        }
}

// --------------------------------------------------------------------------
// barrier-free triangular solves
// --------------------------------------------------------------------------
__device__ __forceinline__ int ld_acquire_i(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_i(int* p, int v) {
    asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Waits (bounded) until flags[j] == epoch.  Returns false on timeout / failure.
__device__ __forceinline__ bool wait_flag(const int* flags, int j, int epoch, int32_t* err) {
    __shared__ int s_ok;
    if (threadIdx.x == 0) {
        int ok = 1;
        unsigned it = 0;
        while (ld_acquire_i(flags + j) != epoch) {
            if (++it > FLAG_SPIN_CAP) {
                atomicExch(err, BEM_ERR_TIMEOUT);
                ok = 0;
                break;
            }
            if ((it & 63u) == 0u && *(volatile int32_t*)err != 0) {
                ok = 0;
                break;
            }
            if (it > 256u) __nanosleep(64);
        }
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// x (FP64, real or complex interleaved, one right-hand side) overwritten by
// U^{-1} L^{-1} x; the input must already be permuted (x = P b).
template <typename T, bool C>
__global__ void __launch_bounds__(256) tile_solve_kernel(const T* LU, int64_t lda, int n, const CE<T>* dinv,
                                                         double* x, int* flags, int epoch, int32_t* err) {
    __shared__ double s_acc[LU_T][2];
    __shared__ double s_part[8][LU_T][2];
    __shared__ double s_y[LU_T][2];
    const int nbk = (n + LU_T - 1) / LU_T;
    const int P = gridDim.x;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int W = C ? 2 : 1;
    for (int pass = 0; pass < 2; ++pass) {
        const bool fwd = pass == 0;
        for (int t = blockIdx.x; t < nbk; t += P) {
            const int k = fwd ? t : nbk - 1 - t;
            const int r0 = k * LU_T, m = min(LU_T, n - r0);
            // partial sums over finished blocks: warp w handles dependency blocks j = w, w+8, ...
            for (int i = threadIdx.x; i < 8 * LU_T * 2; i += blockDim.x) (&s_part[0][0][0])[i] = 0.0;
            __syncthreads();
            const int ndep = fwd ? k : nbk - 1 - k;
            for (int d = 0; d < ndep; ++d) {
                const int j = fwd ? d : nbk - 1 - d;
                if (!wait_flag(flags, pass * nbk + j, epoch, err)) return;
                const int c0 = j * LU_T, mj = min(LU_T, n - c0);
                // x_j segment
                double xr0 = 0, xi0 = 0, xr1 = 0, xi1 = 0;
                if (lane < mj) {
                    xr0 = __ldcg(&x[W * (c0 + lane)]);
                    xi0 = C ? __ldcg(&x[W * (c0 + lane) + 1]) : 0.0;
                }
                if (lane + 32 < mj) {
                    xr1 = __ldcg(&x[W * (c0 + lane + 32)]);
                    xi1 = C ? __ldcg(&x[W * (c0 + lane + 32) + 1]) : 0.0;
                }
                for (int r = wid; r < m; r += 8) {
                    const T* row = LU + (C ? 2 : 1) * ((int64_t)(r0 + r) * lda + c0);
                    double sr = 0.0, si = 0.0;
                    if (lane < mj) {
                        CE<T> l = ldE<T, C>(row, lane);
                        sr += (double)l.re * xr0 - (double)l.im * xi0;
                        si += (double)l.re * xi0 + (double)l.im * xr0;
                    }
                    if (lane + 32 < mj) {
                        CE<T> l = ldE<T, C>(row, lane + 32);
                        sr += (double)l.re * xr1 - (double)l.im * xi1;
                        si += (double)l.re * xi1 + (double)l.im * xr1;
                    }
                    for (int o = 16; o > 0; o >>= 1) {
                        sr += __shfl_xor_sync(0xffffffffu, sr, o);
                        si += __shfl_xor_sync(0xffffffffu, si, o);
                    }
                    if (lane == 0) {
                        s_part[wid][r][0] += sr;
                        s_part[wid][r][1] += si;
                    }
                }
                __syncthreads();
            }
            // rhs of block k minus the dependencies
            for (int r = threadIdx.x; r < LU_T; r += blockDim.x) {
                double ar = 0.0, ai = 0.0;
                if (r < m) {
                    ar = __ldcg(&x[W * (r0 + r)]);
                    ai = C ? __ldcg(&x[W * (r0 + r) + 1]) : 0.0;
                    for (int w = 0; w < 8; ++w) {
                        ar -= s_part[w][r][0];
                        ai -= s_part[w][r][1];
                    }
                }
                s_acc[r][0] = ar;
                s_acc[r][1] = ai;
            }
            __syncthreads();
            // y = inverse(diagonal block) * acc
            const CE<T>* Dk = dinv + (size_t)k * 2 * LU_T * LU_T + (fwd ? 0 : LU_T * LU_T);
            for (int r = wid; r < m; r += 8) {
                double sr = 0.0, si = 0.0;
                for (int q = lane; q < m; q += 32) {
                    CE<T> d = Dk[r * LU_T + q];
                    sr += (double)d.re * s_acc[q][0] - (double)d.im * s_acc[q][1];
                    si += (double)d.re * s_acc[q][1] + (double)d.im * s_acc[q][0];
                }
                for (int o = 16; o > 0; o >>= 1) {
                    sr += __shfl_xor_sync(0xffffffffu, sr, o);
                    si += __shfl_xor_sync(0xffffffffu, si, o);
                }
                if (lane == 0) {
                    s_y[r][0] = sr;
                    s_y[r][1] = si;
                }
            }
            __syncthreads();
            for (int r = threadIdx.x; r < m; r += blockDim.x) {
                x[W * (r0 + r)] = s_y[r][0];
                if (C) x[W * (r0 + r) + 1] = s_y[r][1];
            }
            __threadfence();
            __syncthreads();
            if (threadIdx.x == 0) st_release_i(flags + pass * nbk + k, epoch);
        }
        // the backward pass of block k needs x_k from the forward pass: every
        // block row's forward flag is checked before its value is read below
        if (fwd) {
            for (int t = blockIdx.x; t < nbk; t += P) {
                const int k = nbk - 1 - t;
                if (!wait_flag(flags, k, epoch, err)) return;
            }
        }
    }
}

__global__ void permute_kernel(const double* b, const int32_t* perm, double* x, int n, int W) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int s = perm[i];
    for (int w = 0; w < W; ++w) x[W * i + w] = b[W * s + w];
}

__global__ void tile_piv_to_perm_kernel(const int32_t* piv, int32_t* perm, int n) {
    extern __shared__ int32_t sp[];
    for (int i = threadIdx.x; i < n; i += blockDim.x) sp[i] = i;
    __syncthreads();
    if (threadIdx.x == 0)
        for (int i = 0; i < n; ++i) {
            int p = piv[i];
            if (p != i && p >= 0 && p < n) {
                int t = sp[i];
                sp[i] = sp[p];
                sp[p] = t;
            }
        }
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) perm[i] = sp[i];
}

template <typename T, bool C>
int factor_t(bem_ctx* ctx, T* A, int64_t n, int64_t lda, int32_t* piv, CE<T>* dinv, int32_t* info,
             cudaStream_t s) {
    cudaMemsetAsync(info, 0, sizeof(int32_t), s);
    const size_t dsmem = sizeof(CE<T>) * 3 * LU_T * LU_T;
    const size_t asmem = sizeof(CE<T>) * 2 * LU_T * LU_T;
    cudaFuncSetAttribute(tile_diag_kernel<T, C>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dsmem);
    cudaFuncSetAttribute(tile_apply_kernel<T, C>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)asmem);
    const int ni = (int)n;
    const int W = C ? 2 : 1;
    for (int64_t k0 = 0; k0 < n; k0 += LU_T) {
        const int m = (int)std::min<int64_t>(LU_T, n - k0);
        const int k0i = (int)k0;
        tile_diag_kernel<T, C><<<1, 256, dsmem, s>>>(A, lda, ni, k0i, piv, dinv, info);
        tile_laswp_kernel<T, C><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(A, lda, ni, k0i, m, piv);
        ctx->launches += 2;
        const int64_t rest = n - k0 - m;
        if (rest > 0) {
            const unsigned tiles = (unsigned)((rest + LU_T - 1) / LU_T);
            tile_apply_kernel<T, C><<<tiles, 256, asmem, s>>>(A, lda, ni, k0i, m, dinv, 0);
            tile_apply_kernel<T, C><<<tiles, 256, asmem, s>>>(A, lda, ni, k0i, m, dinv, 1);
            ctx->launches += 2;
            T* A22 = A + W * ((k0 + m) * lda + k0 + m);
            const T* L21 = A + W * ((k0 + m) * lda + k0);
            const T* U12 = A + W * (k0 * lda + k0 + m);
            if (int rc = bem_gemm_update<T, C>(ctx, A22, L21, U12, rest, rest, m, lda, s)) return rc;
        }
        if (int rc = bem_check_cuda(ctx, cudaGetLastError(), "tiled lu step")) return rc;
    }
    // the tensor-core update records a bounded-wait timeout in flags[4]
    int32_t tc_err = 0;
    if (int rc = bem_check_cuda(ctx, cudaMemcpyAsync(&tc_err, ctx->flags + 4, sizeof(int32_t), cudaMemcpyDeviceToHost,
                                                     s), "flag readback"))
        return rc;
    if (int rc = bem_check_cuda(ctx, cudaStreamSynchronize(s), "tiled lu")) return rc;
    if (tc_err != 0) {
        cudaMemsetAsync(ctx->flags + 4, 0, sizeof(int32_t), s);
        return bem_fail(ctx, BEM_ERR_TIMEOUT, "tiled lu: a tensor-core wait hit its iteration cap");
    }
    return BEM_OK;
}

template <typename T, bool C>
int solve_t(bem_ctx* ctx, const T* LU, int64_t n, int64_t lda, const int32_t* piv, const CE<T>* dinv, double* b,
            cudaStream_t s) {
    const int W = C ? 2 : 1;
    const int nbk = (int)((n + LU_T - 1) / LU_T);
    // workspace: perm [n], flags [2*nbk], x [W*n]
    size_t off_flags = ((size_t)n * 4 + 255) & ~size_t(255);
    size_t off_x = off_flags + (((size_t)2 * nbk * 4 + 255) & ~size_t(255));
    size_t total = off_x + sizeof(double) * W * (size_t)n;
    if (int rc = bem_ws_reserve(ctx, total)) return rc;
    char* base = (char*)ctx->ws;
    int32_t* perm = (int32_t*)base;
    int* flags = (int*)(base + off_flags);
    double* x = (double*)(base + off_x);
    if ((size_t)n * sizeof(int32_t) > 200 * 1024) return bem_fail(ctx, BEM_ERR_INVALID, "tiled solve: n > 51200");
    cudaFuncSetAttribute(tile_piv_to_perm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)(n * sizeof(int32_t)));
    tile_piv_to_perm_kernel<<<1, 256, n * sizeof(int32_t), s>>>(piv, perm, (int)n);
    permute_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(b, perm, x, (int)n, W);
    cudaMemsetAsync(flags, 0, sizeof(int) * 2 * nbk, s);
    cudaMemsetAsync(ctx->flags + 3, 0, sizeof(int32_t), s);
    ctx->launches += 2;
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, tile_solve_kernel<T, C>, 256, 0);
    int P = std::max(1, std::min(nbk, per_sm * ctx->num_sms));
    P = std::min(P, ctx->num_sms);
    int ni = (int)n, epoch = 1;
    int32_t* err = ctx->flags + 3;
    void* args[] = {(void*)&LU, &lda, &ni, (void*)&dinv, &x, &flags, &epoch, &err};
    if (int rc = bem_check_cuda(ctx, cudaLaunchCooperativeKernel((const void*)tile_solve_kernel<T, C>, P, 256, args,
                                                                0, s),
                                "tile_solve_kernel"))
        return rc;
    ctx->launches++;
    if (int rc = bem_check_cuda(ctx, cudaMemcpyAsync(b, x, sizeof(double) * W * n, cudaMemcpyDeviceToDevice, s),
                                "tiled solve copy"))
        return rc;
    int32_t e = 0;
    cudaMemcpyAsync(&e, err, sizeof(int32_t), cudaMemcpyDeviceToHost, s);
    if (int rc = bem_check_cuda(ctx, cudaStreamSynchronize(s), "tiled solve")) return rc;
    if (e != 0) return bem_fail(ctx, BEM_ERR_TIMEOUT, "tiled solve: a ready-flag wait hit its iteration cap");
    return BEM_OK;
}

}  // namespace

extern "C" {

int64_t bem_lu_dinv_elems(int64_t n) { return ((n + LU_T - 1) / LU_T) * 2 * LU_T * LU_T; }

int bem_lu_factor_tiled(bem_ctx* ctx, int dtype, void* A, int64_t n, int64_t lda, int32_t* piv, void* dinv,
                        int32_t* info, void* stream) {
    if (!ctx) return BEM_ERR_INVALID;
    if (!A || !piv || !dinv || !info || n <= 0 || lda < n || n > (1 << 30))
        return bem_fail(ctx, BEM_ERR_INVALID, "lu_factor_tiled: bad arguments");
    cudaStream_t s = (cudaStream_t)stream;
    switch (dtype) {
        case BEM_F64: return factor_t<double, false>(ctx, (double*)A, n, lda, piv, (CE<double>*)dinv, info, s);
        case BEM_C128: return factor_t<double, true>(ctx, (double*)A, n, lda, piv, (CE<double>*)dinv, info, s);
        case BEM_F32: return factor_t<float, false>(ctx, (float*)A, n, lda, piv, (CE<float>*)dinv, info, s);
        case BEM_C64: return factor_t<float, true>(ctx, (float*)A, n, lda, piv, (CE<float>*)dinv, info, s);
        default: return bem_fail(ctx, BEM_ERR_INVALID, "lu_factor_tiled: unknown dtype");
    }
}

int bem_lu_solve_tiled(bem_ctx* ctx, int dtype, const void* LU, int64_t n, int64_t lda, const int32_t* piv,
                       const void* dinv, void* b, void* stream) {
    if (!ctx) return BEM_ERR_INVALID;
    if (!LU || !piv || !dinv || !b || n <= 0 || lda < n)
        return bem_fail(ctx, BEM_ERR_INVALID, "lu_solve_tiled: bad arguments");
    cudaStream_t s = (cudaStream_t)stream;
    switch (dtype) {
        case BEM_F64: return solve_t<double, false>(ctx, (const double*)LU, n, lda, piv, (const CE<double>*)dinv, (double*)b, s);
        case BEM_C128: return solve_t<double, true>(ctx, (const double*)LU, n, lda, piv, (const CE<double>*)dinv, (double*)b, s);
        case BEM_F32: return solve_t<float, false>(ctx, (const float*)LU, n, lda, piv, (const CE<float>*)dinv, (double*)b, s);
        case BEM_C64: return solve_t<float, true>(ctx, (const float*)LU, n, lda, piv, (const CE<float>*)dinv, (double*)b, s);
        default: return bem_fail(ctx, BEM_ERR_INVALID, "lu_solve_tiled: unknown dtype");
    }
}

}  // extern "C"

// ----------------------------------------------------------------------------
// Allocation-free variant of bem_lu_solve_tiled.
//
// Its scratch (row permutation, ready flags, error word, work vector) lives in
// one file-scope __device__ array instead of a context workspace, so the call
// needs no bem_ctx and performs no device allocation.  The array is sized for
// n <= BEM_STATIC_SOLVE_MAX_N and is held by every GPU that loads this library
// until the process exits.  Host code only ever sees the array's host-side
// stand-in name; its device address comes from cudaGetSymbolAddress, taken
// once per device (with that device current) on the first call there.
// ----------------------------------------------------------------------------
#include <mutex>

namespace {

constexpr int64_t kStaticSolveMaxN = BEM_STATIC_SOLVE_MAX_N;
constexpr int kStaticSolveMaxTiles = (int)((kStaticSolveMaxN + LU_T - 1) / LU_T);

struct StaticSolveScratch {
    int32_t perm[kStaticSolveMaxN];
    int flags[2 * kStaticSolveMaxTiles];
    int32_t err[4];
    double x[2 * kStaticSolveMaxN];
};

__device__ __align__(256) StaticSolveScratch g_static_solve_scratch;

constexpr int kMaxDevices = 64;
std::mutex g_static_mu;
StaticSolveScratch* g_static_addr[kMaxDevices] = {};

// Device address of the scratch array on the current device (set-up on the
// first call per device).
int static_scratch(StaticSolveScratch** out) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return BEM_ERR_CUDA;
    }
    if (dev < 0 || dev >= kMaxDevices) return BEM_ERR_INVALID;
    std::lock_guard<std::mutex> lock(g_static_mu);
    if (!g_static_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_static_solve_scratch);
        if (e != cudaSuccess || p == nullptr) {
            cudaGetLastError();
            return BEM_ERR_CUDA;
        }
        g_static_addr[dev] = static_cast<StaticSolveScratch*>(p);
    }
    *out = g_static_addr[dev];
    return BEM_OK;
}

template <typename T, bool C>
int solve_static_t(const T* LU, int64_t n, int64_t lda, const int32_t* piv, const CE<T>* dinv, double* b,
                   cudaStream_t s) {
    StaticSolveScratch* sc = nullptr;
    if (int rc = static_scratch(&sc)) return rc;
    const int W = C ? 2 : 1;
    const int nbk = (int)((n + LU_T - 1) / LU_T);
    int dev = 0, sms = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int32_t* perm = sc->perm;
    int* flags = sc->flags;
    int32_t* err = sc->err;
    double* x = sc->x;
    if (cudaFuncSetAttribute(tile_piv_to_perm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(n * sizeof(int32_t))) != cudaSuccess) {
        cudaGetLastError();
        return BEM_ERR_CUDA;
    }
    tile_piv_to_perm_kernel<<<1, 256, n * sizeof(int32_t), s>>>(piv, perm, (int)n);
    permute_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(b, perm, x, (int)n, W);
    // the array keeps the previous call's contents: the flags and the error
    // word must start at zero
    if (cudaMemsetAsync(flags, 0, sizeof(int) * 2 * nbk, s) != cudaSuccess ||
        cudaMemsetAsync(err, 0, sizeof(int32_t), s) != cudaSuccess) {
        cudaGetLastError();
        return BEM_ERR_CUDA;
    }
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, tile_solve_kernel<T, C>, 256, 0);
    int P = std::max(1, std::min(nbk, std::min(per_sm * sms, sms)));
    int ni = (int)n, epoch = 1;
    void* args[] = {(void*)&LU, &lda, &ni, (void*)&dinv, &x, &flags, &epoch, &err};
    if (cudaLaunchCooperativeKernel((const void*)tile_solve_kernel<T, C>, P, 256, args, 0, s) != cudaSuccess) {
        cudaGetLastError();
        return BEM_ERR_CUDA;
    }
    if (cudaMemcpyAsync(b, x, sizeof(double) * W * n, cudaMemcpyDeviceToDevice, s) != cudaSuccess) {
        cudaGetLastError();
        return BEM_ERR_CUDA;
    }
    int32_t e = 0;
    if (cudaMemcpyAsync(&e, err, sizeof(int32_t), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) {
        cudaGetLastError();
        return BEM_ERR_CUDA;
    }
    return e != 0 ? BEM_ERR_TIMEOUT : BEM_OK;
}

}  // namespace

extern "C" int bem_lu_solve_tiled_static(int dtype, const void* LU, int64_t n, int64_t lda, const int32_t* piv,
                                         const void* dinv, void* b, void* stream) {
    if (!LU || !piv || !dinv || !b || n <= 0 || lda < n) return BEM_ERR_INVALID;
    if (n > kStaticSolveMaxN) return BEM_ERR_INVALID;  // beyond the static scratch
    cudaStream_t s = (cudaStream_t)stream;
    switch (dtype) {
        case BEM_F64: return solve_static_t<double, false>((const double*)LU, n, lda, piv, (const CE<double>*)dinv, (double*)b, s);
        case BEM_C128: return solve_static_t<double, true>((const double*)LU, n, lda, piv, (const CE<double>*)dinv, (double*)b, s);
        case BEM_F32: return solve_static_t<float, false>((const float*)LU, n, lda, piv, (const CE<float>*)dinv, (double*)b, s);
        case BEM_C64: return solve_static_t<float, true>((const float*)LU, n, lda, piv, (const CE<float>*)dinv, (double*)b, s);
        default: return BEM_ERR_INVALID;
    }
}
