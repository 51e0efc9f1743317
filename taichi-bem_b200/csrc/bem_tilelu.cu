// Tile-pivoted LU and barrier-free triangular solves (the low-precision factor
// of the mixed path).
//
// Factorisation, per diagonal block k (LU_T = 64 columns):
//   diag   : one CTA factors the 64x64 diagonal block with partial pivoting
//            restricted to the block's rows;
//   laswp  : the block's row swaps applied to the other columns;
//   U12 = L11^{-1} A12 and L21 = A21 U11^{-1}: one CTA per 64-wide tile,
//            substitution against the factored diagonal block, blocked by 8
//            rows (columns), in shared memory (two CTA barriers per block);
//   update : A22 -= L21 U12 (the trailing GEMM of bem_gemm.cuh).
// After the last block, one launch forms the explicit inverses Linv_k (unit
// lower) and Uinv_k (upper) of every diagonal block (`dinv`, used by the
// solves), one CTA per block, off the factorisation's dependency chain.
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
// diagonal tile: GEPP inside the tile; explicit inverses of the factored tiles
// --------------------------------------------------------------------------
// Pivot key of a candidate: |re| + |im| as float bits (monotonic for
// non-negative floats) above 63 - row, so that atomicMax picks the largest
// magnitude and, among equal ones, the smallest row (the first maximum).  NaN
// counts as 0.
template <typename T>
__device__ __forceinline__ unsigned long long pivot_key(CE<T> v, int r) {
    float a = (float)(fabs(v.re) + fabs(v.im));
    if (!(a == a)) a = 0.0f;
    return ((unsigned long long)__float_as_uint(a) << 32) | (unsigned)(LU_T - 1 - r);
}

constexpr int DIAG_LD = LU_T + 1;  // padded row stride: column reads hit distinct banks
constexpr int DIAG_PW = 8;         // panel width of the blocked factorisation
constexpr size_t diag_smem_bytes(size_t elem) { return elem * LU_T * DIAG_LD; }
// tile_inv_kernel: the factored block and the inverse being built
constexpr size_t inv_smem_bytes(size_t elem) { return elem * (LU_T * DIAG_LD + LU_T * LU_T); }

// One CTA of 256 threads factors the 64x64 diagonal tile (GEPP restricted to
// the tile's rows).  Blocked by panels of
// DIAG_PW columns:
//   panel  : the 64 x DIAG_PW panel in registers (two elements per thread);
//            per column a pivot max over packed keys (shuffles, then across
//            the 8 warps), the pivot row exchanged through shared memory,
//            multipliers shuffled within each row's four threads; two CTA
//            barriers per column; the panel's row swaps are applied to the
//            other columns once the panel is done;
//   U12    : the panel's rows right of it, L11^{-1} applied by substitution
//            (one thread per column);
//   update : rank-DIAG_PW update of the trailing block, one column per thread
//            with the column's U12 values held in registers.
// The explicit inverses are formed later, by tile_inv_kernel.  Shared memory
// (33 KB for complex FP32) leaves room for the trailing GEMM's CTAs on an SM.
template <typename T, bool C>
__global__ void __launch_bounds__(256) tile_diag_kernel(T* A, int64_t lda, int n, int k0, int32_t* piv,
                                                        int32_t* info) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    CE<T>* S = reinterpret_cast<CE<T>*>(smem_raw);  // [LU_T][DIAG_LD]
    __shared__ int s_zero_pivot;                    // first zero pivot of this tile (1-based), 0 = none
    __shared__ unsigned long long s_wkey[8];        // per-warp pivot keys
    __shared__ CE<T> s_rowj[DIAG_PW], s_rowp[DIAG_PW];
    __shared__ int s_perm[DIAG_PW];                 // pivot rows of the current panel
    const int m = min(LU_T, n - k0);
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    if (tid == 0) s_zero_pivot = 0;
    for (int e = tid; e < LU_T * LU_T; e += blockDim.x) {
        const int r = e / LU_T, c = e - r * LU_T;
        CE<T> v = CE<T>{T(0), T(0)};
        if (r < m && c < m) v = ldE<T, C>(A, (int64_t)(k0 + r) * lda + k0 + c);
        S[r * DIAG_LD + c] = v;
    }
    __syncthreads();
    // panel registers: thread t holds row pr = t >> 2, panel columns 2*pc, 2*pc+1 (pc = t & 3)
    const int pr = tid >> 2, pc = tid & 3;
    for (int j0 = 0; j0 < m; j0 += DIAG_PW) {
        const int w = min(DIAG_PW, m - j0);
        CE<T> e0 = S[pr * DIAG_LD + j0 + 2 * pc], e1 = S[pr * DIAG_LD + j0 + 2 * pc + 1];
        for (int j = j0; j < j0 + w; ++j) {
            const int jq = j - j0;  // panel column of j, held by threads with pc == jq / 2
            // pivot: largest |re| + |im| in column j among rows j..m-1 (first one on ties):
            // owners post keys, max over the warp's rows, then over the 8 warps
            unsigned long long key = 0ull;
            if (pc == (jq >> 1) && pr >= j && pr < m) key = pivot_key((jq & 1) ? e1 : e0, pr);
#pragma unroll
            for (int o = 4; o < 32; o <<= 1) {
                const unsigned long long ko = __shfl_xor_sync(0xffffffffu, key, o);
                key = ko > key ? ko : key;
            }
            if (lane == (jq >> 1)) s_wkey[wid] = key;
            __syncthreads();
            unsigned long long best = s_wkey[0];
#pragma unroll
            for (int q = 1; q < 8; ++q) best = s_wkey[q] > best ? s_wkey[q] : best;
            const int p = LU_T - 1 - (int)(best & 0xffffffffull);
            const int prow = (p >= j && p < m) ? p : j;  // all-zero or NaN column: no swap
            // exchange rows j and prow inside the panel; everyone reads the new pivot row
            if (pr == j) {
                s_rowj[2 * pc] = e0;
                s_rowj[2 * pc + 1] = e1;
            }
            if (pr == prow) {
                s_rowp[2 * pc] = e0;
                s_rowp[2 * pc + 1] = e1;
            }
            __syncthreads();
            if (prow != j) {
                if (pr == j) {
                    e0 = s_rowp[2 * pc];
                    e1 = s_rowp[2 * pc + 1];
                } else if (pr == prow) {
                    e0 = s_rowj[2 * pc];
                    e1 = s_rowj[2 * pc + 1];
                }
            }
            const CE<T> pv = s_rowp[jq];
            if (tid == 0) {
                s_perm[jq] = prow;
                piv[k0 + j] = k0 + prow;
                if (!((double)pv.re != 0.0 || (double)pv.im != 0.0) && s_zero_pivot == 0) s_zero_pivot = k0 + j + 1;
            }
            // multiplier of row pr (held by the thread of column j), shared within the row's 4 lanes
            CE<T> l = CE<T>{T(0), T(0)};
            if (pc == (jq >> 1)) l = cmul((jq & 1) ? e1 : e0, cinv(pv));
            const int src = (lane & ~3) | (jq >> 1);
            l.re = __shfl_sync(0xffffffffu, l.re, src);
            l.im = __shfl_sync(0xffffffffu, l.im, src);
            if (pr > j && pr < m) {
                const int c0 = j0 + 2 * pc, c1e = c0 + 1;
                if (c0 == j) {
                    e0 = l;
                } else if (c0 > j && c0 < j0 + w) {
                    const CE<T> u = s_rowp[2 * pc];
                    e0.re -= l.re * u.re - l.im * u.im;
                    e0.im -= l.re * u.im + l.im * u.re;
                }
                if (c1e == j) {
                    e1 = l;
                } else if (c1e > j && c1e < j0 + w) {
                    const CE<T> u = s_rowp[2 * pc + 1];
                    e1.re -= l.re * u.re - l.im * u.im;
                    e1.im -= l.re * u.im + l.im * u.re;
                }
            }
            __syncthreads();  // s_rowj / s_rowp / s_wkey are reused by the next column
        }
        // panel back to shared memory; the panel's swaps applied to the other columns
        if (pr < m) {
            if (2 * pc < w) S[pr * DIAG_LD + j0 + 2 * pc] = e0;
            if (2 * pc + 1 < w) S[pr * DIAG_LD + j0 + 2 * pc + 1] = e1;
        }
        if (tid < LU_T && (tid < j0 || tid >= j0 + w)) {
            for (int q = 0; q < w; ++q) {
                const int ra = j0 + q, rb = s_perm[q];
                if (rb != ra) {
                    const CE<T> t = S[ra * DIAG_LD + tid];
                    S[ra * DIAG_LD + tid] = S[rb * DIAG_LD + tid];
                    S[rb * DIAG_LD + tid] = t;
                }
            }
        }
        __syncthreads();
        const int c1 = j0 + w;  // first column right of the panel
        if (c1 < m) {
            // U12 = L11^{-1} A12: rows j0..c1-1, one thread per column
            for (int c = c1 + tid; c < m; c += blockDim.x) {
                CE<T> u[DIAG_PW];
#pragma unroll
                for (int i = 0; i < DIAG_PW; ++i) {
                    if (i < w) {
                        CE<T> v = S[(j0 + i) * DIAG_LD + c];
#pragma unroll
                        for (int q = 0; q < i; ++q) {
                            const CE<T> l = S[(j0 + i) * DIAG_LD + j0 + q];
                            v.re -= l.re * u[q].re - l.im * u[q].im;
                            v.im -= l.re * u[q].im + l.im * u[q].re;
                        }
                        u[i] = v;
                        S[(j0 + i) * DIAG_LD + c] = v;
                    }
                }
            }
            __syncthreads();
            // A22 -= L21 U12: thread column c1 + (tid & 63), rows (tid >> 6) + 4k
            const int cc = c1 + (tid & 63);
            if (cc < m) {
                CE<T> u[DIAG_PW];
#pragma unroll
                for (int q = 0; q < DIAG_PW; ++q)
                    u[q] = q < w ? S[(j0 + q) * DIAG_LD + cc] : CE<T>{T(0), T(0)};
                for (int r = c1 + (tid >> 6); r < m; r += 4) {
                    CE<T> v = S[r * DIAG_LD + cc];
#pragma unroll
                    for (int q = 0; q < DIAG_PW; ++q) {
                        const CE<T> l = S[r * DIAG_LD + j0 + q];
                        v.re -= l.re * u[q].re - l.im * u[q].im;
                        v.im -= l.re * u[q].im + l.im * u[q].re;
                    }
                    S[r * DIAG_LD + cc] = v;
                }
            }
            __syncthreads();
        }
    }
    if (tid == 0 && s_zero_pivot != 0 && *info == 0) *info = s_zero_pivot;
    for (int e = tid; e < LU_T * LU_T; e += blockDim.x) {
        const int r = e / LU_T, cc = e - r * LU_T;
        if (r < m && cc < m) stE<T, C>(A, (int64_t)(k0 + r) * lda + k0 + cc, S[r * DIAG_LD + cc]);
    }
}


// Explicit inverses Linv (unit lower) and Uinv (upper) of every factored
// diagonal block, one CTA per block (blockIdx.x = block), by block
// substitution over DIAG_PW-row blocks against the identity.  Runs once the
// factorisation is complete: later row swaps never touch a diagonal block.
template <typename T, bool C>
__global__ void __launch_bounds__(256) tile_inv_kernel(const T* A, int64_t lda, int n, CE<T>* dinv) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    CE<T>* S = reinterpret_cast<CE<T>*>(smem_raw);  // [LU_T][DIAG_LD] factored block
    CE<T>* X = S + LU_T * DIAG_LD;                  // [LU_T][LU_T] inverse being built
    const int k0 = blockIdx.x * LU_T;
    const int m = min(LU_T, n - k0);
    const int tid = threadIdx.x;
    for (int e = tid; e < LU_T * LU_T; e += blockDim.x) {
        const int r = e / LU_T, c = e - r * LU_T;
        CE<T> v = CE<T>{T(0), T(0)};
        if (r < m && c < m) v = ldE<T, C>(A, (int64_t)(k0 + r) * lda + k0 + c);
        S[r * DIAG_LD + c] = v;
    }
    __syncthreads();
    CE<T>* D = dinv + (size_t)blockIdx.x * 2 * LU_T * LU_T;
    // ---- explicit inverses by block substitution against the identity ----
    // Linv: for row block i: X_i = L_ii^{-1} (E_i - sum_{k<i} L_ik X_k)
    // Uinv: for row block i (descending): X_i = U_ii^{-1} (E_i - sum_{k>i} U_ik X_k)
    // thread: column c = tid & 63, rows (tid >> 6) * 2 + {0, 1} of the block
    __shared__ CE<T> s_rdiag[LU_T];  // 1 / U[r][r], formed in parallel off the substitution chain
    if (tid < LU_T) s_rdiag[tid] = tid < m ? cinv(S[tid * DIAG_LD + tid]) : CE<T>{T(1), T(0)};
    const int c = tid & 63, rq = (tid >> 6) * 2;
    for (int which = 0; which < 2; ++which) {
        for (int bs = 0; bs < LU_T / DIAG_PW; ++bs) {
            const int ib = which == 0 ? bs : LU_T / DIAG_PW - 1 - bs;
            const int r0 = ib * DIAG_PW;
            // T = E_i - sum over finished blocks, two rows per thread
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int r = r0 + rq + h;
                CE<T> v = CE<T>{r == c ? T(1) : T(0), T(0)};
                if (r < m) {
                    if (which == 0) {
                        for (int q = 0; q < r0; ++q) {
                            const CE<T> l = S[r * DIAG_LD + q], x = X[q * LU_T + c];
                            v.re -= l.re * x.re - l.im * x.im;
                            v.im -= l.re * x.im + l.im * x.re;
                        }
                    } else {
                        for (int q = r0 + DIAG_PW; q < m; ++q) {
                            const CE<T> uu = S[r * DIAG_LD + q], x = X[q * LU_T + c];
                            v.re -= uu.re * x.re - uu.im * x.im;
                            v.im -= uu.re * x.im + uu.im * x.re;
                        }
                    }
                }
                X[r * LU_T + c] = v;
            }
            __syncthreads();
            // diagonal block: substitution down (Linv) or up (Uinv) the 8 rows, one thread per column
            if (tid < LU_T) {
                CE<T> y[DIAG_PW];
#pragma unroll
                for (int i = 0; i < DIAG_PW; ++i) y[i] = X[(r0 + i) * LU_T + c];
                if (which == 0) {
#pragma unroll
                    for (int i = 0; i < DIAG_PW; ++i) {
                        const int r = r0 + i;
                        if (r >= m) {
                            y[i] = CE<T>{r == c ? T(1) : T(0), T(0)};  // identity padding of a short last tile
                            continue;
                        }
#pragma unroll
                        for (int q = 0; q < i; ++q) {
                            const CE<T> l = S[r * DIAG_LD + r0 + q];
                            y[i].re -= l.re * y[q].re - l.im * y[q].im;
                            y[i].im -= l.re * y[q].im + l.im * y[q].re;
                        }
                    }
                } else {
#pragma unroll
                    for (int i = DIAG_PW - 1; i >= 0; --i) {
                        const int r = r0 + i;
                        if (r >= m) {
                            y[i] = CE<T>{r == c ? T(1) : T(0), T(0)};
                            continue;
                        }
                        if (c >= m) {
                            y[i] = CE<T>{T(0), T(0)};
                            continue;
                        }
#pragma unroll
                        for (int q = i + 1; q < DIAG_PW; ++q) {
                            if (r0 + q >= m) continue;
                            const CE<T> uu = S[r * DIAG_LD + r0 + q];
                            y[i].re -= uu.re * y[q].re - uu.im * y[q].im;
                            y[i].im -= uu.re * y[q].im + uu.im * y[q].re;
                        }
                        y[i] = cmul(y[i], s_rdiag[r]);
                    }
                }
#pragma unroll
                for (int i = 0; i < DIAG_PW; ++i) X[(r0 + i) * LU_T + c] = y[i];
            }
            __syncthreads();
        }
        for (int e = tid; e < LU_T * LU_T; e += blockDim.x) D[which * LU_T * LU_T + e] = X[e];
        __syncthreads();
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

// blockIdx.y = 0: U12 tile (rows k0.., 64 columns) <- L11^{-1} tile (unit lower)
// blockIdx.y = 1: L21 tile (64 rows, columns k0..) <- tile U11^{-1} (upper)
// Both run in one launch (they touch disjoint parts of A).  The factored
// diagonal block and the tile are staged in shared memory and the
// substitution is blocked by APPLY_B rows (mode 0) or columns (mode 1): the
// block's own triangle is solved by one thread per column (row), sequentially
// over the APPLY_B entries, then every thread applies the block's rank-APPLY_B
// update to its entries below (right of) it -- two CTA barriers per block.
constexpr int APPLY_LD = LU_T + 1;
constexpr int APPLY_B = 8;
constexpr size_t apply_smem_bytes(size_t elem) { return 2 * elem * LU_T * APPLY_LD; }

template <typename T, bool C>
__global__ void __launch_bounds__(256) tile_apply_kernel(T* A, int64_t lda, int n, int k0, int m) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    CE<T>* M = reinterpret_cast<CE<T>*>(smem_raw);  // [LU_T][APPLY_LD] factored diagonal block
    CE<T>* X = M + LU_T * APPLY_LD;                 // [LU_T][APPLY_LD] the tile
    __shared__ CE<T> s_rdiag[LU_T];
    const int mode = blockIdx.y;
    const int base = k0 + m + blockIdx.x * LU_T;  // first column (mode 0) / row (mode 1) of the tile
    const int cnt = min(LU_T, n - base);
    for (int e = threadIdx.x; e < LU_T * LU_T; e += blockDim.x) {
        const int r = e / LU_T, c = e - r * LU_T;
        CE<T> d = CE<T>{T(0), T(0)}, v = CE<T>{T(0), T(0)};
        if (r < m && c < m) d = ldE<T, C>(A, (int64_t)(k0 + r) * lda + k0 + c);
        if (mode == 0) {
            if (r < m && c < cnt) v = ldE<T, C>(A, (int64_t)(k0 + r) * lda + base + c);
        } else {
            if (r < cnt && c < m) v = ldE<T, C>(A, (int64_t)(base + r) * lda + k0 + c);
        }
        M[r * APPLY_LD + c] = d;
        X[r * APPLY_LD + c] = v;
    }
    __syncthreads();
    if (mode == 1 && threadIdx.x < LU_T)
        s_rdiag[threadIdx.x] = threadIdx.x < m ? cinv(M[threadIdx.x * APPLY_LD + threadIdx.x]) : CE<T>{T(0), T(0)};
    __syncthreads();
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int t = threadIdx.x;
    for (int b0 = 0; b0 < m; b0 += APPLY_B) {
        const int bw = min(APPLY_B, m - b0);
        if (mode == 0) {
            // rows b0..b0+bw-1: X_b <- L_bb^{-1} X_b, one thread per column
            if (t < LU_T) {
                CE<T> y[APPLY_B];
#pragma unroll
                for (int i = 0; i < APPLY_B; ++i) {
                    if (i >= bw) break;
                    CE<T> v = X[(b0 + i) * APPLY_LD + t];
#pragma unroll
                    for (int q = 0; q < i; ++q) {
                        const CE<T> l = M[(b0 + i) * APPLY_LD + b0 + q];
                        v.re -= l.re * y[q].re - (C ? l.im * y[q].im : T(0));
                        if (C) v.im -= l.re * y[q].im + l.im * y[q].re;
                    }
                    y[i] = v;
                    X[(b0 + i) * APPLY_LD + t] = v;
                }
            }
            __syncthreads();
            // rows below the block: X_r -= L_rb X_b
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int r = ty + 16 * i;
                if (r < b0 + bw) continue;
                CE<T> l[APPLY_B];
#pragma unroll
                for (int q = 0; q < APPLY_B; ++q)
                    l[q] = q < bw ? M[r * APPLY_LD + b0 + q] : CE<T>{T(0), T(0)};
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int c = tx + 16 * j;
                    CE<T> v = X[r * APPLY_LD + c];
#pragma unroll
                    for (int q = 0; q < APPLY_B; ++q) {
                        if (q >= bw) break;
                        const CE<T> u = X[(b0 + q) * APPLY_LD + c];
                        v.re -= l[q].re * u.re - (C ? l[q].im * u.im : T(0));
                        if (C) v.im -= l[q].re * u.im + l[q].im * u.re;
                    }
                    X[r * APPLY_LD + c] = v;
                }
            }
            __syncthreads();
        } else {
            // columns b0..b0+bw-1: X_b <- X_b U_bb^{-1}, one thread per row
            if (t < LU_T) {
                CE<T> y[APPLY_B];
#pragma unroll
                for (int j = 0; j < APPLY_B; ++j) {
                    if (j >= bw) break;
                    CE<T> v = X[t * APPLY_LD + b0 + j];
#pragma unroll
                    for (int q = 0; q < j; ++q) {
                        const CE<T> u = M[(b0 + q) * APPLY_LD + b0 + j];
                        v.re -= y[q].re * u.re - (C ? y[q].im * u.im : T(0));
                        if (C) v.im -= y[q].re * u.im + y[q].im * u.re;
                    }
                    y[j] = cmul(v, s_rdiag[b0 + j]);
                    X[t * APPLY_LD + b0 + j] = y[j];
                }
            }
            __syncthreads();
            // columns right of the block: X_c -= X_b U_bc
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int c = tx + 16 * j;
                if (c < b0 + bw) continue;
                CE<T> u[APPLY_B];
#pragma unroll
                for (int q = 0; q < APPLY_B; ++q)
                    u[q] = q < bw ? M[(b0 + q) * APPLY_LD + c] : CE<T>{T(0), T(0)};
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const int r = ty + 16 * i;
                    CE<T> v = X[r * APPLY_LD + c];
#pragma unroll
                    for (int q = 0; q < APPLY_B; ++q) {
                        if (q >= bw) break;
                        const CE<T> l = X[r * APPLY_LD + b0 + q];
                        v.re -= l.re * u[q].re - (C ? l.im * u[q].im : T(0));
                        if (C) v.im -= l.re * u[q].im + l.im * u[q].re;
                    }
                    X[r * APPLY_LD + c] = v;
                }
            }
            __syncthreads();
        }
    }
    for (int e = threadIdx.x; e < LU_T * LU_T; e += blockDim.x) {
        const int r = e / LU_T, c = e - r * LU_T;
        if (mode == 0) {
            if (r < m && c < cnt) stE<T, C>(A, (int64_t)(k0 + r) * lda + base + c, X[r * APPLY_LD + c]);
        } else {
            if (r < cnt && c < m) stE<T, C>(A, (int64_t)(base + r) * lda + k0 + c, X[r * APPLY_LD + c]);
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

// Warp-level bounded wait for a ready flag: lane 0 spins with acquire loads,
// the warp barrier that follows orders the other lanes' reads after it.
__device__ __forceinline__ bool warp_wait_flag(const int* flags, int j, int epoch, int32_t* err) {
    int ok = 1;
    if ((threadIdx.x & 31) == 0) {
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
    }
    ok = __shfl_sync(0xffffffffu, ok, 0);
    __syncwarp();
    return ok != 0;
}

// x (FP64, real or complex interleaved, one right-hand side) overwritten by
// U^{-1} L^{-1} x; the input must already be permuted (x = P b).
// Block row k, per pass (forward with L, backward with U):
//   * the block of the last dependency (L_k,k-1 or U_k,k+1) and the diagonal
//     inverse (Linv_k or Uinv_k) are prefetched into shared memory;
//   * every other finished block j is streamed from memory: warp w owns rows
//     w, w+8, ... and keeps per-lane partial sums of L_kj x_j (in the factor's
//     precision), two blocks per iteration, no CTA barrier, one cross-lane
//     reduction at the end;
//   * once the last dependency's flag is set only two GEMVs out of shared
//     memory remain on the critical path; x_k is then published with a
//     release store of its flag.
constexpr int SOLVE_LD = LU_T + 4;  // padded row stride of the staged blocks
constexpr size_t solve_smem_bytes(size_t elem) { return 2 * elem * LU_T * SOLVE_LD; }

template <typename T, bool C>
__global__ void __launch_bounds__(256) tile_solve_kernel(const T* LU, int64_t lda, int n, const CE<T>* dinv,
                                                         double* x, int* flags, int epoch, int32_t* err,
                                                         const int* skip) {
    // skip != NULL: a device word set by the asynchronous refinement once it
    // has converged; the later, already queued solves return at once
    if (skip != nullptr && *skip != 0) return;
    constexpr int RW = LU_T / 8;  // rows per warp in the streamed part
    extern __shared__ __align__(16) unsigned char smem_raw[];
    CE<T>* sB = reinterpret_cast<CE<T>*>(smem_raw);  // [LU_T][SOLVE_LD] last dependency block
    CE<T>* sD = sB + LU_T * SOLVE_LD;                 // [LU_T][SOLVE_LD] diagonal inverse
    __shared__ double s_acc[LU_T][2];
    __shared__ double s_x[LU_T][2];
    __shared__ int s_abort;
    const int nbk = (n + LU_T - 1) / LU_T;
    const int P = gridDim.x;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int gr = tid >> 2, gq = tid & 3;  // GEMV mapping: row gr, columns gq + 4i
    const int W = C ? 2 : 1;
    if (tid == 0) s_abort = 0;
    __syncthreads();
    for (int pass = 0; pass < 2; ++pass) {
        const bool fwd = pass == 0;
        for (int t = blockIdx.x; t < nbk; t += P) {
            const int k = fwd ? t : nbk - 1 - t;
            const int r0 = k * LU_T, m = min(LU_T, n - r0);
            const int ndep = fwd ? k : nbk - 1 - k;
            const int jc = ndep > 0 ? (fwd ? k - 1 : k + 1) : -1;  // critical (last) dependency
            // prefetch: diagonal inverse and the critical block
            const CE<T>* Dk = dinv + (size_t)k * 2 * LU_T * LU_T + (fwd ? 0 : LU_T * LU_T);
            for (int e = tid; e < LU_T * LU_T; e += blockDim.x) {
                const int r = e / LU_T, c = e - r * LU_T;
                sD[r * SOLVE_LD + c] = Dk[e];
                CE<T> v = CE<T>{T(0), T(0)};
                if (jc >= 0) {
                    const int c0 = jc * LU_T;
                    if (r < m && c0 + c < n) v = ldE<T, C>(LU, (int64_t)(r0 + r) * lda + c0 + c);
                }
                sB[r * SOLVE_LD + c] = v;
            }
            // streamed dependencies
            T acc_re[RW], acc_im[RW];
#pragma unroll
            for (int i = 0; i < RW; ++i) acc_re[i] = acc_im[i] = T(0);
            auto accum = [&](int j) {
                const int c0 = j * LU_T, mj = min(LU_T, n - c0);
                T xr0 = T(0), xi0 = T(0), xr1 = T(0), xi1 = T(0);
                if (lane < mj) {
                    xr0 = (T)__ldcg(&x[W * (c0 + lane)]);
                    if (C) xi0 = (T)__ldcg(&x[W * (c0 + lane) + 1]);
                }
                if (lane + 32 < mj) {
                    xr1 = (T)__ldcg(&x[W * (c0 + lane + 32)]);
                    if (C) xi1 = (T)__ldcg(&x[W * (c0 + lane + 32) + 1]);
                }
                // all 2 RW loads of the block first, so that they are in flight
                // together, then the products (entries outside the block are zero)
                CE<T> la[RW], lb[RW];
#pragma unroll
                for (int i = 0; i < RW; ++i) {
                    const int r = wid + 8 * i;
                    const T* row = LU + W * ((int64_t)(r0 + r) * lda + c0);
                    la[i] = (r < m && lane < mj) ? ldE<T, C>(row, lane) : CE<T>{T(0), T(0)};
                    lb[i] = (r < m && lane + 32 < mj) ? ldE<T, C>(row, lane + 32) : CE<T>{T(0), T(0)};
                }
#pragma unroll
                for (int i = 0; i < RW; ++i) {
                    acc_re[i] += la[i].re * xr0 - la[i].im * xi0;
                    acc_im[i] += la[i].re * xi0 + la[i].im * xr0;
                    acc_re[i] += lb[i].re * xr1 - lb[i].im * xi1;
                    acc_im[i] += lb[i].re * xi1 + lb[i].im * xr1;
                }
            };
            const int nstream = ndep > 0 ? ndep - 1 : 0;  // all but the critical one
            bool ok = true;
            int d = 0;
            for (; d + 1 < nstream && ok; d += 2) {
                const int j0 = fwd ? d : nbk - 1 - d, j1 = fwd ? d + 1 : nbk - 2 - d;
                ok = warp_wait_flag(flags, pass * nbk + j0, epoch, err) &&
                     warp_wait_flag(flags, pass * nbk + j1, epoch, err);
                if (ok) {
                    accum(j0);
                    accum(j1);
                }
            }
            if (ok && d < nstream) {
                const int j0 = fwd ? d : nbk - 1 - d;
                ok = warp_wait_flag(flags, pass * nbk + j0, epoch, err);
                if (ok) accum(j0);
            }
            if (!ok && lane == 0) s_abort = 1;
#pragma unroll
            for (int i = 0; i < RW; ++i) {
                T sr = acc_re[i], si = acc_im[i];
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    sr += __shfl_xor_sync(0xffffffffu, sr, o);
                    si += __shfl_xor_sync(0xffffffffu, si, o);
                }
                const int r = wid + 8 * i;
                if (lane == 0) {
                    double br = 0.0, bi = 0.0;
                    if (r < m) {
                        br = __ldcg(&x[W * (r0 + r)]) - (double)sr;
                        bi = C ? __ldcg(&x[W * (r0 + r) + 1]) - (double)si : 0.0;
                    }
                    s_acc[r][0] = br;
                    s_acc[r][1] = bi;
                }
            }
            __syncthreads();
            if (s_abort) return;
            // critical dependency out of shared memory
            if (jc >= 0) {
                if (!wait_flag(flags, pass * nbk + jc, epoch, err)) return;
                const int c0 = jc * LU_T, mj = min(LU_T, n - c0);
                if (tid < LU_T) {
                    s_x[tid][0] = tid < mj ? __ldcg(&x[W * (c0 + tid)]) : 0.0;
                    s_x[tid][1] = (C && tid < mj) ? __ldcg(&x[W * (c0 + tid) + 1]) : 0.0;
                }
                __syncthreads();
                T sr = T(0), si = T(0);
#pragma unroll
                for (int i = 0; i < LU_T / 4; ++i) {
                    const int c = gq + 4 * i;
                    const CE<T> l = sB[gr * SOLVE_LD + c];
                    const T xr = (T)s_x[c][0], xi = (T)s_x[c][1];
                    sr += l.re * xr - l.im * xi;
                    si += l.re * xi + l.im * xr;
                }
                sr += __shfl_xor_sync(0xffffffffu, sr, 1);
                si += __shfl_xor_sync(0xffffffffu, si, 1);
                sr += __shfl_xor_sync(0xffffffffu, sr, 2);
                si += __shfl_xor_sync(0xffffffffu, si, 2);
                if (gq == 0 && gr < m) {
                    s_acc[gr][0] -= (double)sr;
                    s_acc[gr][1] -= (double)si;
                }
                __syncthreads();
            }
            // y = inverse(diagonal block) * acc, in FP64
            double yr = 0.0, yi = 0.0;
#pragma unroll
            for (int i = 0; i < LU_T / 4; ++i) {
                const int c = gq + 4 * i;
                const CE<T> dd = sD[gr * SOLVE_LD + c];
                yr += (double)dd.re * s_acc[c][0] - (double)dd.im * s_acc[c][1];
                yi += (double)dd.re * s_acc[c][1] + (double)dd.im * s_acc[c][0];
            }
            yr += __shfl_xor_sync(0xffffffffu, yr, 1);
            yi += __shfl_xor_sync(0xffffffffu, yi, 1);
            yr += __shfl_xor_sync(0xffffffffu, yr, 2);
            yi += __shfl_xor_sync(0xffffffffu, yi, 2);
            if (gq == 0 && gr < m) {
                x[W * (r0 + gr)] = yr;
                if (C) x[W * (r0 + gr) + 1] = yi;
            }
            __threadfence();
            __syncthreads();
            if (tid == 0) st_release_i(flags + pass * nbk + k, epoch);
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

// Row permutation of the tile-pivoted factor: every swap of diagonal tile k
// stays inside the tile's rows, so each tile's permutation is built by its own
// thread (64 sequential swaps in registers-free local order).
__global__ void tile_piv_to_perm_kernel(const int32_t* piv, int32_t* perm, int n) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int k0 = k * LU_T;
    if (k0 >= n) return;
    const int m = min(LU_T, n - k0);
    for (int i = 0; i < m; ++i) perm[k0 + i] = k0 + i;
    for (int i = 0; i < m; ++i) {
        const int p = piv[k0 + i];
        if (p != k0 + i && p >= k0 && p < k0 + m) {
            const int t = perm[k0 + i];
            perm[k0 + i] = perm[p];
            perm[p] = t;
        }
    }
}

template <typename T, bool C>
int factor_t(bem_ctx* ctx, T* A, int64_t n, int64_t lda, int32_t* piv, CE<T>* dinv, int32_t* info,
             cudaStream_t s) {
    cudaMemsetAsync(info, 0, sizeof(int32_t), s);
    const size_t dsmem = diag_smem_bytes(sizeof(CE<T>));
    const size_t asmem = apply_smem_bytes(sizeof(CE<T>));
    cudaFuncSetAttribute(tile_diag_kernel<T, C>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dsmem);
    const size_t ismem = inv_smem_bytes(sizeof(CE<T>));
    cudaFuncSetAttribute(tile_inv_kernel<T, C>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ismem);
    cudaFuncSetAttribute(tile_apply_kernel<T, C>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)asmem);
    if (int rc = bem_lookahead_stream(ctx)) return rc;
    const int ni = (int)n;
    const int W = C ? 2 : 1;
    auto at = [&](int64_t r, int64_t c) { return A + W * (r * lda + c); };
    // A[r0:r0+rows, c0:c0+cols] -= A[r0:r0+rows, q0:q0+kk] A[q0:q0+kk, c0:c0+cols]
    auto update = [&](int64_t r0, int64_t c0, int64_t rows, int64_t cols, int64_t q0, int64_t kk) -> int {
        if (rows <= 0 || cols <= 0 || kk <= 0) return BEM_OK;
        return bem_gemm_update<T, C>(ctx, at(r0, c0), at(r0, q0), at(q0, c0), rows, cols, kk, lda, s);
    };
    // diagonal tile at k0 on the high-priority side stream, after the work queued on s so far
    auto diag_aside = [&](int64_t k0) {
        cudaEventRecord(ctx->ev_next, s);
        cudaStreamWaitEvent(ctx->aux, ctx->ev_next, 0);
        tile_diag_kernel<T, C><<<1, 256, dsmem, ctx->aux>>>(A, lda, ni, (int)k0, piv, info);
        cudaEventRecord(ctx->ev_diag, ctx->aux);
        ctx->launches++;
    };
    // row swaps of tile k0 outside it, then U12 = Linv A12 and L21 = A21 Uinv
    auto panel = [&](int64_t k0, int m) {
        tile_laswp_kernel<T, C><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(A, lda, ni, (int)k0, m, piv);
        ctx->launches++;
        const int64_t rest = n - k0 - m;
        if (rest > 0) {
            const unsigned tiles = (unsigned)((rest + LU_T - 1) / LU_T);
            tile_apply_kernel<T, C><<<dim3(tiles, 2), 256, asmem, s>>>(A, lda, ni, (int)k0, m);
            ctx->launches++;
        }
    };
    // Tiles are taken in pairs (k, k+1) with a delayed update: step k updates
    // only tile k+1's column block (so its diagonal factorisation can start on
    // the side stream) and tile k+1's rows right of it; the trailing block then
    // receives steps k and k+1 together as one rank-128 update (K = 128 halves
    // the read-modify-write traffic of the trailing GEMMs).  The update's first
    // tile column goes first so that the next pair's diagonal tile overlaps the
    // rest of it.
    tile_diag_kernel<T, C><<<1, 256, dsmem, s>>>(A, lda, ni, 0, piv, info);
    ctx->launches++;
    bool on_aux = false;
    for (int64_t k0 = 0; k0 < n; k0 += 2 * LU_T) {
        const int m1 = (int)std::min<int64_t>(LU_T, n - k0);
        if (on_aux) cudaStreamWaitEvent(s, ctx->ev_diag, 0);
        panel(k0, m1);
        const int64_t k1 = k0 + m1, rest1 = n - k1;
        if (rest1 <= 0) break;
        const int m2 = (int)std::min<int64_t>(LU_T, rest1);
        if (int rc = update(k1, k1, rest1, m2, k0, m1)) return rc;
        diag_aside(k1);
        on_aux = true;
        const int64_t c2 = k1 + m2, rest2 = n - c2;
        if (int rc = update(k1, c2, m2, rest2, k0, m1)) return rc;
        cudaStreamWaitEvent(s, ctx->ev_diag, 0);
        panel(k1, m2);
        if (rest2 <= 0) break;
        const int64_t next = std::min<int64_t>(LU_T, rest2);
        if (int rc = update(c2, c2, rest2, next, k0, (int64_t)m1 + m2)) return rc;
        diag_aside(c2);
        if (int rc = update(c2, c2 + next, rest2, rest2 - next, k0, (int64_t)m1 + m2)) return rc;
        if (int rc = bem_check_cuda(ctx, cudaGetLastError(), "tiled lu step")) return rc;
    }
    // explicit inverses of every diagonal block (for the solves)
    tile_inv_kernel<T, C><<<(unsigned)((n + LU_T - 1) / LU_T), 256, ismem, s>>>(A, lda, ni, dinv);
    ctx->launches++;
    // No synchronisation: a tensor-core update whose bounded wait ran out
    // records it in flags[4], which the next solve on this context reads
    // (bem_take_factor_error) after its own synchronisation.
    return bem_check_cuda(ctx, cudaGetLastError(), "tiled lu");
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
    const unsigned ptiles = (unsigned)((n + LU_T - 1) / LU_T);
    tile_piv_to_perm_kernel<<<(ptiles + 127) / 128, 128, 0, s>>>(piv, perm, (int)n);
    permute_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(b, perm, x, (int)n, W);
    cudaMemsetAsync(flags, 0, sizeof(int) * 2 * nbk, s);
    cudaMemsetAsync(ctx->flags + 3, 0, sizeof(int32_t), s);
    ctx->launches += 2;
    const size_t ssmem = solve_smem_bytes(sizeof(CE<T>));
    if (int rc = bem_check_cuda(ctx, cudaFuncSetAttribute(tile_solve_kernel<T, C>,
                                                          cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ssmem),
                                "tile_solve_kernel smem"))
        return rc;
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, tile_solve_kernel<T, C>, 256, ssmem);
    int P = std::max(1, std::min(nbk, per_sm * ctx->num_sms));
    P = std::min(P, ctx->num_sms);
    int ni = (int)n, epoch = 1;
    int32_t* err = ctx->flags + 3;
    const int* no_skip = nullptr;
    void* args[] = {(void*)&LU, &lda, &ni, (void*)&dinv, &x, &flags, &epoch, &err, (void*)&no_skip};
    if (int rc = bem_check_cuda(ctx, cudaLaunchCooperativeKernel((const void*)tile_solve_kernel<T, C>, P, 256, args,
                                                                ssmem, s),
                                "tile_solve_kernel"))
        return rc;
    ctx->launches++;
    if (int rc = bem_check_cuda(ctx, cudaMemcpyAsync(b, x, sizeof(double) * W * n, cudaMemcpyDeviceToDevice, s),
                                "tiled solve copy"))
        return rc;
    int32_t e[2] = {0, 0};
    cudaMemcpyAsync(&e[0], err, sizeof(int32_t), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(&e[1], ctx->flags + 4, sizeof(int32_t), cudaMemcpyDeviceToHost, s);
    if (int rc = bem_check_cuda(ctx, cudaStreamSynchronize(s), "tiled solve")) return rc;
    if (int rc = bem_take_factor_error(ctx, e[1], s)) return rc;
    if (e[0] != 0) return bem_fail(ctx, BEM_ERR_TIMEOUT, "tiled solve: a ready-flag wait hit its iteration cap");
    return BEM_OK;
}

// One preconditioner application of the asynchronous refinement:
// out = (P^T L U)^{-1} r with the tile-pivoted factor, left in the solve
// workspace (*out), queued without synchronisation and skipped on the device
// when *skip != 0.  The caller resets ctx->flags[3] once before its loop and
// reads it after its final synchronisation.
__global__ void permute_if_kernel(const double* b, const int32_t* perm, double* x, int n, int W, const int* skip) {
    if (*skip != 0) return;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int s = perm[i];
    for (int w = 0; w < W; ++w) x[W * i + w] = b[W * s + w];
}

template <typename T, bool C>
int precond_t(bem_ctx* ctx, const T* LU, int64_t n, int64_t lda, const int32_t* piv, const CE<T>* dinv,
              const double* r, double** out, const int* skip, cudaStream_t s) {
    const int W = C ? 2 : 1;
    const int nbk = (int)((n + LU_T - 1) / LU_T);
    size_t off_flags = ((size_t)n * 4 + 255) & ~size_t(255);
    size_t off_x = off_flags + (((size_t)2 * nbk * 4 + 255) & ~size_t(255));
    size_t total = off_x + sizeof(double) * W * (size_t)n;
    if (int rc = bem_ws_reserve(ctx, total)) return rc;
    char* base = (char*)ctx->ws;
    int32_t* perm = (int32_t*)base;
    int* flags = (int*)(base + off_flags);
    double* x = (double*)(base + off_x);
    if ((size_t)n * sizeof(int32_t) > 200 * 1024) return bem_fail(ctx, BEM_ERR_INVALID, "tiled solve: n > 51200");
    const unsigned ptiles = (unsigned)((n + LU_T - 1) / LU_T);
    tile_piv_to_perm_kernel<<<(ptiles + 127) / 128, 128, 0, s>>>(piv, perm, (int)n);
    permute_if_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(r, perm, x, (int)n, W, skip);
    cudaMemsetAsync(flags, 0, sizeof(int) * 2 * nbk, s);
    ctx->launches += 2;
    const size_t ssmem = solve_smem_bytes(sizeof(CE<T>));
    if (int rc = bem_check_cuda(ctx, cudaFuncSetAttribute(tile_solve_kernel<T, C>,
                                                          cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ssmem),
                                "tile_solve_kernel smem"))
        return rc;
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, tile_solve_kernel<T, C>, 256, ssmem);
    int P = std::max(1, std::min(nbk, per_sm * ctx->num_sms));
    P = std::min(P, ctx->num_sms);
    int ni = (int)n, epoch = 1;
    int32_t* err = ctx->flags + 3;
    void* args[] = {(void*)&LU, &lda, &ni, (void*)&dinv, &x, &flags, &epoch, &err, (void*)&skip};
    if (int rc = bem_check_cuda(ctx, cudaLaunchCooperativeKernel((const void*)tile_solve_kernel<T, C>, P, 256, args,
                                                                ssmem, s),
                                "tile_solve_kernel"))
        return rc;
    ctx->launches++;
    *out = x;
    return BEM_OK;
}

}  // namespace

extern "C" {

int bem_lu_factor_status(bem_ctx* ctx, void* stream) {
    if (!ctx) return BEM_ERR_INVALID;
    cudaStream_t s = (cudaStream_t)stream;
    int32_t e = 0;
    if (int rc = bem_check_cuda(ctx, cudaMemcpyAsync(&e, ctx->flags + 4, sizeof(int32_t), cudaMemcpyDeviceToHost, s),
                                "factor status"))
        return rc;
    if (int rc = bem_check_cuda(ctx, cudaStreamSynchronize(s), "factor status")) return rc;
    return bem_take_factor_error(ctx, e, s);
}

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

template <typename T, bool C>
int tile_inverses_t(bem_ctx* ctx, const T* A, int64_t n, int64_t lda, CE<T>* dinv, cudaStream_t s) {
    const size_t ismem = inv_smem_bytes(sizeof(CE<T>));
    cudaFuncSetAttribute(tile_inv_kernel<T, C>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ismem);
    tile_inv_kernel<T, C><<<(unsigned)((n + LU_T - 1) / LU_T), 256, ismem, s>>>(A, lda, (int)n, dinv);
    ctx->launches++;
    return bem_check_cuda(ctx, cudaGetLastError(), "tile_inv_kernel");
}

int bem_tile_inverses(bem_ctx* ctx, int dtype, const void* A, int64_t n, int64_t lda, void* dinv, cudaStream_t s) {
    switch (dtype) {
        case BEM_F64: return tile_inverses_t<double, false>(ctx, (const double*)A, n, lda, (CE<double>*)dinv, s);
        case BEM_C128: return tile_inverses_t<double, true>(ctx, (const double*)A, n, lda, (CE<double>*)dinv, s);
        case BEM_F32: return tile_inverses_t<float, false>(ctx, (const float*)A, n, lda, (CE<float>*)dinv, s);
        case BEM_C64: return tile_inverses_t<float, true>(ctx, (const float*)A, n, lda, (CE<float>*)dinv, s);
        default: return bem_fail(ctx, BEM_ERR_INVALID, "tile inverses: unknown dtype");
    }
}

int bem_tiled_precond_async(bem_ctx* ctx, int dtype, const void* LU, int64_t n, int64_t lda, const int32_t* piv,
                            const void* dinv, const double* r, double** out, const int* skip, cudaStream_t s) {
    switch (dtype) {
        case BEM_F64: return precond_t<double, false>(ctx, (const double*)LU, n, lda, piv, (const CE<double>*)dinv, r, out, skip, s);
        case BEM_C128: return precond_t<double, true>(ctx, (const double*)LU, n, lda, piv, (const CE<double>*)dinv, r, out, skip, s);
        case BEM_F32: return precond_t<float, false>(ctx, (const float*)LU, n, lda, piv, (const CE<float>*)dinv, r, out, skip, s);
        case BEM_C64: return precond_t<float, true>(ctx, (const float*)LU, n, lda, piv, (const CE<float>*)dinv, r, out, skip, s);
        default: return bem_fail(ctx, BEM_ERR_INVALID, "tiled precond: unknown dtype");
    }
}

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
    tile_piv_to_perm_kernel<<<(unsigned)((nbk + 127) / 128), 128, 0, s>>>(piv, perm, (int)n);
    permute_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(b, perm, x, (int)n, W);
    if (cudaGetLastError() != cudaSuccess) return BEM_ERR_CUDA;
    // the array keeps the previous call's contents: the flags and the error
    // word must start at zero
    if (cudaMemsetAsync(flags, 0, sizeof(int) * 2 * nbk, s) != cudaSuccess ||
        cudaMemsetAsync(err, 0, sizeof(int32_t), s) != cudaSuccess) {
        cudaGetLastError();
        return BEM_ERR_CUDA;
    }
    const size_t ssmem = solve_smem_bytes(sizeof(CE<T>));
    if (cudaFuncSetAttribute(tile_solve_kernel<T, C>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ssmem) !=
        cudaSuccess) {
        cudaGetLastError();
        return BEM_ERR_CUDA;
    }
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, tile_solve_kernel<T, C>, 256, ssmem);
    int P = std::max(1, std::min(nbk, std::min(per_sm * sms, sms)));
    int ni = (int)n, epoch = 1;
    const int* no_skip = nullptr;
    void* args[] = {(void*)&LU, &lda, &ni, (void*)&dinv, &x, &flags, &epoch, &err, (void*)&no_skip};
    if (cudaLaunchCooperativeKernel((const void*)tile_solve_kernel<T, C>, P, 256, args, ssmem, s) != cudaSuccess) {
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
