// Dense LU with partial pivoting, triangular solves, GEMV and mixed-precision
// iterative refinement (replaces torch.linalg.solve at
// src/managers/BEM_manager.py:1056; no cuSOLVER).
//
// Factorisation (right-looking, block width LU_NB):
//   panel   : one cooperative launch per column panel; each CTA owns a slice
//             of the panel's rows; per column one grid barrier publishes every
//             CTA's pivot candidate, after which all CTAs agree on the pivot,
//             swap it in and apply the rank-1 update to their rows.
//   laswp   : the panel's row swaps applied to the columns outside the panel.
//   trsm    : U12 = L11^-1 A12, L11 staged in shared memory.
//   update  : A22 -= L21 U12 (bem_gemm.cu: FP64 SIMT tiles for the plain path,
//             tcgen05 TF32 tensor-core tiles for the FP32 factor).
// Every device-side wait (grid barriers) is bounded; a timeout sets a flag and
// the host call returns BEM_ERR_TIMEOUT.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <complex>
#include <functional>
#include <vector>

#include <cmath>
#include <vector>

#include "bem_gemm.cuh"
#include "bem_internal.cuh"

namespace {

constexpr int LU_NB = 64;
constexpr unsigned SPIN_CAP = 1u << 22;  // x ~256 ns sleep ~ 1 s

struct GridBar {
    unsigned count;
    unsigned gen;
};

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(unsigned* p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned atom_add_acq_rel(unsigned* p, unsigned v) {
    unsigned old;
    asm volatile("atom.add.acq_rel.gpu.global.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}

// Bounded software grid barrier (the launch is cooperative, so all CTAs are
// co-resident).  The last CTA to arrive resets the counter and releases the
// generation word; the others poll it with acquire loads, first without and
// then with a short sleep.  Returns false when the wait hit its cap (flag set)
// or another CTA reported a failure.
__device__ __forceinline__ bool grid_barrier(GridBar* bar, unsigned nblocks, int32_t* flag) {
    __syncthreads();
    __shared__ int s_ok;
    if (threadIdx.x == 0) {
        int ok = 1;
        const unsigned g = ld_acquire(&bar->gen);
        __threadfence();
        const unsigned arrived = atom_add_acq_rel(&bar->count, 1u);
        if (arrived == nblocks - 1) {
            bar->count = 0u;
            st_release(&bar->gen, g + 1u);
        } else {
            unsigned it = 0;
            while (ld_acquire(&bar->gen) == g) {
                if (++it > SPIN_CAP) {
                    atomicExch(flag, BEM_ERR_TIMEOUT);
                    ok = 0;
                    break;
                }
                if ((it & 63u) == 0u && *(volatile int32_t*)flag != 0) {
                    ok = 0;
                    break;
                }
                if (it > 4096u) __nanosleep(64);
            }
        }
        __threadfence();
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

template <typename T, bool C>
struct El {
    T re, im;
};

template <typename T, bool C>
__device__ __forceinline__ El<T, C> ld(const T* A, int64_t i) {
    El<T, C> e;
    if (C) {
        e.re = A[2 * i];
        e.im = A[2 * i + 1];
    } else {
        e.re = A[i];
        e.im = T(0);
    }
    return e;
}
template <typename T, bool C>
__device__ __forceinline__ void st(T* A, int64_t i, El<T, C> e) {
    if (C) {
        A[2 * i] = e.re;
        A[2 * i + 1] = e.im;
    } else {
        A[i] = e.re;
    }
}
template <typename T, bool C>
__device__ __forceinline__ T mag1(El<T, C> e) {
    return C ? fabs(e.re) + fabs(e.im) : fabs(e.re);
}
template <typename T, bool C>
__device__ __forceinline__ El<T, C> ld_volatile(const El<T, C>* p) {
    const volatile T* v = reinterpret_cast<const volatile T*>(p);
    El<T, C> e;
    e.re = v[0];
    e.im = C ? v[1] : T(0);
    return e;
}

struct PivSlot {
    double val;
    int idx;
    int pad;
};

// ----------------------------------------------------------------------------
// panel factorisation (cooperative)
//
// Each CTA owns a contiguous slice of the panel's rows, held in shared memory
// for the whole panel (SMEM_ROWS) or read from global memory when the slice
// does not fit.  Per column j: every CTA publishes its best pivot candidate
// (value, row) and a copy of that row, and the owner of row jj publishes row
// jj, into buffers indexed by the parity of j; one grid barrier; every CTA
// reads the winner's row and row jj from those buffers (never from another
// CTA's slice), swaps, and updates its own rows.  Double buffering by parity
// keeps a CTA that is one column ahead from overwriting buffers still read.
// ----------------------------------------------------------------------------
constexpr int PANEL_MAXB = 256;

template <typename T, bool C, bool SMEM_ROWS>
__global__ void __launch_bounds__(256) lu_panel_kernel(T* A, int64_t lda, int n, int k0, int nb, int chunk,
                                                       int32_t* piv, int32_t* info, GridBar* bar, PivSlot* slots,
                                                       El<T, C>* rowbuf, int32_t* flag) {
    using E = El<T, C>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    E* srows = reinterpret_cast<E*>(smem_raw);  // [chunk][nb] when SMEM_ROWS
    const unsigned nblk = gridDim.x;
    const int r_begin = k0 + blockIdx.x * chunk;
    const int r_end = min(n, r_begin + chunk);
    __shared__ E s_prow[LU_NB];
    __shared__ E s_jrow[LU_NB];
    __shared__ double s_red_v[8];
    __shared__ int s_red_i[8];
    __shared__ int s_red_b[8];
    __shared__ int s_best_idx;
    __shared__ int s_p, s_pb;
    __shared__ double s_pv;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nwarps = blockDim.x >> 5;

    auto row_ptr_g = [&](int r) { return A + (C ? 2 : 1) * ((int64_t)r * lda + k0); };
    auto get = [&](int r, int c) -> E {
        if (SMEM_ROWS) return srows[(r - r_begin) * nb + c];
        return ld<T, C>(row_ptr_g(r), c);
    };
    auto put = [&](int r, int c, E v) {
        if (SMEM_ROWS)
            srows[(r - r_begin) * nb + c] = v;
        else
            st<T, C>(row_ptr_g(r), c, v);
    };
    if (SMEM_ROWS) {
        for (int e = threadIdx.x; e < (r_end - r_begin) * nb; e += blockDim.x) {
            int r = e / nb, c = e - r * nb;
            srows[e] = ld<T, C>(row_ptr_g(r_begin + r), c);
        }
        __syncthreads();
    }

    for (int j = 0; j < nb; ++j) {
        const int jj = k0 + j;
        const int par = j & 1;
        PivSlot* slot = slots + par * PANEL_MAXB;
        E* rb = rowbuf + (size_t)par * (PANEL_MAXB + 1) * LU_NB;
        // 1. local pivot candidate
        double best = -1.0;
        int bidx = 0x7fffffff;
        for (int r = max(r_begin, jj) + threadIdx.x; r < r_end; r += blockDim.x) {
            double v = (double)mag1<T, C>(get(r, j));
            if (v > best || (v == best && r < bidx)) {
                best = v;
                bidx = r;
            }
        }
        for (int o = 16; o > 0; o >>= 1) {
            double ov = __shfl_xor_sync(0xffffffffu, best, o);
            int oi = __shfl_xor_sync(0xffffffffu, bidx, o);
            if (ov > best || (ov == best && oi < bidx)) {
                best = ov;
                bidx = oi;
            }
        }
        if (lane == 0) {
            s_red_v[wid] = best;
            s_red_i[wid] = bidx;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int w = 1; w < nwarps; ++w)
                if (s_red_v[w] > best || (s_red_v[w] == best && s_red_i[w] < bidx)) {
                    best = s_red_v[w];
                    bidx = s_red_i[w];
                }
            slot[blockIdx.x].val = best;
            slot[blockIdx.x].idx = bidx;
            s_best_idx = bidx;
        }
        __syncthreads();
        const int cand = s_best_idx;
        if (cand >= r_begin && cand < r_end)
            for (int c = threadIdx.x; c < nb; c += blockDim.x) rb[(size_t)blockIdx.x * LU_NB + c] = get(cand, c);
        if (jj >= r_begin && jj < r_end)
            for (int c = threadIdx.x; c < nb; c += blockDim.x) rb[(size_t)PANEL_MAXB * LU_NB + c] = get(jj, c);
        // 2. publish
        if (!grid_barrier(bar, nblk, flag)) return;
        // 3. global pivot, slots read in parallel
        {
            double bv = -1.0;
            int bi = 0x7fffffff, bb = -1;
            for (unsigned b = threadIdx.x; b < nblk; b += blockDim.x) {
                double v = ((volatile PivSlot*)slot)[b].val;
                int i = ((volatile PivSlot*)slot)[b].idx;
                if (v > bv || (v == bv && i < bi)) {
                    bv = v;
                    bi = i;
                    bb = (int)b;
                }
            }
            for (int o = 16; o > 0; o >>= 1) {
                double ov = __shfl_xor_sync(0xffffffffu, bv, o);
                int oi = __shfl_xor_sync(0xffffffffu, bi, o);
                int ob = __shfl_xor_sync(0xffffffffu, bb, o);
                if (ov > bv || (ov == bv && oi < bi)) {
                    bv = ov;
                    bi = oi;
                    bb = ob;
                }
            }
            if (lane == 0) {
                s_red_v[wid] = bv;
                s_red_i[wid] = bi;
                s_red_b[wid] = bb;
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                for (int w = 1; w < nwarps; ++w)
                    if (s_red_v[w] > bv || (s_red_v[w] == bv && s_red_i[w] < bi)) {
                        bv = s_red_v[w];
                        bi = s_red_i[w];
                        bb = s_red_b[w];
                    }
                if (bb < 0 || bi < jj || bi >= n) {  // no candidate: keep the diagonal
                    bi = jj;
                    bb = -1;
                    bv = 0.0;
                }
                s_p = bi;
                s_pb = bb;
                s_pv = bv;
                if (blockIdx.x == 0) {
                    piv[jj] = bi;
                    if (!(bv > 0.0) && *info == 0) *info = jj + 1;
                }
            }
            __syncthreads();
        }
        const int p = s_p;
        for (int c = threadIdx.x; c < nb; c += blockDim.x) {
            E ej = ld_volatile<T, C>(rb + (size_t)PANEL_MAXB * LU_NB + c);
            s_jrow[c] = ej;
            s_prow[c] = s_pb >= 0 ? ld_volatile<T, C>(rb + (size_t)s_pb * LU_NB + c) : ej;
        }
        __syncthreads();
        // 4. swap rows jj and p (panel columns)
        if (p != jj) {
            if (jj >= r_begin && jj < r_end)
                for (int c = threadIdx.x; c < nb; c += blockDim.x) put(jj, c, s_prow[c]);
            if (p >= r_begin && p < r_end)
                for (int c = threadIdx.x; c < nb; c += blockDim.x) put(p, c, s_jrow[c]);
        }
        __syncthreads();
        // 5. scale column jj below the diagonal, rank-1 update of the panel
        const E pv = s_prow[j];
        const bool nonzero = s_pv > 0.0;
        E inv;
        if (C) {
            T d = pv.re * pv.re + pv.im * pv.im;
            inv.re = nonzero ? pv.re / d : T(0);
            inv.im = nonzero ? -pv.im / d : T(0);
        } else {
            inv.re = nonzero ? T(1) / pv.re : T(0);
            inv.im = T(0);
        }
        for (int r = max(r_begin, jj + 1) + wid; r < r_end; r += nwarps) {
            E a = get(r, j);
            E l;
            l.re = a.re * inv.re - (C ? a.im * inv.im : T(0));
            l.im = C ? a.re * inv.im + a.im * inv.re : T(0);
            for (int c = j + 1 + lane; c < nb; c += 32) {
                E v = get(r, c);
                E u = s_prow[c];
                v.re -= l.re * u.re - (C ? l.im * u.im : T(0));
                if (C) v.im -= l.re * u.im + l.im * u.re;
                put(r, c, v);
            }
            __syncwarp();
            if (lane == 0) put(r, j, l);
        }
        __syncthreads();
    }
    if (SMEM_ROWS) {
        for (int e = threadIdx.x; e < (r_end - r_begin) * nb; e += blockDim.x) {
            int r = e / nb, c = e - r * nb;
            st<T, C>(row_ptr_g(r_begin + r), c, srows[e]);
        }
    }
}

// row swaps of one panel applied to the columns outside it
template <typename T, bool C>
__global__ void laswp_kernel(T* A, int64_t lda, int n, int k0, int nb, const int32_t* piv) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n || (c >= k0 && c < k0 + nb)) return;
    for (int j = 0; j < nb; ++j) {
        int r1 = k0 + j, r2 = piv[k0 + j];
        if (r1 == r2) continue;
        El<T, C> a = ld<T, C>(A, (int64_t)r1 * lda + c);
        El<T, C> b = ld<T, C>(A, (int64_t)r2 * lda + c);
        st<T, C>(A, (int64_t)r1 * lda + c, b);
        st<T, C>(A, (int64_t)r2 * lda + c, a);
    }
}

// U12 = L11^{-1} A12 (unit lower L11 = rows/cols k0..k0+nb): L11 and a tile
// of TRSM_COLS columns of A12 are staged in shared memory; one thread per
// column runs the forward substitution out of shared memory.
constexpr int TRSM_COLS = 64;

template <typename T, bool C>
__global__ void __launch_bounds__(TRSM_COLS) trsm_kernel(T* A, int64_t lda, int n, int k0, int nb) {
    using E = El<T, C>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    E* L = reinterpret_cast<E*>(smem_raw);  // [nb][nb]
    E* X = L + nb * nb;                     // [nb][TRSM_COLS]
    const int c0 = k0 + nb + blockIdx.x * TRSM_COLS;
    const int ncol = min(TRSM_COLS, n - c0);
    for (int idx = threadIdx.x; idx < nb * nb; idx += blockDim.x) {
        int r = idx / nb, c = idx - r * nb;
        L[idx] = ld<T, C>(A, (int64_t)(k0 + r) * lda + k0 + c);
    }
    for (int idx = threadIdx.x; idx < nb * TRSM_COLS; idx += blockDim.x) {
        int r = idx / TRSM_COLS, c = idx - r * TRSM_COLS;
        X[idx] = c < ncol ? ld<T, C>(A, (int64_t)(k0 + r) * lda + c0 + c) : E{T(0), T(0)};
    }
    __syncthreads();
    const int c = threadIdx.x;
    for (int r = 1; r < nb; ++r) {
        E acc = X[r * TRSM_COLS + c];
        for (int q = 0; q < r; ++q) {
            E l = L[r * nb + q];
            E x = X[q * TRSM_COLS + c];
            acc.re -= l.re * x.re - (C ? l.im * x.im : T(0));
            if (C) acc.im -= l.re * x.im + l.im * x.re;
        }
        X[r * TRSM_COLS + c] = acc;
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < nb * TRSM_COLS; idx += blockDim.x) {
        int r = idx / TRSM_COLS, cc = idx - r * TRSM_COLS;
        if (cc < ncol) st<T, C>(A, (int64_t)(k0 + r) * lda + c0 + cc, X[idx]);
    }
}

// perm[i] = original row that ends up at row i after the LAPACK swap sequence
// (sequential by nature; run in shared memory by one thread)
__global__ void piv_to_perm_kernel(const int32_t* piv, int32_t* perm, int n) {
    extern __shared__ int32_t sp[];
    for (int i = threadIdx.x; i < n; i += blockDim.x) sp[i] = i;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int i = 0; i < n; ++i) {
            int p = piv[i];
            if (p != i && p >= 0 && p < n) {
                int t = sp[i];
                sp[i] = sp[p];
                sp[p] = t;
            }
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) perm[i] = sp[i];
}

// ----------------------------------------------------------------------------
// triangular solves: x = U^{-1} L^{-1} P b, one cooperative launch.
// Vectors are FP64 (real or complex) whatever the factor storage type.
// ----------------------------------------------------------------------------
constexpr int TRSV_NB = 64;

template <typename T, bool C>
__global__ void __launch_bounds__(256) lu_solve_kernel(const T* LU, int64_t lda, int n, const int32_t* perm,
                                                        const double* b, double* x, double* tmp, int64_t nrhs,
                                                        int64_t ldb, GridBar* bar, int32_t* flag) {
    using E = El<T, C>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    E* sL = reinterpret_cast<E*>(smem_raw);                                  // [TRSV_NB][TRSV_NB]
    double* sx = reinterpret_cast<double*>(sL + TRSV_NB * TRSV_NB);          // [TRSV_NB][8][2]
    const unsigned nblk = gridDim.x;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int gwarp = blockIdx.x * (blockDim.x >> 5) + wid;
    const int nwarp_total = nblk * (blockDim.x >> 5);
    const int W = C ? 2 : 1;
    // y = P b  (x is the work vector)
    for (int64_t idx = blockIdx.x * blockDim.x + threadIdx.x; idx < (int64_t)n * nrhs;
         idx += (int64_t)nblk * blockDim.x) {
        int i = (int)(idx / nrhs), c = (int)(idx % nrhs);
        int src = perm[i];
        for (int w = 0; w < W; ++w) x[W * ((int64_t)i * ldb + c) + w] = b[W * ((int64_t)src * ldb + c) + w];
    }
    if (!grid_barrier(bar, nblk, flag)) return;
    const int nblocks_r = (n + TRSV_NB - 1) / TRSV_NB;

    // Diagonal block solve on CTA 0: the block of LU and the x segment are
    // staged in shared memory, one warp per right-hand side.
    auto diag_solve = [&](int r0, int r1, bool lower) {
        const int m = r1 - r0;
        for (int e = threadIdx.x; e < m * m; e += blockDim.x) {
            int r = e / m, q = e - r * m;
            sL[r * TRSV_NB + q] = ld<T, C>(LU, (int64_t)(r0 + r) * lda + r0 + q);
        }
        for (int e = threadIdx.x; e < m * nrhs; e += blockDim.x) {
            int r = e / (int)nrhs, c = e - r * (int)nrhs;
            sx[(r * 8 + c) * 2] = __ldcg(&x[W * ((int64_t)(r0 + r) * ldb + c)]);
            sx[(r * 8 + c) * 2 + 1] = C ? __ldcg(&x[W * ((int64_t)(r0 + r) * ldb + c) + 1]) : 0.0;
        }
        __syncthreads();
        if (wid < nrhs) {
            const int c = wid;
            for (int t = 0; t < m; ++t) {
                const int r = lower ? t : m - 1 - t;
                double sr = 0.0, si = 0.0;
                const int q0 = lower ? 0 : r + 1, q1 = lower ? r : m;
                for (int q = q0 + lane; q < q1; q += 32) {
                    E l = sL[r * TRSV_NB + q];
                    double xr = sx[(q * 8 + c) * 2], xi = sx[(q * 8 + c) * 2 + 1];
                    sr += (double)l.re * xr - (C ? (double)l.im * xi : 0.0);
                    if (C) si += (double)l.re * xi + (double)l.im * xr;
                }
                for (int o = 16; o > 0; o >>= 1) {
                    sr += __shfl_xor_sync(0xffffffffu, sr, o);
                    if (C) si += __shfl_xor_sync(0xffffffffu, si, o);
                }
                if (lane == 0) {
                    double vr = sx[(r * 8 + c) * 2] - sr, vi = sx[(r * 8 + c) * 2 + 1] - si;
                    if (!lower) {
                        E d = sL[r * TRSV_NB + r];
                        if (C) {
                            double dr = d.re, di = d.im, den = dr * dr + di * di;
                            double tr = (vr * dr + vi * di) / den;
                            vi = (vi * dr - vr * di) / den;
                            vr = tr;
                        } else {
                            vr = vr / (double)d.re;
                        }
                    }
                    sx[(r * 8 + c) * 2] = vr;
                    sx[(r * 8 + c) * 2 + 1] = vi;
                }
                __syncwarp();
            }
        }
        __syncthreads();
        for (int e = threadIdx.x; e < m * nrhs; e += blockDim.x) {
            int r = e / (int)nrhs, c = e - r * (int)nrhs;
            x[W * ((int64_t)(r0 + r) * ldb + c)] = sx[(r * 8 + c) * 2];
            if (C) x[W * ((int64_t)(r0 + r) * ldb + c) + 1] = sx[(r * 8 + c) * 2 + 1];
        }
    };
    // rows [i0, i1) (distributed over all warps): x[i] -= LU[i, r0:r1] x[r0:r1]
    auto update = [&](int i0, int i1, int r0, int r1) {
        for (int i = i0 + gwarp; i < i1; i += nwarp_total) {
            for (int c = 0; c < nrhs; ++c) {
                double sr = 0.0, si = 0.0;
                for (int q = r0 + lane; q < r1; q += 32) {
                    E l = ld<T, C>(LU, (int64_t)i * lda + q);
                    double xr = __ldcg(&x[W * ((int64_t)q * ldb + c)]);
                    double xi = C ? __ldcg(&x[W * ((int64_t)q * ldb + c) + 1]) : 0.0;
                    sr += (double)l.re * xr - (C ? (double)l.im * xi : 0.0);
                    if (C) si += (double)l.re * xi + (double)l.im * xr;
                }
                for (int o = 16; o > 0; o >>= 1) {
                    sr += __shfl_xor_sync(0xffffffffu, sr, o);
                    if (C) si += __shfl_xor_sync(0xffffffffu, si, o);
                }
                if (lane == 0) {
                    x[W * ((int64_t)i * ldb + c)] = __ldcg(&x[W * ((int64_t)i * ldb + c)]) - sr;
                    if (C) x[W * ((int64_t)i * ldb + c) + 1] = __ldcg(&x[W * ((int64_t)i * ldb + c) + 1]) - si;
                }
            }
        }
    };
    // forward: L y = P b (unit diagonal)
    for (int kb = 0; kb < nblocks_r; ++kb) {
        const int r0 = kb * TRSV_NB, r1 = min(n, r0 + TRSV_NB);
        if (blockIdx.x == 0) diag_solve(r0, r1, true);
        if (!grid_barrier(bar, nblk, flag)) return;
        if (r1 < n) {
            update(r1, n, r0, r1);
            if (!grid_barrier(bar, nblk, flag)) return;
        }
    }
    // backward: U x = y
    for (int kb = nblocks_r - 1; kb >= 0; --kb) {
        const int r0 = kb * TRSV_NB, r1 = min(n, r0 + TRSV_NB);
        if (blockIdx.x == 0) diag_solve(r0, r1, false);
        if (!grid_barrier(bar, nblk, flag)) return;
        if (r0 > 0) {
            update(0, r0, r0, r1);
            if (!grid_barrier(bar, nblk, flag)) return;
        }
    }
    (void)tmp;
}

// y = alpha A x + beta y, A stored as T (real/complex), x/y FP64
template <typename T, bool C>
__global__ void __launch_bounds__(256) gemv_kernel(const T* A, int64_t m, int64_t n, int64_t lda, const double* x,
                                                    double* y, double alpha, double beta) {
    const int lane = threadIdx.x & 31;
    const int64_t row = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (row >= m) return;
    double sr = 0.0, si = 0.0;
    const T* a = A + (C ? 2 : 1) * row * lda;
    for (int64_t q = lane; q < n; q += 32) {
        El<T, C> e = ld<T, C>(a, q);
        double xr = C ? x[2 * q] : x[q], xi = C ? x[2 * q + 1] : 0.0;
        sr += (double)e.re * xr - (C ? (double)e.im * xi : 0.0);
        if (C) si += (double)e.re * xi + (double)e.im * xr;
    }
    for (int o = 16; o > 0; o >>= 1) {
        sr += __shfl_xor_sync(0xffffffffu, sr, o);
        if (C) si += __shfl_xor_sync(0xffffffffu, si, o);
    }
    if (lane == 0) {
        if (C) {
            double yr = beta == 0.0 ? 0.0 : beta * y[2 * row];
            double yi = beta == 0.0 ? 0.0 : beta * y[2 * row + 1];
            y[2 * row] = yr + alpha * sr;
            y[2 * row + 1] = yi + alpha * si;
        } else {
            double yr = beta == 0.0 ? 0.0 : beta * y[row];
            y[row] = yr + alpha * sr;
        }
    }
}

__global__ void sumsq_kernel(const double* v, int64_t n, double* out) {
    __shared__ double s[8];
    double acc = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        acc += v[i] * v[i];
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += s[w];
        atomicAdd(out, t);
    }
}

__global__ void axpy_kernel(double* y, const double* x, int64_t n, double a) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) y[i] += a * x[i];
}

// ---- asynchronous refinement: state and step kernels ----------------------
// Every kernel of an iteration returns at once when `done` is set, so the
// host can queue several iterations and synchronise once.
struct RefState {
    double bn2;    // ||b||^2
    double rn2;    // ||r||^2 of the current iteration (accumulated)
    double prev2;  // ||r||^2 of the previous iteration
    double rel2;   // last ||r||^2 / ||b||^2
    int done;      // 0 running, 1 converged, 2 stagnated, 3 maxit
    int it;        // iterations completed
};

__global__ void ref_init_kernel(RefState* st) {
    st->bn2 = st->rn2 = st->prev2 = st->rel2 = 0.0;
    st->done = 0;
    st->it = 0;
}

__global__ void ref_start_kernel(RefState* st) {
    st->prev2 = st->bn2;
    if (st->bn2 == 0.0) st->done = 1;  // b = 0: x = 0 is exact
}

__global__ void ref_axpy_kernel(double* y, const double* x, int64_t n, const RefState* st) {
    if (st->done) return;
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) y[i] += x[i];
}

__global__ void ref_sumsq_kernel(const double* v, int64_t n, RefState* st) {
    if (st->done) return;
    __shared__ double s[8];
    double acc = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        acc += v[i] * v[i];
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += s[w];
        atomicAdd(&st->rn2, t);
    }
}

// r = b - A x, one warp per row (the FP64 residual of the refinement)
template <typename T, bool C>
__global__ void __launch_bounds__(256) ref_residual_kernel(const T* A, int64_t n, int64_t lda, const double* x,
                                                            const double* b, double* r, const RefState* st) {
    if (st->done) return;
    const int lane = threadIdx.x & 31;
    const int64_t row = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (row >= n) return;
    double sr = 0.0, si = 0.0;
    const T* a = A + (C ? 2 : 1) * row * lda;
    for (int64_t q = lane; q < n; q += 32) {
        El<T, C> e = ld<T, C>(a, q);
        double xr = C ? x[2 * q] : x[q], xi = C ? x[2 * q + 1] : 0.0;
        sr += (double)e.re * xr - (C ? (double)e.im * xi : 0.0);
        if (C) si += (double)e.re * xi + (double)e.im * xr;
    }
    for (int o = 16; o > 0; o >>= 1) {
        sr += __shfl_xor_sync(0xffffffffu, sr, o);
        if (C) si += __shfl_xor_sync(0xffffffffu, si, o);
    }
    if (lane == 0) {
        if (C) {
            r[2 * row] = b[2 * row] - sr;
            r[2 * row + 1] = b[2 * row + 1] - si;
        } else {
            r[row] = b[row] - sr;
        }
    }
}

// convergence test of one iteration: relative residual <= tol (done = 1),
// stagnation after three iterations (residual above half the previous, 2),
// iteration cap (3)
__global__ void ref_decide_kernel(RefState* st, double tol2, int maxit) {
    if (st->done) return;
    st->it += 1;
    const double rn2 = st->rn2;
    st->rn2 = 0.0;
    st->rel2 = rn2 / st->bn2;
    if (rn2 <= tol2 * st->bn2)
        st->done = 1;
    else if (st->it >= 3 && rn2 > 0.25 * st->prev2)
        st->done = 2;
    else if (st->it >= maxit)
        st->done = 3;
    st->prev2 = rn2;
}

struct LinWs {
    GridBar* bar;
    PivSlot* slots;  // [2][PANEL_MAXB]
    void* rowbuf;    // [2][PANEL_MAXB+1][LU_NB] panel-row copies (16 B per element)
    int32_t* perm;
    double* vec;     // scratch vectors for the triangular solves
};

int linws(bem_ctx* ctx, int64_t n, int64_t nvec_doubles, LinWs* w) {
    size_t off_bar = 0;
    size_t off_slots = 256;
    size_t off_rows = off_slots + sizeof(PivSlot) * 2 * PANEL_MAXB;
    size_t off_perm = off_rows + 16 * (size_t)2 * (PANEL_MAXB + 1) * LU_NB;
    size_t off_vec = (off_perm + sizeof(int32_t) * (size_t)n + 255) & ~size_t(255);
    size_t total = off_vec + sizeof(double) * (size_t)nvec_doubles;
    if (int rc = bem_ws_reserve(ctx, total)) return rc;
    char* base = (char*)ctx->ws;
    w->bar = (GridBar*)(base + off_bar);
    w->slots = (PivSlot*)(base + off_slots);
    w->rowbuf = (void*)(base + off_rows);
    w->perm = (int32_t*)(base + off_perm);
    w->vec = (double*)(base + off_vec);
    return BEM_OK;
}

int coop_blocks(bem_ctx* ctx, const void* fn, int threads, size_t smem, int want) {
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem);
    int maxb = per_sm * ctx->num_sms;
    if (maxb < 1) return 0;
    return std::max(1, std::min(want, std::min(maxb, ctx->num_sms)));
}

int check_flag(bem_ctx* ctx, cudaStream_t s, const char* what) {
    int32_t f = 0;
    if (int rc = bem_check_cuda(ctx, cudaMemcpyAsync(&f, ctx->flags + 2, sizeof(int32_t), cudaMemcpyDeviceToHost, s),
                                "flag readback"))
        return rc;
    if (int rc = bem_check_cuda(ctx, cudaStreamSynchronize(s), what)) return rc;
    if (f != 0) {
        cudaMemsetAsync(ctx->flags + 2, 0, sizeof(int32_t), s);
        return bem_fail(ctx, BEM_ERR_TIMEOUT, std::string(what) + ": device wait hit its iteration cap");
    }
    return BEM_OK;
}

template <typename T, bool C>
int lu_factor_t(bem_ctx* ctx, T* A, int64_t n, int64_t lda, int32_t* piv, int32_t* info, cudaStream_t s) {
    LinWs w;
    if (int rc = linws(ctx, n, 0, &w)) return rc;
    cudaMemsetAsync(w.bar, 0, sizeof(GridBar), s);
    cudaMemsetAsync(info, 0, sizeof(int32_t), s);
    cudaMemsetAsync(ctx->flags + 2, 0, sizeof(int32_t), s);
    const int threads = 256;
    int32_t* flag = ctx->flags + 2;
    // CTAs of the panel: at most one per SM and at most PANEL_MAXB; each keeps
    // its row slice in shared memory when it fits in PANEL_SMEM bytes
    const size_t PANEL_SMEM = 200 * 1024;
    const int maxb = std::min(PANEL_MAXB, ctx->num_sms);
    const size_t smem_full = sizeof(El<T, C>) * (size_t)((n + maxb - 1) / maxb) * LU_NB;
    const bool use_smem = smem_full <= PANEL_SMEM;
    const void* pk = use_smem ? (const void*)lu_panel_kernel<T, C, true> : (const void*)lu_panel_kernel<T, C, false>;
    if (use_smem)
        cudaFuncSetAttribute(lu_panel_kernel<T, C, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)PANEL_SMEM);
    int nblk = std::min(maxb, coop_blocks(ctx, pk, threads, use_smem ? smem_full : 0, maxb));
    if (nblk < 1) return bem_fail(ctx, BEM_ERR_CUDA, "lu_panel_kernel cannot be made co-resident");
    if (use_smem && sizeof(El<T, C>) * (size_t)std::max<int64_t>(32, (n + nblk - 1) / nblk) * LU_NB > PANEL_SMEM)
        return bem_fail(ctx, BEM_ERR_CUDA, "lu_panel_kernel: fewer co-resident CTAs than SMs");
    for (int64_t k0 = 0; k0 < n; k0 += LU_NB) {
        int nb = (int)std::min<int64_t>(LU_NB, n - k0);
        int rows = (int)(n - k0);
        int blocks = std::min(nblk, std::max(1, (rows + 31) / 32));
        int chunk = (rows + blocks - 1) / blocks;
        int ni = (int)n, k0i = (int)k0;
        El<T, C>* rb = (El<T, C>*)w.rowbuf;
        size_t smem = use_smem ? sizeof(El<T, C>) * (size_t)chunk * LU_NB : 0;
        void* args[] = {&A, &lda, &ni, &k0i, &nb, &chunk, &piv, &info, &w.bar, &w.slots, &rb, &flag};
        if (int rc = bem_check_cuda(ctx, cudaLaunchCooperativeKernel(pk, blocks, threads, args, smem, s),
                                    "lu_panel_kernel"))
            return rc;
        ctx->launches++;
        laswp_kernel<T, C><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(A, lda, ni, k0i, nb, piv);
        ctx->launches++;
        int64_t rest = n - k0 - nb;
        if (rest > 0) {
            size_t tsmem = sizeof(El<T, C>) * nb * (nb + TRSM_COLS);
            cudaFuncSetAttribute(trsm_kernel<T, C>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tsmem);
            trsm_kernel<T, C><<<(unsigned)((rest + TRSM_COLS - 1) / TRSM_COLS), TRSM_COLS, tsmem, s>>>(A, lda, ni,
                                                                                                   k0i, nb);
            ctx->launches++;
            // A22 -= L21 U12
            T* A22 = A + (C ? 2 : 1) * ((k0 + nb) * lda + k0 + nb);
            const T* L21 = A + (C ? 2 : 1) * ((k0 + nb) * lda + k0);
            const T* U12 = A + (C ? 2 : 1) * (k0 * lda + k0 + nb);
            if (int rc = bem_gemm_update<T, C>(ctx, A22, L21, U12, rest, rest, nb, lda, s)) return rc;
        }
        if (int rc = bem_check_cuda(ctx, cudaGetLastError(), "lu step")) return rc;
    }
    return check_flag(ctx, s, "lu_factor");
}

template <typename T, bool C>
int lu_solve_t(bem_ctx* ctx, const T* LU, int64_t n, int64_t lda, const int32_t* piv, double* b, int64_t nrhs,
               int64_t ldb, cudaStream_t s) {
    if (nrhs < 1 || nrhs > 8) return bem_fail(ctx, BEM_ERR_INVALID, "lu_solve supports 1..8 right-hand sides");
    const int W = C ? 2 : 1;
    LinWs w;
    if (int rc = linws(ctx, n, (int64_t)W * n * ldb, &w)) return rc;
    cudaMemsetAsync(w.bar, 0, sizeof(GridBar), s);
    cudaMemsetAsync(ctx->flags + 2, 0, sizeof(int32_t), s);
    if ((size_t)n * sizeof(int32_t) > 200 * 1024) return bem_fail(ctx, BEM_ERR_INVALID, "lu_solve: n > 51200");
    cudaFuncSetAttribute(piv_to_perm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)(n * sizeof(int32_t)));
    piv_to_perm_kernel<<<1, 256, n * sizeof(int32_t), s>>>(piv, w.perm, (int)n);
    ctx->launches++;
    const int threads = 256;
    const size_t smem = sizeof(El<T, C>) * TRSV_NB * TRSV_NB + sizeof(double) * TRSV_NB * 8 * 2;
    cudaFuncSetAttribute(lu_solve_kernel<T, C>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int nblk = coop_blocks(ctx, (const void*)lu_solve_kernel<T, C>, threads, smem, ctx->num_sms);
    if (nblk < 1) return bem_fail(ctx, BEM_ERR_CUDA, "lu_solve_kernel cannot be made co-resident");
    int ni = (int)n;
    double* xw = w.vec;
    double* tmp = nullptr;
    int32_t* flag = ctx->flags + 2;
    const double* bc = b;
    void* args[] = {(void*)&LU, &lda, &ni, &w.perm, &bc, &xw, &tmp, &nrhs, &ldb, &w.bar, &flag};
    if (int rc = bem_check_cuda(ctx, cudaLaunchCooperativeKernel((const void*)lu_solve_kernel<T, C>, nblk, threads,
                                                                args, smem, s),
                                "lu_solve_kernel"))
        return rc;
    ctx->launches++;
    if (int rc = bem_check_cuda(ctx, cudaMemcpyAsync(b, xw, sizeof(double) * W * n * ldb, cudaMemcpyDeviceToDevice, s),
                                "lu_solve copy"))
        return rc;
    return check_flag(ctx, s, "lu_solve");
}

// Refinement with the tile-pivoted factor, queued in batches of iterations
// with one synchronisation per batch (normally one per call): the convergence
// test runs on the device and the remaining kernels of a finished refinement
// return at once.  Same iterations and stopping rules as the synchronous
// loop of bem_refine_solve.
int refine_async(bem_ctx* ctx, bool C, const void* A_hi, const void* LU_lo, const int32_t* piv, const void* dinv,
                 int64_t n, int64_t lda, const double* b, double* x, double tol, int maxit, int* iters,
                 double* relres, cudaStream_t s) {
    const int W = C ? 2 : 1;
    const int64_t nd = W * n;
    // r (nd) and the state
    double* r = nullptr;
    if (int rc = bem_check_cuda(ctx, cudaMallocAsync((void**)&r, sizeof(double) * nd + 64, s), "refine alloc"))
        return rc;
    RefState* st = reinterpret_cast<RefState*>(r + nd);
    int rc = BEM_OK;
    const unsigned vblocks = (unsigned)((nd + 255) / 256);
    const unsigned sblocks = (unsigned)std::min<int64_t>(ctx->num_sms * 4, (nd + 255) / 256);
    ref_init_kernel<<<1, 1, 0, s>>>(st);
    sumsq_kernel<<<sblocks, 256, 0, s>>>(b, nd, &st->bn2);
    ref_start_kernel<<<1, 1, 0, s>>>(st);
    ctx->launches += 3;
    cudaMemsetAsync(ctx->flags + 3, 0, sizeof(int32_t), s);
    cudaMemsetAsync(x, 0, sizeof(double) * nd, s);
    cudaMemcpyAsync(r, b, sizeof(double) * nd, cudaMemcpyDeviceToDevice, s);
    const int* skip = &st->done;
    RefState h{};
    int32_t flg[2] = {0, 0};
    int queued = 0;
    while (rc == BEM_OK) {
        const int batch = std::min(3, maxit - queued);
        for (int i = 0; i < batch && rc == BEM_OK; ++i) {
            double* d = nullptr;
            rc = bem_tiled_precond_async(ctx, C ? BEM_C64 : BEM_F32, LU_lo, n, lda, piv, dinv, r, &d, skip, s);
            if (rc) break;
            ref_axpy_kernel<<<vblocks, 256, 0, s>>>(x, d, nd, st);
            const unsigned rblocks = (unsigned)((n + 7) / 8);
            if (C)
                ref_residual_kernel<double, true><<<rblocks, 256, 0, s>>>((const double*)A_hi, n, lda, x, b, r, st);
            else
                ref_residual_kernel<double, false><<<rblocks, 256, 0, s>>>((const double*)A_hi, n, lda, x, b, r, st);
            ref_sumsq_kernel<<<sblocks, 256, 0, s>>>(r, nd, st);
            ref_decide_kernel<<<1, 1, 0, s>>>(st, tol * tol, maxit);
            ctx->launches += 4;
            rc = bem_check_cuda(ctx, cudaGetLastError(), "refinement step");
            ++queued;
        }
        if (rc) break;
        cudaMemcpyAsync(&h, st, sizeof(RefState), cudaMemcpyDeviceToHost, s);
        cudaMemcpyAsync(&flg[0], ctx->flags + 3, sizeof(int32_t), cudaMemcpyDeviceToHost, s);
        cudaMemcpyAsync(&flg[1], ctx->flags + 4, sizeof(int32_t), cudaMemcpyDeviceToHost, s);
        rc = bem_check_cuda(ctx, cudaStreamSynchronize(s), "refinement");
        if (rc) break;
        if ((rc = bem_take_factor_error(ctx, flg[1], s))) break;
        if (flg[0] != 0) {
            rc = bem_fail(ctx, BEM_ERR_TIMEOUT, "tiled solve: a ready-flag wait hit its iteration cap");
            break;
        }
        if (h.done != 0 || queued >= maxit) break;
    }
    cudaFreeAsync(r, s);
    if (rc) return rc;
    if (iters) *iters = h.it;
    if (relres) *relres = std::sqrt(h.rel2);
    if (h.done != 1) return bem_fail(ctx, BEM_ERR_NOCONVERGE, "refinement did not reach tol in maxit iterations");
    return BEM_OK;
}

// ---- GMRES: block inner products and updates on FP64 vectors ------------
// out[i] = sum_q conj(V_i[q]) w[q] for the k vectors V_i (stride nd doubles);
// grid (chunks, k), partial sums of a chunk added atomically
template <bool C>
__global__ void gm_dot_kernel(const double* V, int64_t nd, int k, const double* w, double* out) {
    __shared__ double s_re[8], s_im[8];
    const int i = blockIdx.y;
    const double* v = V + (int64_t)i * nd;
    const int W = C ? 2 : 1;
    const int64_t n = nd / W;
    double re = 0.0, im = 0.0;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
        if (C) {
            const double vr = v[2 * q], vi = v[2 * q + 1], wr = w[2 * q], wi = w[2 * q + 1];
            re += vr * wr + vi * wi;
            im += vr * wi - vi * wr;
        } else {
            re += v[q] * w[q];
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        re += __shfl_xor_sync(0xffffffffu, re, o);
        im += __shfl_xor_sync(0xffffffffu, im, o);
    }
    if ((threadIdx.x & 31) == 0) {
        s_re[threadIdx.x >> 5] = re;
        s_im[threadIdx.x >> 5] = im;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double tr = 0.0, ti = 0.0;
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q) {
            tr += s_re[q];
            ti += s_im[q];
        }
        atomicAdd(out + 2 * i, tr);
        if (C) atomicAdd(out + 2 * i + 1, ti);
    }
}

// w[q] -= sum_i V_i[q] h_i (h: k complex values, interleaved; real part only
// when !C)
template <bool C>
__global__ void gm_update_kernel(double* w, const double* V, int64_t nd, int k, const double* h) {
    const int W = C ? 2 : 1;
    const int64_t n = nd / W;
    const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (q >= n) return;
    double ar = 0.0, ai = 0.0;
    for (int i = 0; i < k; ++i) {
        const double* v = V + (int64_t)i * nd;
        const double hr = h[2 * i], hi = h[2 * i + 1];
        if (C) {
            const double vr = v[2 * q], vi = v[2 * q + 1];
            ar += vr * hr - vi * hi;
            ai += vr * hi + vi * hr;
        } else {
            ar += v[q] * hr;
        }
    }
    if (C) {
        w[2 * q] -= ar;
        w[2 * q + 1] -= ai;
    } else {
        w[q] -= ar;
    }
}

__global__ void gm_scale_kernel(double* dst, const double* src, int64_t nd, double a) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < nd) dst[i] = a * src[i];
}

// Restarted GMRES(m) in FP64 on A_hi x = b, right-preconditioned by the
// low-precision factors (tile-pivoted when dinv != NULL, else partial
// pivoting).  Arnoldi with classical Gram-Schmidt applied twice, Givens
// rotations of the Hessenberg matrix on the host.  Each restart starts from
// the true FP64 residual; a restart cycle that no longer halves it ends the
// iteration once the residual is <= accept (its floor is about
// eps * cond(A)).
}  // namespace

int bem_fgmres(bem_ctx* ctx, bool C, int64_t n, const std::function<int(const double*, double*)>& apply_op,
               const std::function<int(double*)>& precond, const double* b, double* x, double tol, int maxit,
               int restart, double accept, int* iters, double* relres, cudaStream_t s) {
    const int W = C ? 2 : 1;
    const int64_t nd = W * n;
    const int m = std::max(1, std::min(restart, 200));
    // V (m+1 vectors), Z (m vectors), w, r, dots (2 (m+1) doubles)
    const size_t doubles = (size_t)(2 * m + 3) * nd + 2 * (m + 2);
    double* buf = nullptr;
    if (int rc = bem_check_cuda(ctx, cudaMallocAsync((void**)&buf, sizeof(double) * doubles, s), "gmres alloc"))
        return rc;
    double* V = buf;
    double* Z = V + (size_t)(m + 1) * nd;
    double* w = Z + (size_t)m * nd;
    double* r = w + nd;
    double* dots = r + nd;
    const unsigned vblocks = (unsigned)((n + 255) / 256);
    const unsigned sblocks = (unsigned)std::min<int64_t>(ctx->num_sms * 4, (nd + 255) / 256);
    const unsigned dchunks = (unsigned)std::min<int64_t>(ctx->num_sms, (n + 255) / 256);
    int rc = BEM_OK;
    auto norm = [&](const double* v, double* out) -> int {
        cudaMemsetAsync(dots, 0, sizeof(double), s);
        sumsq_kernel<<<sblocks, 256, 0, s>>>(v, nd, dots);
        ctx->launches++;
        double h = 0.0;
        if (int e = bem_check_cuda(ctx, cudaMemcpyAsync(&h, dots, sizeof(double), cudaMemcpyDeviceToHost, s),
                                   "gmres norm"))
            return e;
        if (int e = bem_check_cuda(ctx, cudaStreamSynchronize(s), "gmres norm")) return e;
        *out = std::sqrt(h);
        return BEM_OK;
    };
    // r = b - op(x), with w as the scratch of op(x)
    auto residual = [&](double* out_norm) -> int {
        if (int e = apply_op(x, w)) return e;
        if (int e = bem_check_cuda(ctx, cudaMemcpyAsync(r, b, sizeof(double) * nd, cudaMemcpyDeviceToDevice, s),
                                   "r=b"))
            return e;
        axpy_kernel<<<(unsigned)((nd + 255) / 256), 256, 0, s>>>(r, w, nd, -1.0);
        ctx->launches++;
        return norm(r, out_norm);
    };
    using cplx = std::complex<double>;
    double bnorm = 0.0;
    rc = norm(b, &bnorm);
    if (bnorm == 0.0) bnorm = 1.0;
    int its = 0;
    double rel = 0.0, prev = INFINITY;
    bool done = false;
    std::vector<cplx> H((size_t)(m + 1) * m), g(m + 1), cs(m), sn(m), y(m);
    std::vector<double> hbuf(2 * (m + 1));
    while (rc == BEM_OK && its < maxit) {
        double beta = 0.0;
        if ((rc = residual(&beta))) break;
        rel = beta / bnorm;
        if (rel <= tol || (rel > 0.5 * prev && rel <= accept)) {
            done = true;
            break;
        }
        prev = rel;
        const int mm = std::min(m, maxit - its);
        gm_scale_kernel<<<(unsigned)((nd + 255) / 256), 256, 0, s>>>(V, r, nd, 1.0 / beta);
        ctx->launches++;
        std::fill(H.begin(), H.end(), cplx(0.0));
        std::fill(g.begin(), g.end(), cplx(0.0));
        g[0] = beta;
        int jd = 0;
        for (int j = 0; j < mm && rc == BEM_OK; ++j) {
            double* Vj = V + (size_t)j * nd;
            double* Zj = Z + (size_t)j * nd;
            if ((rc = bem_check_cuda(ctx, cudaMemcpyAsync(Zj, Vj, sizeof(double) * nd, cudaMemcpyDeviceToDevice, s),
                                     "z=v")))
                break;
            if ((rc = precond(Zj))) break;
            if ((rc = apply_op(Zj, w))) break;
            for (int pass = 0; pass < 2 && rc == BEM_OK; ++pass) {
                cudaMemsetAsync(dots, 0, sizeof(double) * 2 * (j + 1), s);
                if (C)
                    gm_dot_kernel<true><<<dim3(dchunks, j + 1), 256, 0, s>>>(V, nd, j + 1, w, dots);
                else
                    gm_dot_kernel<false><<<dim3(dchunks, j + 1), 256, 0, s>>>(V, nd, j + 1, w, dots);
                if (C)
                    gm_update_kernel<true><<<vblocks, 256, 0, s>>>(w, V, nd, j + 1, dots);
                else
                    gm_update_kernel<false><<<vblocks, 256, 0, s>>>(w, V, nd, j + 1, dots);
                ctx->launches += 2;
                if ((rc = bem_check_cuda(ctx, cudaMemcpyAsync(hbuf.data(), dots, sizeof(double) * 2 * (j + 1),
                                                              cudaMemcpyDeviceToHost, s), "gmres dots")))
                    break;
                if ((rc = bem_check_cuda(ctx, cudaStreamSynchronize(s), "gmres dots"))) break;
                for (int i = 0; i <= j; ++i) H[(size_t)i * m + j] += cplx(hbuf[2 * i], C ? hbuf[2 * i + 1] : 0.0);
            }
            if (rc) break;
            double hn = 0.0;
            if ((rc = norm(w, &hn))) break;
            ++its;
            jd = j + 1;
            if (hn > 0.0) {
                gm_scale_kernel<<<(unsigned)((nd + 255) / 256), 256, 0, s>>>(V + (size_t)(j + 1) * nd, w, nd,
                                                                              1.0 / hn);
                ctx->launches++;
            }
            // Givens rotations: the earlier ones on column j, a new one for H[j+1][j]
            for (int i = 0; i < j; ++i) {
                const cplx a = H[(size_t)i * m + j], c2 = H[(size_t)(i + 1) * m + j];
                H[(size_t)i * m + j] = std::conj(cs[i]) * a + std::conj(sn[i]) * c2;
                H[(size_t)(i + 1) * m + j] = -sn[i] * a + cs[i] * c2;
            }
            const cplx a = H[(size_t)j * m + j];
            const double den = std::sqrt(std::norm(a) + hn * hn);
            if (den > 0.0) {
                cs[j] = a / den;
                sn[j] = cplx(hn / den, 0.0);
            } else {
                cs[j] = 1.0;
                sn[j] = 0.0;
            }
            H[(size_t)j * m + j] = std::conj(cs[j]) * a + std::conj(sn[j]) * hn;
            g[j + 1] = -sn[j] * g[j];
            g[j] = std::conj(cs[j]) * g[j];
            const double est = std::abs(g[j + 1]) / bnorm;
            if (est <= 0.5 * tol || hn == 0.0) break;
        }
        if (rc) break;
        // y = R^{-1} g, x += Z y
        for (int i = jd - 1; i >= 0; --i) {
            cplx t = g[i];
            for (int q = i + 1; q < jd; ++q) t -= H[(size_t)i * m + q] * y[q];
            const cplx d = H[(size_t)i * m + i];
            y[i] = std::abs(d) > 0.0 ? t / d : cplx(0.0);
        }
        for (int i = 0; i < jd; ++i) {
            hbuf[2 * i] = -y[i].real();
            hbuf[2 * i + 1] = -y[i].imag();
        }
        if ((rc = bem_check_cuda(ctx, cudaMemcpyAsync(dots, hbuf.data(), sizeof(double) * 2 * jd,
                                                      cudaMemcpyHostToDevice, s), "gmres y")))
            break;
        if (C)
            gm_update_kernel<true><<<vblocks, 256, 0, s>>>(x, Z, nd, jd, dots);
        else
            gm_update_kernel<false><<<vblocks, 256, 0, s>>>(x, Z, nd, jd, dots);
        ctx->launches++;
        if ((rc = bem_check_cuda(ctx, cudaStreamSynchronize(s), "gmres update"))) break;
    }
    if (rc == BEM_OK && !done) {
        double rn = 0.0;
        rc = residual(&rn);
        rel = rn / bnorm;
    }
    cudaFreeAsync(buf, s);
    if (rc) return rc;
    if (iters) *iters = its;
    if (relres) *relres = rel;
    if (!done && rel > std::max(tol, accept))
        return bem_fail(ctx, BEM_ERR_NOCONVERGE, "GMRES-IR did not reach tol in maxit iterations");
    return BEM_OK;
}

namespace {

int gmres_run(bem_ctx* ctx, int dtype_hi, const void* A_hi, const void* LU_lo, const int32_t* piv, const void* dinv,
              int64_t n, int64_t lda, const double* b, double* x, double tol, int maxit, int restart, double accept,
              int* iters, double* relres, cudaStream_t s) {
    const bool C = dtype_hi == BEM_C128;
    const int lo_dtype = C ? BEM_C64 : BEM_F32;
    auto op = [&](const double* z, double* w) -> int {
        return bem_gemv(ctx, dtype_hi, A_hi, n, n, lda, z, w, 1.0, 0.0, s);
    };
    auto precond = [&](double* z) -> int {
        return dinv ? bem_lu_solve_tiled(ctx, lo_dtype, LU_lo, n, lda, piv, dinv, z, s)
                    : bem_lu_solve(ctx, lo_dtype, LU_lo, n, lda, piv, z, 1, 1, s);
    };
    return bem_fgmres(ctx, C, n, op, precond, b, x, tol, maxit, restart, accept, iters, relres, s);
}

// ---------------------------------------------------------------------------
// CGS2 column append of a growing orthonormal basis, one cooperative launch
// (bem_cgs2_append).  With x = v:
//   twice: h = Q^H x, x -= Q h, r += h;   r_jj = ||x||, x /= r_jj;
//   twice: h = Q^H x, x -= Q h;           x /= ||x||;
//   Q[:, j] = x, Rt[j, 0..j-1] = r, Rt[j, j] = r_jj.
// CTA b owns the rows [b rb, (b + 1) rb) of x and keeps them in shared memory
// for the whole step.  A projection is two grid barriers: the partial dot
// products of every CTA over its rows (thread c takes column c, so the reads
// of a Q row are coalesced) go to part[b][c]; CTA c % nblk sums column c over
// the CTAs in a fixed order into h[c]; then every CTA forms its rows of Q h
// (one warp per row, lanes over the columns).  Norms: per-CTA partial sums,
// one barrier, the same fixed-order sum in every CTA.  Ten barriers per
// column, no host synchronisation; the sums are deterministic.
// ---------------------------------------------------------------------------
constexpr int CG_THREADS = 256;

template <bool C>
struct Cx {
    double re, im;
};

template <bool C>
__device__ __forceinline__ Cx<C> cx_ld(const double* p, int64_t i) {
    return C ? Cx<C>{p[2 * i], p[2 * i + 1]} : Cx<C>{p[i], 0.0};
}
template <bool C>
__device__ __forceinline__ void cx_st(double* p, int64_t i, Cx<C> v) {
    if (C) {
        p[2 * i] = v.re;
        p[2 * i + 1] = v.im;
    } else {
        p[i] = v.re;
    }
}

__device__ __forceinline__ double block_sum(double v, double* red) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < CG_THREADS / 32; ++w) t += red[w];
    __syncthreads();
    if (threadIdx.x == 0) red[0] = t;
    __syncthreads();
    const double out = red[0];
    __syncthreads();
    return out;
}

template <bool C>
__global__ void __launch_bounds__(CG_THREADS) cgs2_append_kernel(double* Q, int64_t n, int64_t ldq, int j,
                                                                  const double* v, int64_t ldv, double* Rt,
                                                                  int64_t ldr, double* part, double* hbuf,
                                                                  double* rbuf, double* npart, GridBar* bar,
                                                                  int32_t* flag) {
    extern __shared__ double cg_smem[];
    __shared__ double red[CG_THREADS / 32];
    const int W = C ? 2 : 1;
    const unsigned nblk = gridDim.x;
    const int b = blockIdx.x, tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int64_t rb = (n + nblk - 1) / nblk;
    const int64_t r0 = (int64_t)b * rb, r1 = r0 + rb < n ? r0 + rb : n;
    const int nr = r1 > r0 ? (int)(r1 - r0) : 0;
    double* sx = cg_smem;                 // [rb] this CTA's rows of x
    double* sh = cg_smem + (size_t)W * rb;  // [j] h
    for (int i = tid; i < nr; i += CG_THREADS) {
        const Cx<C> e = cx_ld<C>(v, (r0 + i) * ldv);
        sx[W * i] = e.re;
        if (C) sx[W * i + 1] = e.im;
    }
    __syncthreads();

    auto project = [&](bool accumulate, bool first) -> bool {
        // partial h over this CTA's rows
        for (int c = tid; c < j; c += CG_THREADS) {
            double ar = 0.0, ai = 0.0;
#pragma unroll 4
            for (int i = 0; i < nr; ++i) {
                const Cx<C> q = cx_ld<C>(Q, (r0 + i) * ldq + c);
                const double xr = sx[W * i], xi = C ? sx[W * i + 1] : 0.0;
                ar += q.re * xr + q.im * xi;  // conj(q) x
                if (C) ai += q.re * xi - q.im * xr;
            }
            cx_st<C>(part, (int64_t)b * j + c, Cx<C>{ar, ai});
        }
        if (!grid_barrier(bar, nblk, flag)) return false;
        // column c: the fixed-order sum over the CTAs
        for (int c = b; c < j; c += (int)nblk) {
            double sr = 0.0, si = 0.0;
            for (unsigned bb = tid; bb < nblk; bb += CG_THREADS) {
                const Cx<C> e = cx_ld<C>(part, (int64_t)bb * j + c);
                sr += e.re;
                si += e.im;
            }
            sr = block_sum(sr, red);
            if (C) si = block_sum(si, red);
            if (tid == 0) {
                cx_st<C>(hbuf, c, Cx<C>{sr, si});
                if (accumulate) {
                    Cx<C> r = first ? Cx<C>{0.0, 0.0} : cx_ld<C>(rbuf, c);
                    cx_st<C>(rbuf, c, Cx<C>{r.re + sr, r.im + si});
                }
            }
        }
        if (!grid_barrier(bar, nblk, flag)) return false;
        for (int c = tid; c < j; c += CG_THREADS) {
            const Cx<C> e = cx_ld<C>(hbuf, c);
            sh[W * c] = e.re;
            if (C) sh[W * c + 1] = e.im;
        }
        __syncthreads();
        // x -= Q h on this CTA's rows
        for (int i = warp; i < nr; i += CG_THREADS / 32) {
            double ar = 0.0, ai = 0.0;
            for (int c = lane; c < j; c += 32) {
                const Cx<C> q = cx_ld<C>(Q, (r0 + i) * ldq + c);
                const double hr = sh[W * c], hi = C ? sh[W * c + 1] : 0.0;
                ar += q.re * hr - q.im * hi;
                if (C) ai += q.re * hi + q.im * hr;
            }
            for (int o = 16; o > 0; o >>= 1) {
                ar += __shfl_xor_sync(0xffffffffu, ar, o);
                if (C) ai += __shfl_xor_sync(0xffffffffu, ai, o);
            }
            if (lane == 0) {
                sx[W * i] -= ar;
                if (C) sx[W * i + 1] -= ai;
            }
        }
        __syncthreads();
        return true;
    };
    auto norm = [&](double& out) -> bool {
        double p = 0.0;
        for (int i = tid; i < nr; i += CG_THREADS) {
            p += sx[W * i] * sx[W * i];
            if (C) p += sx[W * i + 1] * sx[W * i + 1];
        }
        p = block_sum(p, red);
        if (tid == 0) npart[b] = p;
        if (!grid_barrier(bar, nblk, flag)) return false;
        double t = 0.0;
        for (unsigned bb = tid; bb < nblk; bb += CG_THREADS) t += npart[bb];
        t = block_sum(t, red);
        out = sqrt(t > 0.0 ? t : 0.0);
        return true;
    };
    auto scale = [&](double d) {
        const double f = 1.0 / (d > 1e-300 ? d : 1e-300);
        for (int i = tid; i < nr * W; i += CG_THREADS) sx[i] *= f;
        __syncthreads();
    };

    double rjj = 0.0, qn = 0.0;
    if (j > 0 && (!project(true, true) || !project(true, false))) return;
    if (!norm(rjj)) return;
    scale(rjj);
    if (j > 0 && (!project(false, false) || !project(false, false))) return;
    if (!norm(qn)) return;
    scale(qn);
    for (int i = tid; i < nr; i += CG_THREADS)
        cx_st<C>(Q, (r0 + i) * ldq + j, Cx<C>{sx[W * i], C ? sx[W * i + 1] : 0.0});
    if (b == 0) {
        for (int c = tid; c < j; c += CG_THREADS) cx_st<C>(Rt, (int64_t)j * ldr + c, cx_ld<C>(rbuf, c));
        if (tid == 0) cx_st<C>(Rt, (int64_t)j * ldr + j, Cx<C>{rjj, 0.0});
    }
}

template <bool C>
int cgs2_append_t(bem_ctx* ctx, double* Q, int64_t n, int64_t ldq, int j, const double* v, int64_t ldv,
                  double* Rt, int64_t ldr, int check, cudaStream_t s) {
    const int W = C ? 2 : 1;
    int nblk0 = ctx->num_sms;
    const int64_t rb0 = (n + nblk0 - 1) / nblk0;
    const size_t smem = sizeof(double) * W * ((size_t)rb0 + (size_t)std::max(j, 1));
    if (smem > 200 * 1024) return bem_fail(ctx, BEM_ERR_INVALID, "cgs2_append: n or j too large");
    cudaFuncSetAttribute(cgs2_append_kernel<C>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    const int nblk = coop_blocks(ctx, (const void*)cgs2_append_kernel<C>, CG_THREADS, smem, ctx->num_sms);
    if (nblk < 1) return bem_fail(ctx, BEM_ERR_CUDA, "cgs2_append_kernel cannot be made co-resident");
    if (nblk != nblk0) return bem_fail(ctx, BEM_ERR_CUDA, "cgs2_append_kernel: fewer co-resident CTAs than SMs");
    const size_t jb = (size_t)std::max(j, 1);
    const size_t bytes = 256 + sizeof(double) * W * ((size_t)nblk * jb + 2 * jb) + sizeof(double) * nblk;
    if (int rc = bem_ws_reserve(ctx, bytes)) return rc;
    char* base = static_cast<char*>(ctx->ws);
    GridBar* bar = reinterpret_cast<GridBar*>(base);
    double* part = reinterpret_cast<double*>(base + 256);
    double* hbuf = part + (size_t)W * nblk * jb;
    double* rbuf = hbuf + (size_t)W * jb;
    double* npart = rbuf + (size_t)W * jb;
    if (int rc = bem_check_cuda(ctx, cudaMemsetAsync(bar, 0, sizeof(GridBar), s), "cgs2 barrier reset")) return rc;
    int32_t* flag = ctx->flags + 7;
    void* args[] = {&Q, &n, &ldq, &j, (void*)&v, &ldv, &Rt, &ldr, &part, &hbuf, &rbuf, &npart, &bar, &flag};
    if (int rc = bem_check_cuda(ctx, cudaLaunchCooperativeKernel((const void*)cgs2_append_kernel<C>, nblk,
                                                                CG_THREADS, args, smem, s),
                                "cgs2_append_kernel"))
        return rc;
    ctx->launches++;
    if (!check) return BEM_OK;
    int32_t f = 0;
    if (int rc = bem_check_cuda(ctx, cudaMemcpyAsync(&f, flag, sizeof(int32_t), cudaMemcpyDeviceToHost, s),
                                "cgs2 flag readback"))
        return rc;
    if (int rc = bem_check_cuda(ctx, cudaStreamSynchronize(s), "cgs2_append")) return rc;
    if (f != 0) {
        cudaMemsetAsync(flag, 0, sizeof(int32_t), s);
        return bem_fail(ctx, BEM_ERR_TIMEOUT, "cgs2_append: a grid barrier hit its iteration cap");
    }
    return BEM_OK;
}

template <typename T, bool C>
int gemv_t(bem_ctx* ctx, const T* A, int64_t m, int64_t n, int64_t lda, const double* x, double* y, double alpha,
           double beta, cudaStream_t s) {
    unsigned blocks = (unsigned)((m + 7) / 8);
    gemv_kernel<T, C><<<blocks, 256, 0, s>>>(A, m, n, lda, x, y, alpha, beta);
    ctx->launches++;
    return bem_check_cuda(ctx, cudaGetLastError(), "gemv_kernel");
}

}  // namespace

extern "C" {

int bem_cgs2_append(bem_ctx* ctx, int dtype, void* Q, int64_t n, int64_t ldq, int j, const void* v, int64_t ldv,
                    void* Rt, int64_t ldr, int check, void* stream) {
    if (!ctx) return BEM_ERR_INVALID;
    if (!Q || !v || !Rt || n <= 0 || j < 0 || ldq <= j || ldr <= j || ldv <= 0)
        return bem_fail(ctx, BEM_ERR_INVALID, "cgs2_append: bad arguments");
    cudaStream_t s = (cudaStream_t)stream;
    switch (dtype) {
        case BEM_F64:
            return cgs2_append_t<false>(ctx, (double*)Q, n, ldq, j, (const double*)v, ldv, (double*)Rt, ldr, check, s);
        case BEM_C128:
            return cgs2_append_t<true>(ctx, (double*)Q, n, ldq, j, (const double*)v, ldv, (double*)Rt, ldr, check, s);
        default: return bem_fail(ctx, BEM_ERR_INVALID, "cgs2_append: dtype must be BEM_F64 or BEM_C128");
    }
}

int bem_lu_factor(bem_ctx* ctx, int dtype, void* A, int64_t n, int64_t lda, int32_t* piv, int32_t* info,
                  void* stream) {
    if (!ctx) return BEM_ERR_INVALID;
    if (!A || !piv || !info || n <= 0 || lda < n) return bem_fail(ctx, BEM_ERR_INVALID, "lu_factor: bad arguments");
    if (n > (int64_t)1 << 30) return bem_fail(ctx, BEM_ERR_INVALID, "lu_factor: n too large");
    cudaStream_t s = (cudaStream_t)stream;
    switch (dtype) {
        case BEM_F64: return lu_factor_t<double, false>(ctx, (double*)A, n, lda, piv, info, s);
        case BEM_C128: return lu_factor_t<double, true>(ctx, (double*)A, n, lda, piv, info, s);
        case BEM_F32: return lu_factor_t<float, false>(ctx, (float*)A, n, lda, piv, info, s);
        case BEM_C64: return lu_factor_t<float, true>(ctx, (float*)A, n, lda, piv, info, s);
        default: return bem_fail(ctx, BEM_ERR_INVALID, "lu_factor: unknown dtype");
    }
}

int bem_lu_solve(bem_ctx* ctx, int dtype, const void* LU, int64_t n, int64_t lda, const int32_t* piv, void* b,
                 int64_t nrhs, int64_t ldb, void* stream) {
    if (!ctx) return BEM_ERR_INVALID;
    if (!LU || !piv || !b || n <= 0 || lda < n || ldb < nrhs)
        return bem_fail(ctx, BEM_ERR_INVALID, "lu_solve: bad arguments");
    cudaStream_t s = (cudaStream_t)stream;
    switch (dtype) {
        case BEM_F64: return lu_solve_t<double, false>(ctx, (const double*)LU, n, lda, piv, (double*)b, nrhs, ldb, s);
        case BEM_C128: return lu_solve_t<double, true>(ctx, (const double*)LU, n, lda, piv, (double*)b, nrhs, ldb, s);
        case BEM_F32: return lu_solve_t<float, false>(ctx, (const float*)LU, n, lda, piv, (double*)b, nrhs, ldb, s);
        case BEM_C64: return lu_solve_t<float, true>(ctx, (const float*)LU, n, lda, piv, (double*)b, nrhs, ldb, s);
        default: return bem_fail(ctx, BEM_ERR_INVALID, "lu_solve: unknown dtype");
    }
}

int bem_gemv(bem_ctx* ctx, int a_dtype, const void* A, int64_t m, int64_t n, int64_t lda, const void* x, void* y,
             double alpha, double beta, void* stream) {
    if (!ctx) return BEM_ERR_INVALID;
    if (!A || !x || !y || m <= 0 || n <= 0 || lda < n) return bem_fail(ctx, BEM_ERR_INVALID, "gemv: bad arguments");
    cudaStream_t s = (cudaStream_t)stream;
    switch (a_dtype) {
        case BEM_F64: return gemv_t<double, false>(ctx, (const double*)A, m, n, lda, (const double*)x, (double*)y, alpha, beta, s);
        case BEM_C128: return gemv_t<double, true>(ctx, (const double*)A, m, n, lda, (const double*)x, (double*)y, alpha, beta, s);
        case BEM_F32: return gemv_t<float, false>(ctx, (const float*)A, m, n, lda, (const double*)x, (double*)y, alpha, beta, s);
        case BEM_C64: return gemv_t<float, true>(ctx, (const float*)A, m, n, lda, (const double*)x, (double*)y, alpha, beta, s);
        default: return bem_fail(ctx, BEM_ERR_INVALID, "gemv: unknown dtype");
    }
}

int bem_refine_solve(bem_ctx* ctx, int dtype_hi, const void* A_hi, const void* LU_lo, const int32_t* piv,
                     const void* dinv, int64_t n, int64_t lda, const void* b, void* x, double tol, int maxit,
                     int* iters, double* relres, void* stream) {
    if (!ctx) return BEM_ERR_INVALID;
    if (!A_hi || !LU_lo || !piv || !b || !x || n <= 0 || lda < n || maxit < 1 || !(tol > 0))
        return bem_fail(ctx, BEM_ERR_INVALID, "refine_solve: bad arguments");
    if (dtype_hi != BEM_F64 && dtype_hi != BEM_C128)
        return bem_fail(ctx, BEM_ERR_INVALID, "refine_solve: A_hi must be F64 or C128");
    const bool C = dtype_hi == BEM_C128;
    const int W = C ? 2 : 1;
    const int64_t nd = W * n;
    cudaStream_t s = (cudaStream_t)stream;
    if (dinv) return refine_async(ctx, C, A_hi, LU_lo, piv, dinv, n, lda, (const double*)b, (double*)x, tol, maxit,
                                  iters, relres, s);
    // workspace beyond the lu_solve scratch: r (nd), d (nd), norms (2)
    double* r = nullptr;
    if (int rc = bem_check_cuda(ctx, cudaMallocAsync((void**)&r, sizeof(double) * (2 * nd + 4), s), "refine alloc"))
        return rc;
    double* d = r + nd;
    double* nrm = d + nd;
    const double* bd = (const double*)b;
    double* xd = (double*)x;
    int rc = BEM_OK;
    double bnorm = 0.0, rnorm = 0.0;
    int it = 0;
    auto norm2 = [&](const double* v, double* out_host) -> int {
        cudaMemsetAsync(nrm, 0, sizeof(double), s);
        sumsq_kernel<<<std::min<int64_t>(ctx->num_sms * 4, (nd + 255) / 256), 256, 0, s>>>(v, nd, nrm);
        ctx->launches++;
        if (int e = bem_check_cuda(ctx, cudaMemcpyAsync(out_host, nrm, sizeof(double), cudaMemcpyDeviceToHost, s),
                                   "norm readback"))
            return e;
        if (int e = bem_check_cuda(ctx, cudaStreamSynchronize(s), "norm")) return e;
        *out_host = std::sqrt(*out_host);
        return BEM_OK;
    };
    rc = norm2(bd, &bnorm);
    if (rc == BEM_OK) rc = bem_check_cuda(ctx, cudaMemsetAsync(xd, 0, sizeof(double) * nd, s), "x=0");
    if (rc == BEM_OK) rc = bem_check_cuda(ctx, cudaMemcpyAsync(r, bd, sizeof(double) * nd, cudaMemcpyDeviceToDevice, s), "r=b");
    rnorm = bnorm;
    if (bnorm == 0.0) {
        cudaFreeAsync(r, s);
        if (iters) *iters = 0;
        if (relres) *relres = 0.0;
        return rc;
    }
    while (rc == BEM_OK && it < maxit) {
        // d = LU_lo^{-1} r
        rc = bem_check_cuda(ctx, cudaMemcpyAsync(d, r, sizeof(double) * nd, cudaMemcpyDeviceToDevice, s), "d=r");
        if (rc) break;
        if (dinv)
            rc = bem_lu_solve_tiled(ctx, C ? BEM_C64 : BEM_F32, LU_lo, n, lda, piv, dinv, d, s);
        else
            rc = bem_lu_solve(ctx, C ? BEM_C64 : BEM_F32, LU_lo, n, lda, piv, d, 1, 1, s);
        if (rc) break;
        axpy_kernel<<<(unsigned)((nd + 255) / 256), 256, 0, s>>>(xd, d, nd, 1.0);
        ctx->launches++;
        // r = b - A_hi x
        rc = bem_check_cuda(ctx, cudaMemcpyAsync(r, bd, sizeof(double) * nd, cudaMemcpyDeviceToDevice, s), "r=b");
        if (rc) break;
        rc = bem_gemv(ctx, dtype_hi, A_hi, n, n, lda, xd, r, -1.0, 1.0, s);
        if (rc) break;
        ++it;
        const double prev = rnorm;
        rc = norm2(r, &rnorm);
        if (rc) break;
        if (rnorm <= tol * bnorm) break;
        if (it >= 3 && rnorm > 0.5 * prev) break;  // stagnation: the factor is not a good enough preconditioner
    }
    cudaFreeAsync(r, s);
    if (iters) *iters = it;
    if (relres) *relres = rnorm / bnorm;
    if (rc == BEM_OK && rnorm > tol * bnorm)
        return bem_fail(ctx, BEM_ERR_NOCONVERGE, "refinement did not reach tol in maxit iterations");
    return rc;
}

int bem_gmres_ir(bem_ctx* ctx, int dtype_hi, const void* A_hi, const void* LU_lo, const int32_t* piv,
                 const void* dinv, int64_t n, int64_t lda, const void* b, void* x, double tol, int maxit, int restart,
                 double accept, int* iters, double* relres, void* stream) {
    if (!ctx) return BEM_ERR_INVALID;
    if (!A_hi || !LU_lo || !piv || !b || !x || n <= 0 || lda < n || maxit < 1 || restart < 1 || !(tol > 0))
        return bem_fail(ctx, BEM_ERR_INVALID, "gmres_ir: bad arguments");
    if (dtype_hi != BEM_F64 && dtype_hi != BEM_C128)
        return bem_fail(ctx, BEM_ERR_INVALID, "gmres_ir: A_hi must be F64 or C128");
    return gmres_run(ctx, dtype_hi, A_hi, LU_lo, piv, dinv, n, lda, (const double*)b, (double*)x, tol, maxit,
                     restart, accept, iters, relres, (cudaStream_t)stream);
}

}  // extern "C"
