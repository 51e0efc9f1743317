// Least squares of the stacked transmission system [A; P] x = [b1; b2]
// (the reference's torch.linalg.lstsq, BEM_manager.py:1039-1050), by the
// column-equilibrated normal equations
//     N z = g,   N = D (A^H A + P^H P) D,   g = D (A^H b1 + P^H b2),   x = D z,
// with D = diag(2^-e_p) the power of two nearest to 1/||column p of [A; P]||.
//
// Mixed precision: N is formed on the tcgen05 tensor cores from FP16 hi/lo
// splits of the scaled columns (x = hi + 2^-11 lo, both FP16, so each product
// keeps about 22 bits: hi*hi + 2^-11 (hi*lo + lo*hi)), accumulated in FP32 in
// TMEM, factored by the FP32 tile LU, and the solution is refined by flexible
// GMRES in FP64 on the normal equations with FP64 products against the
// FP64-stored A and P.  Plain FP64: N by FP64 tensor-core (DMMA) products,
// the FP64 tile LU, and the same FP64 iteration (it converges in one or two
// steps).
//
// The normal matrix is Hermitian; its real form is S = T T^T with T the
// transposed real view of G = [A; P] D (row 2p + c of T is the real (c = 0)
// or imaginary (c = 1) part of column p of G), and
//     N[p][q] = (S[2p][2q] + S[2p+1][2q+1]) + i (S[2p][2q+1] - S[2p+1][2q]).
// Only tiles on or below the diagonal of S are computed; a mirror pass writes
// the conjugate transpose above the diagonal.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <mutex>

#include "bem_internal.cuh"

namespace {

// ---------------------------------------------------------------------------
// column scaling
// ---------------------------------------------------------------------------
constexpr int CN_ROWS = 512;  // rows of [A; P] per block of the column-norm pass

// cn2[p] += sum over a chunk of rows of |G_kp|^2 (G = [A; P], complex or real)
template <bool C>
__global__ void colnorm_kernel(const double* A, const double* P, int64_t ld, int n, double* cn2) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const int W = C ? 2 : 1;
    const int k0 = blockIdx.y * CN_ROWS, k1 = min(2 * n, k0 + CN_ROWS);
    double acc = 0.0;
    for (int k = k0; k < k1; ++k) {
        const double* row = (k < n ? A + (int64_t)k * ld * W : P + (int64_t)(k - n) * ld * W);
        if (C) {
            const double2 v = reinterpret_cast<const double2*>(row)[p];
            acc += v.x * v.x + v.y * v.y;
        } else {
            const double v = row[p];
            acc += v * v;
        }
    }
    atomicAdd(cn2 + p, acc);
}

// d[p] = 2^-e with e the integer nearest to log2 ||column p|| (1 for a zero column)
__global__ void colscale_kernel(const double* cn2, double* d, int n) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const double c = cn2[p];
    d[p] = c > 0.0 ? ldexp(1.0, -(int)rint(0.5 * log2(c))) : 1.0;
}

// ---------------------------------------------------------------------------
// FP16 hi/lo split of the scaled, transposed real view: T[2p + c][k]
// ---------------------------------------------------------------------------
// Block: 32 columns p x 64 rows k of G (complex), through shared memory, so
// that reads run along p and writes along k.  Padding rows (p >= n) and
// columns (k >= 2n) of T are written as zeros.
template <bool C>
__global__ void __launch_bounds__(256) split_kernel(const double* A, const double* P, int64_t ld, int n,
                                                    const double* d, __half* Thi, __half* Tlo, int64_t ldt) {
    __shared__ double2 tile[64][33];
    const int p0 = blockIdx.x * 32, k0 = blockIdx.y * 64;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int W = C ? 2 : 1;
    for (int kk = warp; kk < 64; kk += 8) {
        const int k = k0 + kk, p = p0 + lane;
        double2 v = make_double2(0.0, 0.0);
        if (p < n && k < 2 * n) {
            const double* row = (k < n ? A + (int64_t)k * ld * W : P + (int64_t)(k - n) * ld * W);
            const double s = d[p];
            if (C) {
                v = reinterpret_cast<const double2*>(row)[p];
                v.x *= s;
                v.y *= s;
            } else {
                v.x = row[p] * s;
            }
        }
        tile[kk][lane] = v;
    }
    __syncthreads();
    // T rows of this block: 2 * 32 (complex) or 32 (real); each warp writes one
    // row segment of 64 k values as 32 half2
    const int trows = C ? 64 : 32;
    for (int rr = warp; rr < trows; rr += 8) {
        const int pl = C ? rr >> 1 : rr, c = C ? rr & 1 : 0;
        const int64_t i = C ? 2 * (int64_t)(p0 + pl) + c : (int64_t)(p0 + pl);
        const double2 v0 = tile[2 * lane][pl], v1 = tile[2 * lane + 1][pl];
        const float f0 = (float)(c ? v0.y : v0.x), f1 = (float)(c ? v1.y : v1.x);
        const __half h0 = __float2half_rn(f0), h1 = __float2half_rn(f1);
        const __half l0 = __float2half_rn((f0 - __half2float(h0)) * 2048.0f);
        const __half l1 = __float2half_rn((f1 - __half2float(h1)) * 2048.0f);
        const int64_t off = i * ldt + k0 + 2 * lane;
        *reinterpret_cast<__half2*>(Thi + off) = __halves2half2(h0, h1);
        *reinterpret_cast<__half2*>(Tlo + off) = __halves2half2(l0, l1);
    }
}

// FP16 hi/lo split of a panel L (m x kb, row-major, ld) for the Hermitian
// update L L^H: T[2p + c][k] = (Re, -Im)[c] of L[p][k] (real: T[p][k] =
// L[p][k]), zero padding to Rp x Kp.  Rows of L map to rows of T: no
// transposition.  Grid: (Kp / 64, rows of T / 4), 256 threads (4 rows x 64 k).
template <bool C>
__global__ void __launch_bounds__(256) panel_split_kernel(const double* L, int64_t ld, int m, int kb, __half* Thi,
                                                          __half* Tlo, int64_t Kp, int64_t Rp) {
    const int k = blockIdx.x * 64 + (threadIdx.x & 63);
    const int64_t i = (int64_t)blockIdx.y * 4 + (threadIdx.x >> 6);
    if (i >= Rp) return;
    double v = 0.0;
    if (C) {
        const int64_t p = i >> 1;
        const int c = (int)(i & 1);
        if (p < m && k < kb) v = c ? -L[2 * (p * ld + k) + 1] : L[2 * (p * ld + k)];
    } else if (i < m && k < kb) {
        v = L[i * ld + k];
    }
    const float f = (float)v;
    const __half h = __float2half_rn(f);
    Thi[i * Kp + k] = h;
    Tlo[i * Kp + k] = __float2half_rn((f - __half2float(h)) * 2048.0f);
}

// lower-triangle tile t (row-major order, diagonal included) -> (bi, bj), bi >= bj
__device__ __forceinline__ int tri_row(int t) {
    int i = (int)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
    while (i * (i + 1) / 2 > t) --i;
    while ((i + 1) * (i + 2) / 2 <= t) ++i;
    return i;
}

// Tile t of the lower triangle (bi >= bj) of a T x T tile grid, in bands of G
// tile columns: band b (columns [bG, bG + w), w = min(G, T - bG)) runs down
// its rows from bi = bG, each row's tiles in column order; the first w rows
// are the band's triangle.  Tiles that run at the same time (consecutive t)
// then share about G row panels and T_conc / G column panels, whose K chunks
// the L2 serves to all of them, instead of one column panel per CTA streamed
// from DRAM.  G <= 0: plain row order.
__device__ __forceinline__ void tri_tile(int t, int T, int G, int& bi, int& bj) {
    if (G <= 0 || G >= T) {
        bi = tri_row(t);
        bj = t - bi * (bi + 1) / 2;
        return;
    }
    int b0 = 0;
    for (;;) {
        const int w = min(G, T - b0);
        const int tri = w * (w + 1) / 2;
        const int size = tri + (T - b0 - w) * w;
        if (t < size) {
            if (t < tri) {
                const int r = tri_row(t);
                bi = b0 + r;
                bj = b0 + (t - r * (r + 1) / 2);
            } else {
                const int u = t - tri;
                bi = b0 + w + u / w;
                bj = b0 + u % w;
            }
            return;
        }
        t -= size;
        b0 += w;
    }
}

// ---------------------------------------------------------------------------
// tcgen05 Gram kernel: S_tile = T[rows bi] T[rows bj]^T over all K
// ---------------------------------------------------------------------------
// Persistent: one CTA per SM takes tiles blockIdx.x, + gridDim.x, ...; the
// stage ring and the TMEM accumulator sets run on across tiles, so loads and
// MMAs of the next tile overlap the epilogue of the last one.
// Warp 0 is the TMA producer, warp 1 allocates TMEM and issues the MMAs
// (one elected thread), warps 2-9 are the epilogue (warp w reads TMEM lanes
// 32 (w % 4) .. and half (w - 2) / 4 of the columns).  A stage holds the hi and lo 128 x 64 FP16 tiles of both
// operands, loaded by TMA with the 128-byte swizzle into 1024-byte aligned
// shared memory; the matching UMMA descriptors are K-major SWIZZLE_128B
// (8-row groups 1024 bytes apart), advanced by 32 bytes per K = 16 step.
// Per K = 16 step three MMAs: D1 += A_hi B_hi, D2 += A_hi B_lo + A_lo B_hi.
// K is accumulated in segments of kseg stages; two TMEM accumulator sets
// alternate, so the epilogue adds segment g (D1 + 2^-11 D2, formed in FP32)
// to its FP64 running sums while the MMAs of segment g + 1 run.  The tensor
// core's FP32 accumulation does not round to nearest: its error grows with
// the number of MMA steps a TMEM sum sees (measured on the 30722-unknown
// normal matrix: 2e-5 relative for segments of 64 stages, 1.5e-6 for 4,
// 8e-7 for 2, 4e-7 for 1), so the default folds every two stages (8 MMA steps
// per sum: the fastest setting at which the least-squares iteration still
// converges in about 6 steps), and the FP64 running sums keep the segment
// count from adding its own rounding.
constexpr int GT_BM = 128;
constexpr int GT_BK = 64;
constexpr int GT_STAGES = 3;
constexpr int GT_TILE = GT_BM * GT_BK * 2;  // bytes of one 128 x 64 FP16 tile
constexpr int GT_STAGE = 4 * GT_TILE;
constexpr int GT_KSEG_DEFAULT = 2;
// tile columns per band of the tile order (tri_tile).  Bands of 12 (12 x 12
// tiles ~ one wave of 148 CTAs) cut the operand reads from DRAM 4x at 7682
// unknowns, but single-column bands measured faster under CUDA events at the
// default segment on 7682 and 30722 unknowns (14.4 vs 16.6 ms, 1147 vs
// 1183 ms); the autotuner chooses per problem.
constexpr int GRAM_BAND_DEFAULT = 1;
// form of the tensor-core Gram product (BEM_TUNE_GRAM_PAIR): 1 one CTA per
// 128 x 128 tile (gram_tc_kernel, eight epilogue warps), 2 CTA pairs on 256 x
// 128 tiles (gram_tc2_kernel), 3 one CTA per tile with sixteen epilogue warps
constexpr int GRAM_PAIR_DEFAULT = 1;
constexpr int GT_EPI_WARPS = 8;
constexpr int GT_THREADS = 64 + 32 * GT_EPI_WARPS;
constexpr uint32_t GT_TMEM_COLS = 512;  // 2 sets x (D1, D2) x 128 columns
constexpr uint32_t GT_SPIN_CAP = 1u << 24;
constexpr size_t GT_SMEM = (size_t)GT_STAGES * GT_STAGE + 1024;
constexpr int GT_STG_LD = 64 + 1;  // padded row of the epilogue's staging buffer (doubles)
// instruction descriptor, kind::f16: D F32 (bit 4), A and B F16 (0), both
// K-major, N >> 3 at bits 17-22, M >> 4 at bits 24-28
constexpr uint32_t GT_IDESC = (1u << 4) | ((uint32_t)(GT_BM >> 3) << 17) | ((uint32_t)(GT_BM >> 4) << 24);

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ bool mbar_try(uint32_t addr, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(addr), "r"(parity)
        : "memory");
    return done != 0;
}

__device__ __forceinline__ bool mbar_wait(uint32_t addr, uint32_t parity, volatile int* abort) {
    for (uint32_t it = 0; it < GT_SPIN_CAP; ++it) {
        if (mbar_try(addr, parity)) return true;
        if ((it & 1023u) == 1023u && *abort) return false;
    }
    return false;
}

__device__ __forceinline__ uint64_t desc_sw128(uint32_t saddr) {
    uint64_t dsc = 0;
    dsc |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    dsc |= (uint64_t)1 << 16;              // leading byte offset (not used by swizzled K-major layouts)
    dsc |= (uint64_t)(1024u >> 4) << 32;   // stride byte offset: 8 rows of 128 bytes
    dsc |= (uint64_t)1 << 46;              // descriptor version
    dsc |= (uint64_t)2 << 61;              // SWIZZLE_128B
    return dsc;
}

__device__ __forceinline__ void mma_f16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(GT_IDESC), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void tma_load(uint32_t dst, const CUtensorMap* map, uint32_t mbar, int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(
            dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(mbar), "r"(x), "r"(y)
        : "memory");
}

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float* v) {
    uint32_t u[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(u[0]), "=r"(u[1]), "=r"(u[2]), "=r"(u[3]), "=r"(u[4]), "=r"(u[5]), "=r"(u[6]), "=r"(u[7])
                 : "r"(taddr)
                 : "memory");
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(u[i]);
}

// out: complex (C, interleaved pairs) or real N x N matrix of OT (float or double), ld in elements
template <bool C, typename OT, int EW>
__global__ void __launch_bounds__(64 + 32 * EW, 1) gram_tc_kernel(const __grid_constant__ CUtensorMap tm_hi,
                                                                 const __grid_constant__ CUtensorMap tm_lo,
                                                                 int nchunks, int kseg, int ntiles, int tgrid,
                                                                 int band, OT* out, int64_t ldo, int n, double alpha,
                                                                 int accumulate, int32_t* err) {
    extern __shared__ unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t full_bar[GT_STAGES], empty_bar[GT_STAGES], acc_full[2], acc_empty[2];
    __shared__ uint32_t tmem_slot;
    __shared__ volatile int s_abort;
    // EW epilogue warps: warp w reads TMEM lanes 32 (w % 4) .. and column group (w - 2) / 4 of EW / 4
    constexpr int NCG = EW / 4, EC = GT_BM / NCG, STG_LD = EC + 1;
    __shared__ double s_stage[EW][8 * STG_LD];  // epilogue staging, eight real rows per warp
    unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) &
                                                           ~uintptr_t(1023));
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int nseg = (nchunks + kseg - 1) / kseg;  // per tile

    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                     "r"(GT_TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int s = 0; s < GT_STAGES; ++s) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&full_bar[s])) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&empty_bar[s])) : "memory");
        }
        for (int b = 0; b < 2; ++b) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&acc_full[b])) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&acc_empty[b])), "r"(EW)
                         : "memory");
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_abort = 0;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_slot;

    if (warp == 0) {
        // ---- TMA producer ----
        if (lane == 0) {
            asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tm_hi)) : "memory");
            asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tm_lo)) : "memory");
            uint32_t cg = 0;  // chunks issued by this CTA (the stage ring runs across tiles)
            for (int t = blockIdx.x; t < ntiles && !s_abort; t += gridDim.x) {
                int bi, bj;
                tri_tile(t, tgrid, band, bi, bj);
                for (int c = 0; c < nchunks; ++c, ++cg) {
                    const int s = (int)(cg % GT_STAGES);
                    if (cg >= GT_STAGES &&
                        !mbar_wait(smem_u32(&empty_bar[s]), (uint32_t)((cg / GT_STAGES - 1) & 1), &s_abort)) {
                        s_abort = 1;
                        break;
                    }
                    const uint32_t fb = smem_u32(&full_bar[s]);
                    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(fb), "r"(GT_STAGE)
                                 : "memory");
                    const uint32_t st = smem_u32(smem + (size_t)s * GT_STAGE);
                    const int x = c * GT_BK;
                    tma_load(st, &tm_hi, fb, x, bi * GT_BM);
                    tma_load(st + GT_TILE, &tm_lo, fb, x, bi * GT_BM);
                    tma_load(st + 2 * GT_TILE, &tm_hi, fb, x, bj * GT_BM);
                    tma_load(st + 3 * GT_TILE, &tm_lo, fb, x, bj * GT_BM);
                }
            }
        }
    } else if (warp == 1) {
        // ---- MMA issuer ----
        if (lane == 0) {
            uint32_t cg = 0, gg = 0;  // chunks and segments consumed by this CTA
            for (int t = blockIdx.x; t < ntiles && !s_abort; t += gridDim.x) {
            int c = 0;
            for (int g = 0; g < nseg && !s_abort; ++g, ++gg) {
                const int buf = (int)(gg & 1);
                if (gg >= 2 && !mbar_wait(smem_u32(&acc_empty[buf]), (uint32_t)((gg / 2 - 1) & 1), &s_abort)) {
                    s_abort = 1;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t d1 = tmem + (uint32_t)(buf * 256), d2 = d1 + 128;
                const int cend = min(nchunks, (g + 1) * kseg);
                for (int first = 1; c < cend; ++c, ++cg, first = 0) {
                    const int s = (int)(cg % GT_STAGES);
                    if (!mbar_wait(smem_u32(&full_bar[s]), (uint32_t)((cg / GT_STAGES) & 1), &s_abort)) {
                        s_abort = 1;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const uint32_t st = smem_u32(smem + (size_t)s * GT_STAGE);
#pragma unroll
                    for (int ks = 0; ks < GT_BK / 16; ++ks) {
                        const uint32_t ko = 32u * ks;
                        const uint64_t a_hi = desc_sw128(st + ko), a_lo = desc_sw128(st + GT_TILE + ko);
                        const uint64_t b_hi = desc_sw128(st + 2 * GT_TILE + ko),
                                       b_lo = desc_sw128(st + 3 * GT_TILE + ko);
                        const uint32_t acc = (first && ks == 0) ? 0u : 1u;
                        mma_f16(d1, a_hi, b_hi, acc);
                        mma_f16(d2, a_hi, b_lo, acc);
                        mma_f16(d2, a_lo, b_hi, 1u);
                    }
                    asm volatile(
                        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                            smem_u32(&empty_bar[s]))
                        : "memory");
                }
                if (s_abort) break;
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                 smem_u32(&acc_full[buf]))
                             : "memory");
            }
            }
        }
    } else {
        // ---- epilogue: FP64 running sums of the segments, then the complex combine ----
        const int q = warp & 3, half = (warp - 2) >> 2;  // lane quarter, column group
        uint32_t gg = 0;
        bool ok = true;
        for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
        int bi, bj;
        tri_tile(t, tgrid, band, bi, bj);
        double acc[EC];
#pragma unroll
        for (int i = 0; i < EC; ++i) acc[i] = 0.0;
        for (int g = 0; g < nseg; ++g, ++gg) {
            const int buf = (int)(gg & 1);
            // every lane waits; the vote keeps the warp's TMEM loads and shuffles uniform
            const bool got = mbar_wait(smem_u32(&acc_full[buf]), (uint32_t)((gg / 2) & 1), &s_abort);
            if (!__all_sync(0xffffffffu, got)) {
                ok = false;
                s_abort = 1;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t base = tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(buf * 256 + half * EC);
#pragma unroll
            for (int cc = 0; cc < EC; cc += 8) {
                float v1[8], v2[8];
                tmem_ld8(base + cc, v1);
                tmem_ld8(base + 128 + cc, v2);
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
                for (int i = 0; i < 8; ++i) acc[cc + i] += (double)fmaf(v2[i], 4.8828125e-4f, v1[i]);
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&acc_empty[buf])) : "memory");
        }
        if (ok) {
            const int r = bi * GT_BM + 32 * q + lane;  // real row of S
            const int c0 = bj * GT_BM + half * EC;     // first real column of this thread
            if (C) {
                // coalesced read-modify-write: the warp's 32 real rows pass through
                // shared memory eight at a time (four complex rows); lane l then forms
                // complex column l of each,
                //   N[p][q] = (S[2p][2q] + S[2p+1][2q+1]) + i (S[2p][2q+1] - S[2p+1][2q]),
                // so each access covers 32 contiguous complex entries
                double* stg = s_stage[warp - 2];  // [8][STG_LD]
                constexpr int CC = EC / 2;        // complex columns of the thread's column group
                constexpr int RPL = 4 * CC / 32;  // complex rows per lane and round
                const int lc = lane % CC, lr0 = (lane / CC) * RPL;
                const int pw0 = (bi * GT_BM + 32 * q) >> 1;  // first complex row of this warp
                const int qc = (c0 >> 1) + lc;
#pragma unroll
                for (int c4 = 0; c4 < 4; ++c4) {
                    if ((lane >> 3) == c4) {
#pragma unroll
                        for (int m = 0; m < EC; ++m) stg[(lane & 7) * STG_LD + m] = acc[m];
                    }
                    __syncwarp();
                    double nre[RPL], nim[RPL], ore[RPL], oim[RPL];
#pragma unroll
                    for (int ri = 0; ri < RPL; ++ri) {
                        const int rr = lr0 + ri;
                        const double* e = stg + (2 * rr) * STG_LD + 2 * lc;
                        const double* o = stg + (2 * rr + 1) * STG_LD + 2 * lc;
                        const int pr = pw0 + 4 * c4 + rr;
                        nre[ri] = e[0] + o[1];
                        nim[ri] = pr == qc ? 0.0 : e[1] - o[0];  // a Hermitian matrix has a real diagonal
                        ore[ri] = oim[ri] = 0.0;
                        if (accumulate && pr < n && qc < n) {
                            const OT* ot = out + 2 * ((int64_t)pr * ldo + qc);
                            ore[ri] = (double)ot[0];
                            oim[ri] = (double)ot[1];
                        }
                    }
#pragma unroll
                    for (int ri = 0; ri < RPL; ++ri) {
                        const int pr = pw0 + 4 * c4 + lr0 + ri;
                        if (pr < n && qc < n) {
                            OT* ot = out + 2 * ((int64_t)pr * ldo + qc);
                            ot[0] = (OT)(ore[ri] + alpha * nre[ri]);
                            ot[1] = (OT)(oim[ri] + alpha * nim[ri]);
                        }
                    }
                    __syncwarp();
                }
            } else if (r < n) {
                OT* orow = out + (int64_t)r * ldo + c0;
                double old[EC];
#pragma unroll
                for (int m = 0; m < EC; ++m) old[m] = (accumulate && c0 + m < n) ? (double)orow[m] : 0.0;
#pragma unroll
                for (int m = 0; m < EC; ++m)
                    if (c0 + m < n) orow[m] = (OT)(old[m] + alpha * acc[m]);
            }
        }
        }
    }
    if (s_abort && tid == 0) atomicExch(err, BEM_ERR_TIMEOUT);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 1)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(GT_TMEM_COLS) : "memory");
}

// ---------------------------------------------------------------------------
// CTA-pair variant (tcgen05 cta_group::2, M = 256 over the two CTAs of a
// cluster).  gram_tc_kernel floors where shared memory is busiest: per 64-wide
// K stage its TMA writes 64 KB and its three MMAs read A (16 KB) and B
// (16 KB) each, 160 KB against 813 clocks of tensor work at 128 B per clock.
// Here the pair computes a 256 x 128 tile (rows: tile rows 2p and 2p + 1, one
// per CTA; columns: tile column bj) with one MMA stream issued by the even
// CTA: each CTA holds its own 128 A rows and HALF (64 rows) of the B panel,
// and the hardware feeds both halves to both CTAs' MMAs, so per CTA and stage
// the TMA writes 48 KB and the MMAs read 72 KB (120 KB for the same tensor
// work).  Protocol (all waits bounded, as in gram_tc_kernel):
//  * TMEM: 512 columns allocated by warp 1 of both CTAs (cta_group::2), two
//    accumulator sets x (D1, D2) x 128 columns; each CTA's TMEM holds its own
//    128 rows;
//  * stage s: both producers load into their own shared memory with the
//    cta_group::2 TMA form, completing bytes on the EVEN CTA's full_bar[s],
//    where the even producer alone announces the pair's 96 KB; the even
//    CTA's MMA thread waits on it, and its tcgen05.commit arrives on
//    empty_bar[s] of both CTAs (one commit to the CTA mask 0b11);
//  * accumulators: the commit after a segment arrives on acc_full of both
//    CTAs; the eight epilogue warps of each CTA arrive on the EVEN CTA's
//    acc_empty (count 16) after draining their TMEM;
//  * teardown: a cluster barrier (neither CTA leaves while the other's MMAs
//    may still read its shared memory), then both CTAs free the TMEM.
// Tiles run in column order (the pairs of one tile column one after another,
// the order of single-column bands, BEM_TUNE_GRAM_BAND = 1).  Each TMA load
// fills the issuing CTA's own shared memory, and every tensor map covers this
// GPU's memory only.
// ---------------------------------------------------------------------------
constexpr int G2_STAGES = 4;
constexpr int G2_ATILE = GT_BM * GT_BK * 2;            // 16 KB: 128 x 64 FP16 rows of this CTA
constexpr int G2_BTILE = (GT_BM / 2) * GT_BK * 2;      // 8 KB: this CTA's 64-row half of the B panel
constexpr int G2_STAGE = 2 * G2_ATILE + 2 * G2_BTILE;  // 48 KB per CTA and stage
constexpr size_t G2_SMEM = (size_t)G2_STAGES * G2_STAGE + 1024;
// kind::f16, D F32, M = 256 (the pair), N = 128
constexpr uint32_t G2_IDESC = (1u << 4) | ((uint32_t)(GT_BM >> 3) << 17) | ((uint32_t)(256 >> 4) << 24);

// Pair tile t, column order over the lower triangle of a T x T grid of 128 x
// 128 tiles: tile column bj holds row pairs p = floor(bj / 2) .. P - 1 (P =
// ceil(T / 2)); columns 2c and 2c + 1 both hold P - c pairs.
__device__ __forceinline__ void pair_tile(int t, int T, int& p, int& bj) {
    const int P = (T + 1) >> 1;
    for (int c = 0; c < P; ++c) {
        const int cnt = P - c, ncol = min(2, T - 2 * c);
        if (t < ncol * cnt) {
            bj = 2 * c + t / cnt;
            p = c + t % cnt;
            return;
        }
        t -= ncol * cnt;
    }
    p = bj = 0;  // not reached for t < pair_tiles(T)
}

__host__ __device__ inline int64_t pair_tiles(int T) {
    const int P = (T + 1) >> 1;
    int64_t n = 0;
    for (int c = 0; c < P; ++c) n += (int64_t)(T - 2 * c < 2 ? T - 2 * c : 2) * (P - c);
    return n;
}

__device__ __forceinline__ uint32_t cluster_rank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
__device__ __forceinline__ uint32_t cluster_id_x() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%clusterid.x;" : "=r"(r));
    return r;
}
__device__ __forceinline__ uint32_t cluster_count_x() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%nclusterid.x;" : "=r"(r));
    return r;
}
// shared::cluster address of the same shared variable in CTA `rank` of the cluster
__device__ __forceinline__ uint32_t map_rank(uint32_t saddr, uint32_t rank) {
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(saddr), "r"(rank));
    return r;
}
__device__ __forceinline__ void cluster_sync_all() {
    asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");
    asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory");
}
// try_wait with cluster-scope acquire: the barrier receives arrivals from the peer CTA
__device__ __forceinline__ bool mbar_wait_cl(uint32_t addr, uint32_t parity, volatile int* abort) {
    for (uint32_t it = 0; it < GT_SPIN_CAP; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(addr), "r"(parity)
            : "memory");
        if (done) return true;
        if ((it & 1023u) == 1023u && *abort) return false;
    }
    return false;
}
__device__ __forceinline__ void tma_load_pair(uint32_t dst, const CUtensorMap* map, uint32_t mbar_leader, int x,
                                              int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, "
        "%4}], [%2];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(mbar_leader), "r"(x), "r"(y)
        : "memory");
}
__device__ __forceinline__ void mma_f16_pair(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(G2_IDESC), "r"(accumulate)
        : "memory");
}
// tcgen05.commit of the pair's MMAs: one arrival on the barrier at this
// shared address in both CTAs
__device__ __forceinline__ void commit_pair(uint32_t bar) {
    const uint16_t mask = 0x3;
    asm volatile(
        "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;" ::"r"(
            bar),
        "h"(mask)
        : "memory");
}

template <bool C, typename OT>
__global__ void __launch_bounds__(GT_THREADS, 1) gram_tc2_kernel(
    const __grid_constant__ CUtensorMap tm_hi, const __grid_constant__ CUtensorMap tm_lo,
    const __grid_constant__ CUtensorMap tmb_hi, const __grid_constant__ CUtensorMap tmb_lo, int nchunks, int kseg,
    int ntiles, int tgrid, OT* out, int64_t ldo, int n, double alpha, int accumulate, int32_t* err) {
    extern __shared__ unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t full_bar[G2_STAGES], empty_bar[G2_STAGES], acc_full[2], acc_empty[2];
    __shared__ uint32_t tmem_slot;
    __shared__ volatile int s_abort;
    __shared__ double s_stage[GT_EPI_WARPS][8 * GT_STG_LD];
    unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) &
                                                           ~uintptr_t(1023));
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int nseg = (nchunks + kseg - 1) / kseg;
    const uint32_t rank = cluster_rank();
    const int cid = (int)cluster_id_x(), ncl = (int)cluster_count_x();
    const bool leader = rank == 0;

    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                     "r"(GT_TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int s = 0; s < G2_STAGES; ++s) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&full_bar[s])) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&empty_bar[s])) : "memory");
        }
        for (int b = 0; b < 2; ++b) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&acc_full[b])) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&acc_empty[b])),
                         "r"(2 * GT_EPI_WARPS)
                         : "memory");
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_abort = 0;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    // both CTAs' barriers are initialised before any TMA or arrival of the peer reaches them
    cluster_sync_all();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_slot;

    if (warp == 0) {
        // ---- TMA producer (both CTAs) ----
        if (lane == 0) {
            asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tm_hi)) : "memory");
            asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tm_lo)) : "memory");
            asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tmb_hi)) : "memory");
            asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tmb_lo)) : "memory");
            uint32_t cg = 0;
            for (int t = cid; t < ntiles && !s_abort; t += ncl) {
                int p, bj;
                pair_tile(t, tgrid, p, bj);
                const int arow = (2 * p + (int)rank) * GT_BM;        // this CTA's A rows
                const int brow = bj * GT_BM + (int)rank * (GT_BM / 2);  // this CTA's half of the B panel
                for (int c = 0; c < nchunks; ++c, ++cg) {
                    const int s = (int)(cg % G2_STAGES);
                    if (cg >= G2_STAGES &&
                        !mbar_wait(smem_u32(&empty_bar[s]), (uint32_t)((cg / G2_STAGES - 1) & 1), &s_abort)) {
                        s_abort = 1;
                        break;
                    }
                    const uint32_t fb = smem_u32(&full_bar[s]);
                    if (leader)
                        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(fb),
                                     "r"(2 * G2_STAGE)
                                     : "memory");
                    const uint32_t fb0 = map_rank(fb, 0);
                    const uint32_t st = smem_u32(smem + (size_t)s * G2_STAGE);
                    const int x = c * GT_BK;
                    tma_load_pair(st, &tm_hi, fb0, x, arow);
                    tma_load_pair(st + G2_ATILE, &tm_lo, fb0, x, arow);
                    tma_load_pair(st + 2 * G2_ATILE, &tmb_hi, fb0, x, brow);
                    tma_load_pair(st + 2 * G2_ATILE + G2_BTILE, &tmb_lo, fb0, x, brow);
                }
            }
        }
    } else if (warp == 1) {
        // ---- MMA issuer (the even CTA) ----
        if (lane == 0 && leader) {
            uint32_t cg = 0, gg = 0;
            for (int t = cid; t < ntiles && !s_abort; t += ncl) {
                int c = 0;
                for (int g = 0; g < nseg && !s_abort; ++g, ++gg) {
                    const int buf = (int)(gg & 1);
                    if (gg >= 2 &&
                        !mbar_wait_cl(smem_u32(&acc_empty[buf]), (uint32_t)((gg / 2 - 1) & 1), &s_abort)) {
                        s_abort = 1;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const uint32_t d1 = tmem + (uint32_t)(buf * 256), d2 = d1 + 128;
                    const int cend = min(nchunks, (g + 1) * kseg);
                    for (int first = 1; c < cend; ++c, ++cg, first = 0) {
                        const int s = (int)(cg % G2_STAGES);
                        if (!mbar_wait(smem_u32(&full_bar[s]), (uint32_t)((cg / G2_STAGES) & 1), &s_abort)) {
                            s_abort = 1;
                            break;
                        }
                        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                        const uint32_t st = smem_u32(smem + (size_t)s * G2_STAGE);
#pragma unroll
                        for (int ks = 0; ks < GT_BK / 16; ++ks) {
                            const uint32_t ko = 32u * ks;
                            const uint64_t a_hi = desc_sw128(st + ko), a_lo = desc_sw128(st + G2_ATILE + ko);
                            const uint64_t b_hi = desc_sw128(st + 2 * G2_ATILE + ko),
                                           b_lo = desc_sw128(st + 2 * G2_ATILE + G2_BTILE + ko);
                            const uint32_t acc = (first && ks == 0) ? 0u : 1u;
                            mma_f16_pair(d1, a_hi, b_hi, acc);
                            mma_f16_pair(d2, a_hi, b_lo, acc);
                            mma_f16_pair(d2, a_lo, b_hi, 1u);
                        }
                        commit_pair(smem_u32(&empty_bar[s]));
                    }
                    if (s_abort) break;
                    commit_pair(smem_u32(&acc_full[buf]));
                }
            }
        }
    } else {
        // ---- epilogue (both CTAs): FP64 running sums of this CTA's 128 rows ----
        constexpr int EC = GT_BM / 2;
        const int q = warp & 3, half = (warp - 2) >> 2;
        uint32_t gg = 0;
        bool ok = true;
        for (int t = cid; t < ntiles && ok; t += ncl) {
            int p, bj;
            pair_tile(t, tgrid, p, bj);
            const int bi = 2 * p + (int)rank;
            double acc[EC];
#pragma unroll
            for (int i = 0; i < EC; ++i) acc[i] = 0.0;
            for (int g = 0; g < nseg; ++g, ++gg) {
                const int buf = (int)(gg & 1);
                const bool got = mbar_wait(smem_u32(&acc_full[buf]), (uint32_t)((gg / 2) & 1), &s_abort);
                if (!__all_sync(0xffffffffu, got)) {
                    ok = false;
                    s_abort = 1;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t base = tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(buf * 256 + half * EC);
#pragma unroll
                for (int cc = 0; cc < EC; cc += 8) {
                    float v1[8], v2[8];
                    tmem_ld8(base + cc, v1);
                    tmem_ld8(base + 128 + cc, v2);
                    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
                    for (int i = 0; i < 8; ++i) acc[cc + i] += (double)fmaf(v2[i], 4.8828125e-4f, v1[i]);
                }
                asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                __syncwarp();
                if (lane == 0)
                    asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(
                                     map_rank(smem_u32(&acc_empty[buf]), 0))
                                 : "memory");
            }
            // the even CTA's half of the pair's diagonal column (bi < bj) lies above the diagonal
            if (ok && bi >= bj) {
                const int r = bi * GT_BM + 32 * q + lane;
                const int c0 = bj * GT_BM + half * EC;
                if (C) {
                    double* stg = s_stage[warp - 2];
                    const int pw0 = (bi * GT_BM + 32 * q) >> 1;
                    const int qc = (c0 >> 1) + lane;
#pragma unroll
                    for (int c4 = 0; c4 < 4; ++c4) {
                        if ((lane >> 3) == c4) {
#pragma unroll
                            for (int m = 0; m < EC; ++m) stg[(lane & 7) * GT_STG_LD + m] = acc[m];
                        }
                        __syncwarp();
                        double nre[4], nim[4], ore[4], oim[4];
#pragma unroll
                        for (int ri = 0; ri < 4; ++ri) {
                            const double* e = stg + (2 * ri) * GT_STG_LD + 2 * lane;
                            const double* o = stg + (2 * ri + 1) * GT_STG_LD + 2 * lane;
                            const int pr = pw0 + 4 * c4 + ri;
                            nre[ri] = e[0] + o[1];
                            nim[ri] = pr == qc ? 0.0 : e[1] - o[0];
                            ore[ri] = oim[ri] = 0.0;
                            if (accumulate && pr < n && qc < n) {
                                const OT* ot = out + 2 * ((int64_t)pr * ldo + qc);
                                ore[ri] = (double)ot[0];
                                oim[ri] = (double)ot[1];
                            }
                        }
#pragma unroll
                        for (int ri = 0; ri < 4; ++ri) {
                            const int pr = pw0 + 4 * c4 + ri;
                            if (pr < n && qc < n) {
                                OT* ot = out + 2 * ((int64_t)pr * ldo + qc);
                                ot[0] = (OT)(ore[ri] + alpha * nre[ri]);
                                ot[1] = (OT)(oim[ri] + alpha * nim[ri]);
                            }
                        }
                        __syncwarp();
                    }
                } else if (r < n) {
                    OT* orow = out + (int64_t)r * ldo + c0;
                    double old[EC];
#pragma unroll
                    for (int m = 0; m < EC; ++m) old[m] = (accumulate && c0 + m < n) ? (double)orow[m] : 0.0;
#pragma unroll
                    for (int m = 0; m < EC; ++m)
                        if (c0 + m < n) orow[m] = (OT)(old[m] + alpha * acc[m]);
                }
            }
        }
    }
    if (s_abort && tid == 0) atomicExch(err, BEM_ERR_TIMEOUT);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    cluster_sync_all();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (warp == 1)
        asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(GT_TMEM_COLS) : "memory");
}

// ---------------------------------------------------------------------------
// FP64 Gram kernel (plain path): DMMA m8n8k4 on 128 x 128 real tiles of
// S = R^T R, R the real view of [A; P] (rows k), read directly; the column
// scaling is applied in the epilogue.
// ---------------------------------------------------------------------------
constexpr int GD_BM = 128, GD_BK = 16, GD_LD = GD_BM + 8;
constexpr int GD_SMEM = 2 * 2 * GD_BK * GD_LD * (int)sizeof(double);

__device__ __forceinline__ void cp_async16(void* dst, const void* src, bool valid) {
    const uint32_t d = smem_u32(dst);
    const int bytes = valid ? 16 : 0;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(src), "r"(bytes) : "memory");
}

__device__ __forceinline__ void cp_async8(void* dst, const void* src, bool valid) {
    const uint32_t d = smem_u32(dst);
    const int bytes = valid ? 8 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(d), "l"(src), "r"(bytes) : "memory");
}

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

template <bool C, typename OT>
__global__ void __launch_bounds__(256) gram_f64_kernel(const double* A, const double* P, int64_t ld, int n,
                                                       const double* d, OT* out, int64_t ldo, int tgrid, int band) {
    extern __shared__ __align__(16) double sm[];
    double* As = sm;                       // [2][GD_BK][GD_LD]
    double* Bs = sm + 2 * GD_BK * GD_LD;   // [2][GD_BK][GD_LD]
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    int bi, bj;
    tri_tile(blockIdx.x, tgrid, band, bi, bj);
    const int W = C ? 2 : 1;
    const int ncol = W * n;       // real columns of R
    const int K = 2 * n;          // rows of R
    const int i0 = bi * GD_BM, j0 = bj * GD_BM;
    const int wi = warp & 1, wj = warp >> 1;  // warp tile 64 x 32
    double acc[8][4][2];
#pragma unroll
    for (int a = 0; a < 8; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;

    // stage loader: 16 rows x 128 doubles of each operand (2048 pairs of
    // doubles), 16 bytes per cp.async for complex rows (16-byte aligned), two
    // 8-byte copies for real rows (any even or odd leading dimension)
    auto load = [&](int stage, int k0) {
#pragma unroll
        for (int h = 0; h < 8; ++h) {
            const int u = tid + 256 * h;  // operand (u >> 10), row, pair of doubles
            const int opnd = u >> 10, v = u & 1023;
            const int kr = v >> 6, cp = (v & 63) * 2;
            const int k = k0 + kr;
            const int col = (opnd ? j0 : i0) + cp;
            const double* row = (k < n ? A + (int64_t)k * ld * W : P + (int64_t)(k - n) * ld * W);
            double* dst = (opnd ? Bs : As) + (stage * GD_BK + kr) * GD_LD + cp;
            if (C) {
                const bool ok = k < K && col < ncol;
                cp_async16(dst, ok ? row + col : A, ok);
            } else {
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const bool ok = k < K && col + e < ncol;
                    cp_async8(dst + e, ok ? row + col + e : A, ok);
                }
            }
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    const int nk = (K + GD_BK - 1) / GD_BK;
    load(0, 0);
    for (int kt = 0; kt < nk; ++kt) {
        const int stage = kt & 1;
        if (kt + 1 < nk) {
            load(stage ^ 1, (kt + 1) * GD_BK);
            asm volatile("cp.async.wait_group 1;" ::: "memory");
        } else {
            asm volatile("cp.async.wait_group 0;" ::: "memory");
        }
        __syncthreads();
        const double* as = As + stage * GD_BK * GD_LD;
        const double* bs = Bs + stage * GD_BK * GD_LD;
#pragma unroll
        for (int k4 = 0; k4 < GD_BK; k4 += 4) {
            const int kr = k4 + (lane & 3);
            double af[8], bf[4];
#pragma unroll
            for (int a = 0; a < 8; ++a) af[a] = as[kr * GD_LD + wi * 64 + a * 8 + (lane >> 2)];
#pragma unroll
            for (int b = 0; b < 4; ++b) bf[b] = bs[kr * GD_LD + wj * 32 + b * 8 + (lane >> 2)];
#pragma unroll
            for (int a = 0; a < 8; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) dmma(acc[a][b][0], acc[a][b][1], af[a], bf[b]);
        }
        __syncthreads();
    }
    // epilogue: acc[a][b][e] = S[i0 + wi*64 + a*8 + lane/4][j0 + wj*32 + b*8 + 2*(lane%4) + e]
#pragma unroll
    for (int a = 0; a < 8; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            const int r = i0 + wi * 64 + a * 8 + (lane >> 2);
            const int cc = j0 + wj * 32 + b * 8 + 2 * (lane & 3);
            if (C) {
                // rows 2p / 2p+1 sit in lanes L / L + 4
                const double o0 = __shfl_xor_sync(0xffffffffu, acc[a][b][0], 4);
                const double o1 = __shfl_xor_sync(0xffffffffu, acc[a][b][1], 4);
                if (((lane >> 2) & 1) == 0) {
                    const int p = r >> 1, qc = cc >> 1;
                    if (p < n && qc < n) {
                        const double s = d[p] * d[qc];
                        const double re = acc[a][b][0] + o1, im = p == qc ? 0.0 : acc[a][b][1] - o0;
                        out[2 * ((int64_t)p * ldo + qc)] = (OT)(s * re);
                        out[2 * ((int64_t)p * ldo + qc) + 1] = (OT)(s * im);
                    }
                }
            } else if (r < n) {
#pragma unroll
                for (int e = 0; e < 2; ++e)
                    if (cc + e < n) out[(int64_t)r * ldo + cc + e] = (OT)(d[r] * d[cc + e] * acc[a][b][e]);
            }
        }
}

// N[p][q] = conj(N[q][p]) for q > p (T = float or double; C: complex pairs)
template <typename T, bool C>
__global__ void mirror_kernel(T* out, int64_t ldo, int n) {
    const int bx = blockIdx.x, by = blockIdx.y;
    if (bx < by) return;  // blocks with column block >= row block
    __shared__ T re[32][33], im[32][33];
    const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
    const int W = C ? 2 : 1;
    for (int yy = ty; yy < 32; yy += 8) {
        // source: rows from the column block, columns from the row block (the lower part)
        const int sr = bx * 32 + yy, sc = by * 32 + tx;
        if (sr < n && sc < n) {
            re[yy][tx] = out[W * ((int64_t)sr * ldo + sc)];
            if (C) im[yy][tx] = out[W * ((int64_t)sr * ldo + sc) + 1];
        }
    }
    __syncthreads();
    for (int yy = ty; yy < 32; yy += 8) {
        const int dr = by * 32 + yy, dc = bx * 32 + tx;
        if (dr < n && dc < n && dc > dr) {
            out[W * ((int64_t)dr * ldo + dc)] = re[tx][yy];
            if (C) out[W * ((int64_t)dr * ldo + dc) + 1] = -im[tx][yy];
        }
    }
}

// ---------------------------------------------------------------------------
// products of the refinement
// ---------------------------------------------------------------------------
// y[p] (+)= scale_p * sum_k conj(M1[k][p]) x1[k] + conj(M2[k][p]) x2[k] over a
// chunk of rows k (grid.y), added atomically; columns along threads
constexpr int GH_ROWS = 256;
template <bool C>
__global__ void __launch_bounds__(256) gemvh2_kernel(const double* M1, const double* M2, int64_t ld, int n,
                                                     const double* x1, const double* x2, double* y) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const int k0 = blockIdx.y * GH_ROWS, k1 = min(2 * n, k0 + GH_ROWS);
    double ar = 0.0, ai = 0.0;
    for (int k = k0; k < k1; ++k) {
        const bool top = k < n;
        const int kk = top ? k : k - n;
        const double* row = (top ? M1 : M2) + (int64_t)kk * ld * (C ? 2 : 1);
        const double* xv = top ? x1 : x2;
        if (C) {
            const double2 m = reinterpret_cast<const double2*>(row)[p];
            const double xr = xv[2 * kk], xi = xv[2 * kk + 1];
            ar += m.x * xr + m.y * xi;
            ai += m.x * xi - m.y * xr;
        } else {
            ar += row[p] * xv[kk];
        }
    }
    if (C) {
        atomicAdd(y + 2 * p, ar);
        atomicAdd(y + 2 * p + 1, ai);
    } else {
        atomicAdd(y + p, ar);
    }
}

// v[p] *= d[p] (complex pairs when C)
template <bool C>
__global__ void dscale_kernel(double* v, const double* d, int n) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    if (C) {
        v[2 * p] *= d[p];
        v[2 * p + 1] *= d[p];
    } else {
        v[p] *= d[p];
    }
}

// dst = src / d (d a power of two: exact)
template <bool C>
__global__ void dunscale_copy_kernel(double* dst, const double* src, const double* d, int n) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    if (C) {
        dst[2 * p] = src[2 * p] / d[p];
        dst[2 * p + 1] = src[2 * p + 1] / d[p];
    } else {
        dst[p] = src[p] / d[p];
    }
}

template <bool C>
__global__ void dscale_copy_kernel(double* dst, const double* src, const double* d, int n) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    if (C) {
        dst[2 * p] = src[2 * p] * d[p];
        dst[2 * p + 1] = src[2 * p + 1] * d[p];
    } else {
        dst[p] = src[p] * d[p];
    }
}

PFN_cuTensorMapEncodeTiled_v12000 encode_tiled() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
        else
            cudaGetLastError();
    });
    return fn;
}

int big_ws(bem_ctx* ctx, size_t bytes, void** out) {
    if (bytes > ctx->big_ws_bytes) {
        if (ctx->big_ws) cudaFree(ctx->big_ws);
        ctx->big_ws = nullptr;
        ctx->big_ws_bytes = 0;
        if (int rc = bem_check_cuda(ctx, cudaMalloc(&ctx->big_ws, bytes), "cudaMalloc(normal-matrix workspace)"))
            return rc;
        ctx->big_ws_bytes = bytes;
    }
    *out = ctx->big_ws;
    return BEM_OK;
}

int column_scale(bem_ctx* ctx, bool C, const double* A, const double* P, int64_t ld, int n, double* d,
                 cudaStream_t s) {
    // cn2 lives in d itself, then is replaced by the scale
    if (int rc = bem_check_cuda(ctx, cudaMemsetAsync(d, 0, sizeof(double) * n, s), "colnorm memset")) return rc;
    dim3 grid((unsigned)((n + 255) / 256), (unsigned)((2 * n + CN_ROWS - 1) / CN_ROWS));
    if (C)
        colnorm_kernel<true><<<grid, 256, 0, s>>>(A, P, ld, n, d);
    else
        colnorm_kernel<false><<<grid, 256, 0, s>>>(A, P, ld, n, d);
    colscale_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(d, d, n);
    ctx->launches += 2;
    return bem_check_cuda(ctx, cudaGetLastError(), "column scale");
}

template <bool C, typename OT>
int launch_gram_tc(bem_ctx* ctx, __half* Thi, __half* Tlo, int64_t Rp, int64_t Kp, OT* out, int64_t ldo, int n,
                   double alpha, int accumulate, cudaStream_t s);

template <bool C, typename OT>
int gram_mixed(bem_ctx* ctx, const double* A, const double* P, int64_t ld, int n, const double* d, OT* out,
               int64_t ldo, cudaStream_t s) {
    const int W = C ? 2 : 1;
    const int64_t rows = (int64_t)W * n;                    // rows of T
    // padded rows: a whole number of 256-row CTA-pair tiles (the split writes the padding as zeros)
    const int64_t Rp = (rows + 2 * GT_BM - 1) / (2 * GT_BM) * (2 * GT_BM);
    const int64_t Kp = (2 * (int64_t)n + GT_BK - 1) / GT_BK * GT_BK;
    if (Kp > (int64_t)1 << 31 || Rp / GT_BM > 65535) return bem_fail(ctx, BEM_ERR_INVALID, "gram: n too large");
    void* ws = nullptr;
    const size_t arr = (size_t)Rp * (size_t)Kp * sizeof(__half);
    if (int rc = big_ws(ctx, 2 * arr, &ws)) return rc;
    __half* Thi = static_cast<__half*>(ws);
    __half* Tlo = reinterpret_cast<__half*>(static_cast<char*>(ws) + arr);
    {
        // the split covers every T row block of 32 columns (64 rows when complex) and K in blocks of 64
        const int64_t pcols = Rp / W;
        dim3 grid((unsigned)(pcols / 32), (unsigned)(Kp / 64));
        split_kernel<C><<<grid, 256, 0, s>>>(A, P, ld, n, d, Thi, Tlo, Kp);
        ctx->launches++;
        if (int rc = bem_check_cuda(ctx, cudaGetLastError(), "split_kernel")) return rc;
    }
    return launch_gram_tc<C, OT>(ctx, Thi, Tlo, Rp, Kp, out, ldo, n, 1.0, 0, s);
}

// The tcgen05 product over split operands Thi / Tlo (Rp x Kp FP16, row
// stride Kp): out = alpha S (+ out when accumulate), lower tiles of S.
template <bool C, typename OT>
int launch_gram_tc(bem_ctx* ctx, __half* Thi, __half* Tlo, int64_t Rp, int64_t Kp, OT* out, int64_t ldo, int n,
                   double alpha, int accumulate, cudaStream_t s) {
    PFN_cuTensorMapEncodeTiled_v12000 enc = encode_tiled();
    if (!enc) return bem_fail(ctx, BEM_ERR_CUDA, "gram: cuTensorMapEncodeTiled is not available");
    CUtensorMap tm[2];
    for (int h = 0; h < 2; ++h) {
        cuuint64_t gdim[2] = {(cuuint64_t)Kp, (cuuint64_t)Rp};
        cuuint64_t gstride[1] = {(cuuint64_t)Kp * sizeof(__half)};
        cuuint32_t box[2] = {(cuuint32_t)GT_BK, (cuuint32_t)GT_BM};
        cuuint32_t estr[2] = {1, 1};
        CUresult r = enc(&tm[h], CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2, h ? (void*)Tlo : (void*)Thi, gdim, gstride, box,
                         estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                         CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) return bem_fail(ctx, BEM_ERR_CUDA, "gram: cuTensorMapEncodeTiled failed");
    }
    const int tr = (int)(Rp / GT_BM);
    const int64_t tiles = (int64_t)tr * (tr + 1) / 2;
    cudaMemsetAsync(ctx->flags + 5, 0, sizeof(int32_t), s);
    const int kseg = ctx->tune[BEM_TUNE_GRAM_KSEG] > 0 ? ctx->tune[BEM_TUNE_GRAM_KSEG] : GT_KSEG_DEFAULT;
    const int form = ctx->tune[BEM_TUNE_GRAM_PAIR] > 0 ? ctx->tune[BEM_TUNE_GRAM_PAIR] : GRAM_PAIR_DEFAULT;
    if (form == 2 && ctx->num_sms >= 2) {
        // CTA pairs: the B panel's tensor maps load 64-row halves
        CUtensorMap tmb[2];
        for (int h = 0; h < 2; ++h) {
            cuuint64_t gdim[2] = {(cuuint64_t)Kp, (cuuint64_t)Rp};
            cuuint64_t gstride[1] = {(cuuint64_t)Kp * sizeof(__half)};
            cuuint32_t box[2] = {(cuuint32_t)GT_BK, (cuuint32_t)(GT_BM / 2)};
            cuuint32_t estr[2] = {1, 1};
            CUresult r = enc(&tmb[h], CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2, h ? (void*)Tlo : (void*)Thi, gdim, gstride,
                             box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
            if (r != CUDA_SUCCESS) return bem_fail(ctx, BEM_ERR_CUDA, "gram: cuTensorMapEncodeTiled failed");
        }
        if (tr % 2) return bem_fail(ctx, BEM_ERR_INVALID, "gram: CTA pairs need an even number of tile rows");
        const int64_t ptiles = pair_tiles(tr);
        if (int rc = bem_check_cuda(ctx, cudaFuncSetAttribute(gram_tc2_kernel<C, OT>,
                                                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                              (int)G2_SMEM),
                                    "gram_tc2_kernel smem"))
            return rc;
        const unsigned clusters = (unsigned)std::min<int64_t>(ptiles, ctx->num_sms / 2);
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(2 * clusters);
        cfg.blockDim = dim3(GT_THREADS);
        cfg.dynamicSmemBytes = G2_SMEM;
        cfg.stream = s;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = 2;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        cudaError_t e = cudaLaunchKernelEx(&cfg, gram_tc2_kernel<C, OT>, tm[0], tm[1], tmb[0], tmb[1],
                                           (int)(Kp / GT_BK), kseg, (int)ptiles, tr, out, ldo, n, alpha, accumulate,
                                           ctx->flags + 5);
        ctx->launches++;
        return bem_check_cuda(ctx, e, "gram_tc2_kernel");
    }
    const int band = ctx->tune[BEM_TUNE_GRAM_BAND] > 0 ? ctx->tune[BEM_TUNE_GRAM_BAND] : GRAM_BAND_DEFAULT;
    // persistent: one CTA per SM (its shared memory and 512 TMEM columns allow no second), tiles in turn
    const unsigned grid = (unsigned)std::min<int64_t>(tiles, ctx->num_sms);
    if (form == 3) {
        // sixteen epilogue warps, 32 columns of FP64 running sums per thread
        if (int rc = bem_check_cuda(ctx, cudaFuncSetAttribute(gram_tc_kernel<C, OT, 16>,
                                                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                              (int)GT_SMEM),
                                    "gram_tc_kernel smem"))
            return rc;
        gram_tc_kernel<C, OT, 16><<<grid, 64 + 32 * 16, GT_SMEM, s>>>(tm[0], tm[1], (int)(Kp / GT_BK), kseg,
                                                                       (int)tiles, tr, band, out, ldo, n, alpha,
                                                                       accumulate, ctx->flags + 5);
    } else {
        if (int rc = bem_check_cuda(ctx, cudaFuncSetAttribute(gram_tc_kernel<C, OT, GT_EPI_WARPS>,
                                                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                              (int)GT_SMEM),
                                    "gram_tc_kernel smem"))
            return rc;
        gram_tc_kernel<C, OT, GT_EPI_WARPS><<<grid, GT_THREADS, GT_SMEM, s>>>(tm[0], tm[1], (int)(Kp / GT_BK), kseg,
                                                                             (int)tiles, tr, band, out, ldo, n,
                                                                             alpha, accumulate, ctx->flags + 5);
    }
    ctx->launches++;
    return bem_check_cuda(ctx, cudaGetLastError(), "gram_tc_kernel");
}

template <bool C, typename OT>
int gram_fp64(bem_ctx* ctx, const double* A, const double* P, int64_t ld, int n, const double* d, OT* out,
              int64_t ldo, cudaStream_t s) {
    const int W = C ? 2 : 1;
    const int64_t rows = (int64_t)W * n;
    const int tr = (int)((rows + GD_BM - 1) / GD_BM);
    const int64_t tiles = (int64_t)tr * (tr + 1) / 2;
    if (int rc = bem_check_cuda(ctx, cudaFuncSetAttribute(gram_f64_kernel<C, OT>,
                                                          cudaFuncAttributeMaxDynamicSharedMemorySize, GD_SMEM),
                                "gram_f64_kernel smem"))
        return rc;
    const int band = ctx->tune[BEM_TUNE_GRAM_BAND] > 0 ? ctx->tune[BEM_TUNE_GRAM_BAND] : GRAM_BAND_DEFAULT;
    gram_f64_kernel<C, OT><<<(unsigned)tiles, 256, GD_SMEM, s>>>(A, P, ld, n, d, out, ldo, tr, band);
    ctx->launches++;
    return bem_check_cuda(ctx, cudaGetLastError(), "gram_f64_kernel");
}

template <typename T, bool C>
int mirror(bem_ctx* ctx, T* out, int64_t ldo, int n, cudaStream_t s) {
    const unsigned nb = (unsigned)((n + 31) / 32);
    mirror_kernel<T, C><<<dim3(nb, nb), dim3(32, 8), 0, s>>>(out, ldo, n);
    ctx->launches++;
    return bem_check_cuda(ctx, cudaGetLastError(), "mirror_kernel");
}

}  // namespace

int bem_big_ws(bem_ctx* ctx, size_t bytes, void** out) { return big_ws(ctx, bytes, out); }

int bem_herk_tc_update(bem_ctx* ctx, bool C, const double* L, int64_t ld, int m, int kb, double* out, int64_t ldo,
                       cudaStream_t s) {
    if (m <= 0 || kb <= 0) return BEM_OK;
    const int W = C ? 2 : 1;
    const int64_t Rp = ((int64_t)W * m + 2 * GT_BM - 1) / (2 * GT_BM) * (2 * GT_BM);  // whole CTA-pair tiles
    const int64_t Kp = ((int64_t)kb + GT_BK - 1) / GT_BK * GT_BK;
    if (Rp / GT_BM > 65535) return bem_fail(ctx, BEM_ERR_INVALID, "herk update: m too large");
    void* ws = nullptr;
    const size_t arr = (size_t)Rp * (size_t)Kp * sizeof(__half);
    if (int rc = big_ws(ctx, 2 * arr, &ws)) return rc;
    __half* Thi = static_cast<__half*>(ws);
    __half* Tlo = reinterpret_cast<__half*>(static_cast<char*>(ws) + arr);
    dim3 grid((unsigned)(Kp / 64), (unsigned)((Rp + 3) / 4));
    if (C)
        panel_split_kernel<true><<<grid, 256, 0, s>>>(L, ld, m, kb, Thi, Tlo, Kp, Rp);
    else
        panel_split_kernel<false><<<grid, 256, 0, s>>>(L, ld, m, kb, Thi, Tlo, Kp, Rp);
    ctx->launches++;
    if (int rc = bem_check_cuda(ctx, cudaGetLastError(), "panel_split_kernel")) return rc;
    return C ? launch_gram_tc<true, double>(ctx, Thi, Tlo, Rp, Kp, out, ldo, m, -1.0, 1, s)
             : launch_gram_tc<false, double>(ctx, Thi, Tlo, Rp, Kp, out, ldo, m, -1.0, 1, s);
}

extern "C" {

int bem_gram(bem_ctx* ctx, int dtype, const void* A, const void* P, int64_t n, int64_t ld, double* colscale,
             int method, int out_dtype, void* out, int64_t ldo, void* stream) {
    if (!ctx) return BEM_ERR_INVALID;
    if (!A || !P || !colscale || !out || n <= 0 || ld < n || ldo < n || n > (1 << 28))
        return bem_fail(ctx, BEM_ERR_INVALID, "gram: bad arguments");
    const bool C = dtype == BEM_C128;
    if (!C && dtype != BEM_F64) return bem_fail(ctx, BEM_ERR_INVALID, "gram: A and P must be F64 or C128");
    if (C && ((reinterpret_cast<uintptr_t>(A) | reinterpret_cast<uintptr_t>(P)) & 15))
        return bem_fail(ctx, BEM_ERR_INVALID, "gram: complex A and P must be 16-byte aligned");
    if (method != BEM_PREC_MIXED && method != BEM_PREC_FP64)
        return bem_fail(ctx, BEM_ERR_INVALID, "gram: method must be BEM_PREC_MIXED or BEM_PREC_FP64");
    const bool want_c = out_dtype == BEM_C64 || out_dtype == BEM_C128;
    if (want_c != C || (out_dtype != BEM_C64 && out_dtype != BEM_C128 && out_dtype != BEM_F32 && out_dtype != BEM_F64))
        return bem_fail(ctx, BEM_ERR_INVALID, "gram: output dtype does not match the input");
    cudaStream_t s = (cudaStream_t)stream;
    const double* a = (const double*)A;
    const double* p = (const double*)P;
    const int ni = (int)n;
    if (int rc = column_scale(ctx, C, a, p, ld, ni, colscale, s)) return rc;
    const bool lo = out_dtype == BEM_C64 || out_dtype == BEM_F32;
    const bool tc = method == BEM_PREC_MIXED;
    int rc;
    if (lo) {
        float* o = (float*)out;
        rc = tc ? (C ? gram_mixed<true, float>(ctx, a, p, ld, ni, colscale, o, ldo, s)
                     : gram_mixed<false, float>(ctx, a, p, ld, ni, colscale, o, ldo, s))
                : (C ? gram_fp64<true, float>(ctx, a, p, ld, ni, colscale, o, ldo, s)
                     : gram_fp64<false, float>(ctx, a, p, ld, ni, colscale, o, ldo, s));
        if (!rc) rc = C ? mirror<float, true>(ctx, o, ldo, ni, s) : mirror<float, false>(ctx, o, ldo, ni, s);
    } else {
        double* o = (double*)out;
        rc = tc ? (C ? gram_mixed<true, double>(ctx, a, p, ld, ni, colscale, o, ldo, s)
                     : gram_mixed<false, double>(ctx, a, p, ld, ni, colscale, o, ldo, s))
                : (C ? gram_fp64<true, double>(ctx, a, p, ld, ni, colscale, o, ldo, s)
                     : gram_fp64<false, double>(ctx, a, p, ld, ni, colscale, o, ldo, s));
        if (!rc) rc = C ? mirror<double, true>(ctx, o, ldo, ni, s) : mirror<double, false>(ctx, o, ldo, ni, s);
    }
    return rc;
}

// FGMRES on D (A^H A + P^H P) D z = g, x = D z, with g = D [A; P]^H b for
// the stacked right-hand side b (2n), or g = D b for a normal-equation
// right-hand side b (n; normal_rhs).
static int normal_refine(bem_ctx* ctx, int dtype, const void* A, const void* P, int64_t n, int64_t ld,
                         const double* colscale, int lu_dtype, const void* LU, int64_t ldlu, const int32_t* piv,
                         const void* dinv, const void* b, bool normal_rhs, void* x, double tol, int maxit,
                         int restart, double accept, int* iters, double* relres, void* stream) {
    if (!ctx) return BEM_ERR_INVALID;
    if (!A || !P || !colscale || !LU || !piv || !dinv || !b || !x || n <= 0 || ld < n || ldlu < n)
        return bem_fail(ctx, BEM_ERR_INVALID, "lstsq_refine: bad arguments");
    const bool C = dtype == BEM_C128;
    if (!C && dtype != BEM_F64) return bem_fail(ctx, BEM_ERR_INVALID, "lstsq_refine: A and P must be F64 or C128");
    const bool lu_c = lu_dtype == BEM_C64 || lu_dtype == BEM_C128;
    if (lu_c != C) return bem_fail(ctx, BEM_ERR_INVALID, "lstsq_refine: factor dtype does not match");
    // a timed-out tensor-core wait of the normal matrix leaves it invalid
    {
        int32_t e = 0;
        cudaStream_t s0 = (cudaStream_t)stream;
        cudaMemcpyAsync(&e, ctx->flags + 5, sizeof(int32_t), cudaMemcpyDeviceToHost, s0);
        if (int rc = bem_check_cuda(ctx, cudaStreamSynchronize(s0), "gram status")) return rc;
        if (e != 0) {
            cudaMemsetAsync(ctx->flags + 5, 0, sizeof(int32_t), s0);
            return bem_fail(ctx, BEM_ERR_TIMEOUT, "gram: a tensor-core wait hit its iteration cap");
        }
    }
    cudaStream_t s = (cudaStream_t)stream;
    const int W = C ? 2 : 1;
    const int ni = (int)n;
    const int64_t nd = (int64_t)W * n;
    const double* a = (const double*)A;
    const double* p = (const double*)P;
    const double* bb = (const double*)b;
    double* xx = (double*)x;
    // scratch: u (n), t1, t2 (n each), g (n), z (n)
    double* buf = nullptr;
    if (int rc = bem_check_cuda(ctx, cudaMallocAsync((void**)&buf, sizeof(double) * 5 * nd, s), "lstsq alloc"))
        return rc;
    double* u = buf;
    double* t1 = u + nd;
    double* t2 = t1 + nd;
    double* g = t2 + nd;
    double* z = g + nd;
    const unsigned vb = (unsigned)((n + 255) / 256);
    const dim3 hgrid(vb, (unsigned)((2 * n + GH_ROWS - 1) / GH_ROWS));
    auto gemvh = [&](const double* x1, const double* x2, double* y) -> int {
        if (int e = bem_check_cuda(ctx, cudaMemsetAsync(y, 0, sizeof(double) * nd, s), "gemvh memset")) return e;
        if (C)
            gemvh2_kernel<true><<<hgrid, 256, 0, s>>>(a, p, ld, ni, x1, x2, y);
        else
            gemvh2_kernel<false><<<hgrid, 256, 0, s>>>(a, p, ld, ni, x1, x2, y);
        if (C)
            dscale_kernel<true><<<vb, 256, 0, s>>>(y, colscale, ni);
        else
            dscale_kernel<false><<<vb, 256, 0, s>>>(y, colscale, ni);
        ctx->launches += 2;
        return bem_check_cuda(ctx, cudaGetLastError(), "gemvh2_kernel");
    };
    // op(z) = D (A^H A + P^H P) D z
    auto op = [&](const double* zz, double* w) -> int {
        if (C)
            dscale_copy_kernel<true><<<vb, 256, 0, s>>>(u, zz, colscale, ni);
        else
            dscale_copy_kernel<false><<<vb, 256, 0, s>>>(u, zz, colscale, ni);
        ctx->launches++;
        if (int e = bem_gemv(ctx, dtype, A, n, n, ld, u, t1, 1.0, 0.0, s)) return e;
        if (int e = bem_gemv(ctx, dtype, P, n, n, ld, u, t2, 1.0, 0.0, s)) return e;
        return gemvh(t1, t2, w);
    };
    auto precond = [&](double* v) -> int { return bem_lu_solve_tiled(ctx, lu_dtype, LU, n, ldlu, piv, dinv, v, s); };
    int rc = BEM_OK;
    if (normal_rhs) {
        if (C)
            dscale_copy_kernel<true><<<vb, 256, 0, s>>>(g, bb, colscale, ni);
        else
            dscale_copy_kernel<false><<<vb, 256, 0, s>>>(g, bb, colscale, ni);
        ctx->launches++;
        rc = bem_check_cuda(ctx, cudaGetLastError(), "normal rhs");
    } else {
        rc = gemvh(bb, bb + nd, g);
    }
    // x holds the initial guess in the original variables: z0 = x / d
    if (!rc) {
        if (C)
            dunscale_copy_kernel<true><<<vb, 256, 0, s>>>(z, xx, colscale, ni);
        else
            dunscale_copy_kernel<false><<<vb, 256, 0, s>>>(z, xx, colscale, ni);
        ctx->launches++;
        rc = bem_check_cuda(ctx, cudaGetLastError(), "lstsq init");
    }
    if (!rc) rc = bem_fgmres(ctx, C, n, op, precond, g, z, tol, maxit, restart, accept, iters, relres, s);
    if (!rc || rc == BEM_ERR_NOCONVERGE) {
        const int keep = rc;
        if (C)
            dscale_copy_kernel<true><<<vb, 256, 0, s>>>(xx, z, colscale, ni);
        else
            dscale_copy_kernel<false><<<vb, 256, 0, s>>>(xx, z, colscale, ni);
        ctx->launches++;
        rc = bem_check_cuda(ctx, cudaGetLastError(), "lstsq x = D z");
        if (!rc) rc = keep;
    }
    cudaFreeAsync(buf, s);
    return rc;
}

}  // extern "C"

int bem_lstsq_refine(bem_ctx* ctx, int dtype, const void* A, const void* P, int64_t n, int64_t ld,
                     const double* colscale, int lu_dtype, const void* LU, int64_t ldlu, const int32_t* piv,
                     const void* dinv, const void* b, void* x, double tol, int maxit, int restart, double accept,
                     int* iters, double* relres, void* stream) {
    return normal_refine(ctx, dtype, A, P, n, ld, colscale, lu_dtype, LU, ldlu, piv, dinv, b, false, x, tol, maxit,
                         restart, accept, iters, relres, stream);
}

int bem_normal_refine(bem_ctx* ctx, int dtype, const void* A, const void* P, int64_t n, int64_t ld,
                      const double* colscale, int lu_dtype, const void* LU, int64_t ldlu, const int32_t* piv,
                      const void* dinv, const void* g, void* x, double tol, int maxit, int restart, double accept,
                      int* iters, double* relres, void* stream) {
    return normal_refine(ctx, dtype, A, P, n, ld, colscale, lu_dtype, LU, ldlu, piv, dinv, g, true, x, tol, maxit,
                         restart, accept, iters, relres, stream);
}
