// Tensor-core (tcgen05, kind::tf32) trailing update of the FP32 LU factor:
// C -= A B with FP32 accuracy from three TF32 products per tile
// (A_hi B_hi + A_hi B_lo + A_lo B_hi, x = x_hi + x_lo with x_hi = x truncated
// to TF32's 19 bits), accumulated in TMEM in FP32.
//
// Complex matrices (interleaved re, im) are handled as ONE real GEMM:
//   A (m x k complex) is read as the real m x 2k matrix of its interleaved
//   floats, B (k x n complex) is expanded while it is staged into shared
//   memory into the real 2k x 2n matrix with 2x2 blocks [[re, im], [-im, re]],
//   and the real m x 2n product is exactly the interleaved complex C update.
//
// CTA: 256 threads, one 128 x 128 (real) tile of C.  K is staged in chunks of
// TC_KC = 16 real columns (two shared-memory stages, 64 KB per CTA, three
// CTAs per SM) in the K-major, no-swizzle canonical layout: element (r, k) of
// a 128 x 16 tile at byte
//   (r / 8) * 512 + (k / 4) * 128 + (r % 8) * 16 + (k % 4) * 4,
// i.e. 8 x 16-byte core matrices, leading byte offset 128 (next core matrix
// along K), stride byte offset 512 (next group of 8 rows).  Thread 0 issues
// the MMAs (M = 128, N = 128, K = 8 per instruction) and commits them to the
// stage's mbarrier; the other threads refill a stage only after that mbarrier
// reports the MMAs reading it complete.  Every wait is bounded; on timeout the
// kernel records an error, stops issuing work and releases its TMEM.
//
// The C tile a thread updates in the epilogue is read into registers before
// the main loop, so that the latency of that read overlaps the MMAs instead
// of following them (two CTAs per SM instead of three, about 10 % less time
// per update).
//
// Updates with fewer C tiles than SMs (the LU's next tile column and tile-row
// strip) split K over up to four CTAs per tile (gridDim.z); each adds its
// partial product to C with FP32 atomics instead of the read-ahead
// read-modify-write.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstdlib>
#include <mutex>

#include "bem_gemm.cuh"

namespace {

constexpr int TC_BM = 128;
constexpr int TC_BN = 128;
constexpr int TC_KC = 16;
constexpr int TC_THREADS = 256;
constexpr int TC_TILE_BYTES = TC_BM * TC_KC * 4;  // 8 KB per operand tile
constexpr uint32_t TC_SBO = TC_KC * 32;            // bytes per group of 8 rows (TC_KC/4 core matrices of 128 B)
constexpr int TC_STAGE_BYTES = 4 * TC_TILE_BYTES;  // A_hi, A_lo, B_hi, B_lo
constexpr int TC_STAGES = 2;
constexpr uint32_t TC_TMEM_COLS = 128;
constexpr uint32_t TC_SPIN_CAP = 1u << 22;

// Instruction descriptor (kind::tf32): D format F32 (bits 4-5 = 1), A and B
// format TF32 (bits 7-9 and 10-12 = 2), both K-major (bits 15, 16 = 0),
// N >> 3 at bits 17-22, M >> 4 at bits 24-28.
constexpr uint32_t TC_IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(TC_BN >> 3) << 17) |
                              ((uint32_t)(TC_BM >> 4) << 24);

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor: start address >> 4 (bits 0-13), leading
// byte offset >> 4 (16-29), stride byte offset >> 4 (32-45), descriptor
// version 1 (46-47), base offset 0, no swizzle (layout type 0, bits 61-63).
__device__ __forceinline__ uint64_t make_desc(uint32_t saddr) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((128u >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((TC_SBO >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

__device__ __forceinline__ void split_tf32(float x, float& hi, float& lo) {
    hi = __uint_as_float(__float_as_uint(x) & 0xFFFFE000u);
    lo = x - hi;
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

__device__ __forceinline__ bool mbar_wait(uint32_t addr, uint32_t parity) {
    for (uint32_t it = 0; it < TC_SPIN_CAP; ++it)
        if (mbar_try(addr, parity)) return true;
    return false;
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(TC_IDESC), "r"(accumulate)
        : "memory");
}

__global__ void __launch_bounds__(TC_THREADS) gemm_tc_kernel(float* __restrict__ Cm, const float* __restrict__ Am,
                                                             const float* __restrict__ Bm, int m, int n_real,
                                                             int k_real, int64_t ldf, int cplx, int chunks_per,
                                                             int32_t* err) {
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ __align__(8) uint64_t mbar[TC_STAGES];
    __shared__ uint32_t tmem_slot;
    __shared__ int s_abort;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.y * TC_BM;
    const int n0 = blockIdx.x * TC_BN;
    // rows of A can be read as float4 when the base and the row stride are 16-byte aligned
    const bool a_vec = ((reinterpret_cast<uintptr_t>(Am) & 15) == 0) && ((ldf & 3) == 0);

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&tmem_slot)),
                     "r"(TC_TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int s = 0; s < TC_STAGES; ++s)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&mbar[s])) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_abort = 0;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_slot;

    // the C tile of this thread's epilogue: TMEM lane row e_row, 64 columns from e_cbase
    const int e_row = 32 * (warp & 3) + lane;
    const int e_cbase = 64 * (warp >> 2);
    // split K (gridDim.z > 1): this CTA takes chunks [c_begin, c_end) and adds
    // its partial product to C atomically, so it reads no C tile ahead
    const bool split = gridDim.z > 1;
    const int nchunks_all = (k_real + TC_KC - 1) / TC_KC;
    const int c_begin = blockIdx.z * chunks_per;
    const int c_end = min(nchunks_all, c_begin + chunks_per);
    float cpre[64];
    if (!split) {
        const int gr = m0 + e_row;
        const float* crow = Cm + (int64_t)(gr < m ? gr : 0) * ldf;
#pragma unroll
        for (int cc = 0; cc < 64; cc += 16) {
            const int gc0 = n0 + e_cbase + cc;
            if (gr < m && gc0 + 16 <= n_real && ((reinterpret_cast<uintptr_t>(crow + gc0) & 15) == 0)) {
#pragma unroll
                for (int i = 0; i < 16; i += 4) {
                    const float4 cv = *reinterpret_cast<const float4*>(crow + gc0 + i);
                    cpre[cc + i] = cv.x;
                    cpre[cc + i + 1] = cv.y;
                    cpre[cc + i + 2] = cv.z;
                    cpre[cc + i + 3] = cv.w;
                }
            } else {
#pragma unroll
                for (int i = 0; i < 16; ++i) cpre[cc + i] = (gr < m && gc0 + i < n_real) ? crow[gc0 + i] : 0.f;
            }
        }
    }
    const int nchunks = c_end - c_begin;  // local chunk lc is global chunk c_begin + lc
    // Software pipeline: the global loads of chunk c+1 are issued into
    // registers right after chunk c is stored, so their latency overlaps the
    // MMAs of chunk c and the wait for the stage to be free again.
    constexpr int UPT = TC_BM * TC_KC / 4 / TC_THREADS;  // staging units per thread
    float ra[UPT][4], rb[UPT][4];
    auto load_chunk = [&](int c) {
        const int kc = c * TC_KC;
#pragma unroll
        for (int h = 0; h < UPT; ++h) {
            const int u = tid + h * TC_THREADS;
            const int r = 8 * (u / (2 * TC_KC)) + (u & 7), k4 = (u >> 3) % (TC_KC / 4);
            const int kk0 = kc + 4 * k4;
            const bool rowok = m0 + r < m;
            const float* arow = Am + (int64_t)(m0 + r) * ldf + kk0;
            if (rowok && kk0 + 3 < k_real && a_vec) {
                const float4 v = *reinterpret_cast<const float4*>(arow);
                ra[h][0] = v.x;
                ra[h][1] = v.y;
                ra[h][2] = v.z;
                ra[h][3] = v.w;
            } else {
#pragma unroll
                for (int i = 0; i < 4; ++i) ra[h][i] = (rowok && kk0 + i < k_real) ? arow[i] : 0.f;
            }
            if (!cplx) {
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const int kk = kk0 + i;
                    rb[h][i] = (n0 + r < n_real && kk < k_real) ? Bm[(int64_t)kk * ldf + n0 + r] : 0.f;
                }
            } else {
                // complex rows q0, q0+1 of column col: (re, im) of each
                const int jc = r >> 1;
                const int q0 = kc / 2 + 2 * k4, col = n0 / 2 + jc;
                // one 8-byte load per complex value (interleaved re, im; 2 * col is even)
                rb[h][0] = rb[h][1] = rb[h][2] = rb[h][3] = 0.f;
                if (2 * col < n_real) {
                    if (2 * q0 < k_real) {
                        const float2 v = *reinterpret_cast<const float2*>(Bm + (int64_t)q0 * ldf + 2 * col);
                        rb[h][0] = v.x;
                        rb[h][1] = v.y;
                    }
                    if (2 * (q0 + 1) < k_real) {
                        const float2 v = *reinterpret_cast<const float2*>(Bm + (int64_t)(q0 + 1) * ldf + 2 * col);
                        rb[h][2] = v.x;
                        rb[h][3] = v.y;
                    }
                }
            }
        }
    };
    if (nchunks > 0) load_chunk(c_begin);
    for (int c = 0; c < nchunks; ++c) {
        const int stage = c & 1;
        unsigned char* st = smem + stage * TC_STAGE_BYTES;
        if (c >= TC_STAGES) {
            // the MMAs of chunk c-2 read this stage
            if (!mbar_wait(smem_addr(&mbar[stage]), (uint32_t)(((c - TC_STAGES) >> 1) & 1))) s_abort = 1;
        }
        __syncthreads();
        if (s_abort) break;
        // Staging: thread unit u owns one 16-byte core-matrix row, (row
        // 8*(u/(2*TC_KC)) + u%8, k-quad (u/8)%(TC_KC/4)), which sits at byte
        // 16*u of the tile, so a warp's shared-memory stores are contiguous.
#pragma unroll
        for (int h = 0; h < UPT; ++h) {
            const int u = tid + h * TC_THREADS;
            float4 hi, lo;
            split_tf32(ra[h][0], hi.x, lo.x);
            split_tf32(ra[h][1], hi.y, lo.y);
            split_tf32(ra[h][2], hi.z, lo.z);
            split_tf32(ra[h][3], hi.w, lo.w);
            *reinterpret_cast<float4*>(st + 16 * u) = hi;
            *reinterpret_cast<float4*>(st + TC_TILE_BYTES + 16 * u) = lo;
            // B stored K-major (row = output column); complex B expanded into
            // the real column 2*jc+s of [[re, im], [-im, re]] blocks
            float vb[4];
            if (!cplx) {
                vb[0] = rb[h][0];
                vb[1] = rb[h][1];
                vb[2] = rb[h][2];
                vb[3] = rb[h][3];
            } else if (((8 * (u / (2 * TC_KC)) + (u & 7)) & 1) == 0) {
                vb[0] = rb[h][0]; vb[1] = -rb[h][1]; vb[2] = rb[h][2]; vb[3] = -rb[h][3];
            } else {
                vb[0] = rb[h][1]; vb[1] = rb[h][0]; vb[2] = rb[h][3]; vb[3] = rb[h][2];
            }
            split_tf32(vb[0], hi.x, lo.x);
            split_tf32(vb[1], hi.y, lo.y);
            split_tf32(vb[2], hi.z, lo.z);
            split_tf32(vb[3], hi.w, lo.w);
            *reinterpret_cast<float4*>(st + 2 * TC_TILE_BYTES + 16 * u) = hi;
            *reinterpret_cast<float4*>(st + 3 * TC_TILE_BYTES + 16 * u) = lo;
        }
        if (c + 1 < nchunks) load_chunk(c_begin + c + 1);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t base = smem_addr(st);
#pragma unroll
            for (int ks = 0; ks < TC_KC / 8; ++ks) {
                const uint32_t koff = ks * 256;
                const uint64_t a_hi = make_desc(base + koff), a_lo = make_desc(base + TC_TILE_BYTES + koff);
                const uint64_t b_hi = make_desc(base + 2 * TC_TILE_BYTES + koff),
                               b_lo = make_desc(base + 3 * TC_TILE_BYTES + koff);
                const uint32_t acc0 = (c > 0 || ks > 0) ? 1u : 0u;
                mma_tf32(tmem, a_hi, b_hi, acc0);
                mma_tf32(tmem, a_hi, b_lo, 1u);
                mma_tf32(tmem, a_lo, b_hi, 1u);
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_addr(&mbar[stage]))
                         : "memory");
        }
    }
    // all MMAs are complete once the last chunk's commit has arrived
    if (!s_abort && nchunks > 0) {
        const int last = nchunks - 1;
        if (!mbar_wait(smem_addr(&mbar[last & 1]), (uint32_t)((last >> 1) & 1))) s_abort = 1;
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (!s_abort && nchunks > 0) {
        // epilogue: warp w reads TMEM lanes 32*(w%4).. (rows), columns half (w/4)
        const int row = 32 * (warp & 3) + lane;
        const int cbase = 64 * (warp >> 2);
#pragma unroll
        for (int cc = 0; cc < 64; cc += 16) {
            uint32_t v[16];
            const uint32_t taddr = tmem + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)(cbase + cc);
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
                "%13, %14, %15}, [%16];"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                  "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
                  "=r"(v[15])
                : "r"(taddr)
                : "memory");
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            const int gr = m0 + row;
            if (gr < m && split) {
                // partial product of this CTA's K range, added atomically
                float* crow = Cm + (int64_t)gr * ldf;
                const int gc0 = n0 + cbase + cc;
#pragma unroll
                for (int i = 0; i < 16; ++i) {
                    const int gc = gc0 + i;
                    if (gc < n_real) atomicAdd(crow + gc, -__uint_as_float(v[i]));
                }
            } else if (gr < m) {
                float* crow = Cm + (int64_t)gr * ldf;
                const int gc0 = n0 + cbase + cc;
                if (gc0 + 16 <= n_real && ((reinterpret_cast<uintptr_t>(crow + gc0) & 15) == 0)) {
#pragma unroll
                    for (int i = 0; i < 16; i += 4) {
                        float4 cv;
                        cv.x = cpre[cc + i] - __uint_as_float(v[i]);
                        cv.y = cpre[cc + i + 1] - __uint_as_float(v[i + 1]);
                        cv.z = cpre[cc + i + 2] - __uint_as_float(v[i + 2]);
                        cv.w = cpre[cc + i + 3] - __uint_as_float(v[i + 3]);
                        *reinterpret_cast<float4*>(crow + gc0 + i) = cv;
                    }
                } else {
#pragma unroll
                    for (int i = 0; i < 16; ++i) {
                        const int gc = gc0 + i;
                        if (gc < n_real) crow[gc] = cpre[cc + i] - __uint_as_float(v[i]);
                    }
                }
            }
        }
    } else if (tid == 0) {
        atomicExch(err, BEM_ERR_TIMEOUT);
        // give in-flight MMAs a bounded chance to finish before TMEM is released
        mbar_wait(smem_addr(&mbar[0]), 0);
        mbar_wait(smem_addr(&mbar[1]), 0);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_TMEM_COLS)
                     : "memory");
}

// ---------------------------------------------------------------------------
// TMA-fed persistent form of the same update (BEM_TUNE_LU_UPDATE = 2).  The
// operands are split once per update into TF32 hi / lo arrays in the K-major
// layout the MMA reads: A's real view (m x 2k floats, its rows as they lie)
// and the real expansion of B transposed, T_B[2q + b][2kk + a] =
// [[re, im], [-im, re]][a][b] of B[kk][q], so that A T_B^T is the interleaved
// complex product (lu_split_a_kernel, lu_split_b_kernel; zero padding to
// whole 128 x 32 tiles).  One persistent kernel then runs over the C tiles:
// warp 0 loads the four 128 x 32 FP32 tiles of a K stage by TMA
// (cp.async.bulk.tensor, 128-byte swizzle, three stages of 64 KB) on an
// mbarrier ring, warp 1 issues three kind::tf32 MMAs per K = 8 step into one
// of two TMEM accumulators, and sixteen epilogue warps move a finished tile out
// of TMEM, release it to the MMAs and subtract it from C, while the MMAs of
// the next tile run.  Every wait is bounded.  The tensor maps cover this
// GPU's memory only, and each TMA load fills this CTA's own shared memory.
// ---------------------------------------------------------------------------
constexpr int LT_BK = 32;                   // floats per K stage: 128 bytes, one swizzle span
constexpr int LT_TILE = TC_BM * LT_BK * 4;  // 16 KB
constexpr int LT_STAGE = 4 * LT_TILE;       // A_hi, A_lo, B_hi, B_lo
constexpr int LT_STAGES = 3;
constexpr int LT_EPI_WARPS = 16;  // four per TMEM lane quarter, 32 columns each
constexpr int LT_SR = 8;          // rows per pass of the epilogue's shared-memory transpose
constexpr int LT_THREADS = 64 + 32 * LT_EPI_WARPS;
constexpr uint32_t LT_TMEM_COLS = 256;  // two accumulators of 128 columns
constexpr size_t LT_SMEM = (size_t)LT_STAGES * LT_STAGE + 1024;

__device__ __forceinline__ uint64_t lt_desc_sw128(uint32_t saddr) {
    uint64_t dsc = 0;
    dsc |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    dsc |= (uint64_t)1 << 16;             // leading byte offset (unused by swizzled K-major layouts)
    dsc |= (uint64_t)(1024u >> 4) << 32;  // stride byte offset: 8 rows of 128 bytes
    dsc |= (uint64_t)1 << 46;             // descriptor version
    dsc |= (uint64_t)2 << 61;             // SWIZZLE_128B
    return dsc;
}

__device__ __forceinline__ void lt_tma_load(uint32_t dst, const CUtensorMap* map, uint32_t mbar, int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(
            dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(mbar), "r"(x), "r"(y)
        : "memory");
}

__device__ __forceinline__ bool lt_wait(uint32_t addr, uint32_t parity, volatile int* abort) {
    for (uint32_t it = 0; it < TC_SPIN_CAP; ++it) {
        if (mbar_try(addr, parity)) return true;
        if ((it & 1023u) == 1023u && *abort) return false;
    }
    return false;
}

// A (m rows of kr floats, row stride ldf) -> hi / lo [Mp x Kp]
__global__ void lu_split_a_kernel(const float* __restrict__ A, int64_t ldf, int m, int kr, float* hi, float* lo,
                                  int Kp, int64_t total) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= total) return;
    const int r = (int)(i / Kp), c = (int)(i - (int64_t)r * Kp);
    const float x = (r < m && c < kr) ? A[(int64_t)r * ldf + c] : 0.0f;
    float h, l;
    split_tf32(x, h, l);
    hi[i] = h;
    lo[i] = l;
}

// B (k x n, row stride ldf floats; complex interleaved when cplx) -> the rows
// of T_B (one per real column of C) over the real K index, hi / lo [Np x Kp]
__global__ void lu_split_b_kernel(const float* __restrict__ B, int64_t ldf, int k, int n, int cplx, float* hi,
                                  float* lo, int Kp, int64_t total) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= total) return;
    const int qq = (int)(i / Kp), kk2 = (int)(i - (int64_t)qq * Kp);
    float x = 0.0f;
    if (cplx) {
        const int q = qq >> 1, b = qq & 1, kk = kk2 >> 1, a = kk2 & 1;
        if (q < n && kk < k) {
            const float re = B[(int64_t)kk * ldf + 2 * q], im = B[(int64_t)kk * ldf + 2 * q + 1];
            x = a == 0 ? (b == 0 ? re : im) : (b == 0 ? -im : re);
        }
    } else if (qq < n && kk2 < k) {
        x = B[(int64_t)kk2 * ldf + qq];
    }
    float h, l;
    split_tf32(x, h, l);
    hi[i] = h;
    lo[i] = l;
}

__global__ void __launch_bounds__(LT_THREADS, 1) lu_tc_kernel(const __grid_constant__ CUtensorMap ta_hi,
                                                              const __grid_constant__ CUtensorMap ta_lo,
                                                              const __grid_constant__ CUtensorMap tb_hi,
                                                              const __grid_constant__ CUtensorMap tb_lo,
                                                              int nchunks, int tiles_m, int ntiles, float* C,
                                                              int64_t ldc, int m, int n_real, int32_t* err) {
    extern __shared__ unsigned char lt_smem_raw[];
    __shared__ __align__(8) uint64_t full_bar[LT_STAGES], empty_bar[LT_STAGES], acc_full[2], acc_empty[2];
    __shared__ uint32_t tmem_slot;
    __shared__ volatile int s_abort;
    __shared__ float s_stg[LT_EPI_WARPS][LT_SR][33];  // epilogue staging, LT_SR rows x 32 columns per warp
    unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(lt_smem_raw) + 1023) &
                                                           ~uintptr_t(1023));
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&tmem_slot)),
                     "r"(LT_TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int s = 0; s < LT_STAGES; ++s) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&full_bar[s])) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&empty_bar[s])) : "memory");
        }
        for (int b = 0; b < 2; ++b) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&acc_full[b])) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&acc_empty[b])),
                         "r"(LT_EPI_WARPS)
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
            uint32_t cg = 0;
            for (int t = blockIdx.x; t < ntiles && !s_abort; t += gridDim.x) {
                const int ti = t % tiles_m, tj = t / tiles_m;
                for (int c = 0; c < nchunks; ++c, ++cg) {
                    const int s = (int)(cg % LT_STAGES);
                    if (cg >= LT_STAGES &&
                        !lt_wait(smem_addr(&empty_bar[s]), (uint32_t)((cg / LT_STAGES - 1) & 1), &s_abort)) {
                        s_abort = 1;
                        break;
                    }
                    const uint32_t fb = smem_addr(&full_bar[s]);
                    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(fb), "r"(LT_STAGE)
                                 : "memory");
                    const uint32_t st = smem_addr(smem + (size_t)s * LT_STAGE);
                    const int x = c * LT_BK;
                    lt_tma_load(st, &ta_hi, fb, x, ti * TC_BM);
                    lt_tma_load(st + LT_TILE, &ta_lo, fb, x, ti * TC_BM);
                    lt_tma_load(st + 2 * LT_TILE, &tb_hi, fb, x, tj * TC_BN);
                    lt_tma_load(st + 3 * LT_TILE, &tb_lo, fb, x, tj * TC_BN);
                }
            }
        }
    } else if (warp == 1) {
        // ---- MMA issuer: one accumulator per tile, two alternating ----
        if (lane == 0) {
            uint32_t cg = 0, gg = 0;
            for (int t = blockIdx.x; t < ntiles && !s_abort; t += gridDim.x, ++gg) {
                const int buf = (int)(gg & 1);
                if (gg >= 2 && !lt_wait(smem_addr(&acc_empty[buf]), (uint32_t)((gg / 2 - 1) & 1), &s_abort)) {
                    s_abort = 1;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t d = tmem + (uint32_t)(buf * TC_BN);
                for (int c = 0; c < nchunks; ++c, ++cg) {
                    const int s = (int)(cg % LT_STAGES);
                    if (!lt_wait(smem_addr(&full_bar[s]), (uint32_t)((cg / LT_STAGES) & 1), &s_abort)) {
                        s_abort = 1;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const uint32_t st = smem_addr(smem + (size_t)s * LT_STAGE);
#pragma unroll
                    for (int ks = 0; ks < LT_BK / 8; ++ks) {
                        const uint32_t ko = 32u * ks;  // 8 floats
                        const uint64_t a_hi = lt_desc_sw128(st + ko), a_lo = lt_desc_sw128(st + LT_TILE + ko);
                        const uint64_t b_hi = lt_desc_sw128(st + 2 * LT_TILE + ko),
                                       b_lo = lt_desc_sw128(st + 3 * LT_TILE + ko);
                        mma_tf32(d, a_hi, b_hi, (c == 0 && ks == 0) ? 0u : 1u);
                        mma_tf32(d, a_hi, b_lo, 1u);
                        mma_tf32(d, a_lo, b_hi, 1u);
                    }
                    asm volatile(
                        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                            smem_addr(&empty_bar[s]))
                        : "memory");
                }
                if (s_abort) break;
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                 smem_addr(&acc_full[buf]))
                             : "memory");
            }
        }
    } else {
        // ---- epilogue: warp w reads TMEM lanes 32 (w % 4) .. and column group (w - 2) / 4 ----
        const int q = warp & 3, half = (warp - 2) >> 2;
        constexpr int EC = TC_BN / (LT_EPI_WARPS / 4);
        uint32_t gg = 0;
        for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++gg) {
            const int ti = t % tiles_m, tj = t / tiles_m;
            const int buf = (int)(gg & 1);
            const bool got = lt_wait(smem_addr(&acc_full[buf]), (uint32_t)((gg / 2) & 1), &s_abort);
            if (!__all_sync(0xffffffffu, got)) {
                s_abort = 1;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            float v[EC];
            const uint32_t base = tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(buf * TC_BN + half * EC);
#pragma unroll
            for (int cc = 0; cc < EC; cc += 32) {
                uint32_t u[32];
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
                    "%13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, "
                    "[%32];"
                    : "=r"(u[0]), "=r"(u[1]), "=r"(u[2]), "=r"(u[3]), "=r"(u[4]), "=r"(u[5]), "=r"(u[6]), "=r"(u[7]),
                      "=r"(u[8]), "=r"(u[9]), "=r"(u[10]), "=r"(u[11]), "=r"(u[12]), "=r"(u[13]), "=r"(u[14]),
                      "=r"(u[15]), "=r"(u[16]), "=r"(u[17]), "=r"(u[18]), "=r"(u[19]), "=r"(u[20]), "=r"(u[21]),
                      "=r"(u[22]), "=r"(u[23]), "=r"(u[24]), "=r"(u[25]), "=r"(u[26]), "=r"(u[27]), "=r"(u[28]),
                      "=r"(u[29]), "=r"(u[30]), "=r"(u[31])
                    : "r"(base + (uint32_t)cc)
                    : "memory");
#pragma unroll
                for (int i = 0; i < 32; ++i) v[cc + i] = __uint_as_float(u[i]);
            }
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0)
                asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(&acc_empty[buf])) : "memory");
            // C -= tile, 32 columns at a time through shared memory, so that
            // a warp's accesses run along rows of C (lane = column)
            const int row0 = ti * TC_BM + 32 * q;
            float(*stg)[33] = s_stg[warp - 2];
#pragma unroll
            for (int cc = 0; cc < EC; cc += 32) {
#pragma unroll
                for (int hr = 0; hr < 32 / LT_SR; ++hr) {  // rows LT_SR hr .. of the warp's 32
                    if (lane / LT_SR == hr) {
#pragma unroll
                        for (int i = 0; i < 32; ++i) stg[lane % LT_SR][i] = v[cc + i];
                    }
                    __syncwarp();
                    const int col = tj * TC_BN + half * EC + cc + lane;
                    const int rb = row0 + LT_SR * hr;
                    if (col < n_real) {
                        // all old values first (independent loads in flight), then the stores
                        float old[LT_SR];
#pragma unroll
                        for (int rr = 0; rr < LT_SR; ++rr)
                            old[rr] = rb + rr < m ? __ldcg(C + (int64_t)(rb + rr) * ldc + col) : 0.0f;
#pragma unroll
                        for (int rr = 0; rr < LT_SR; ++rr)
                            if (rb + rr < m) C[(int64_t)(rb + rr) * ldc + col] = old[rr] - stg[rr][lane];
                    }
                    __syncwarp();
                }
            }
        }
    }
    if (s_abort && tid == 0) atomicExch(err, BEM_ERR_TIMEOUT);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 1)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(LT_TMEM_COLS)
                     : "memory");
}

bool tc_enabled() {
    static int state = -1;
    if (state < 0) {
        const char* e = std::getenv("BEM_DISABLE_TENSOR_CORES");
        state = (e && e[0] == '1') ? 0 : 1;
    }
    return state == 1;
}

}  // namespace

namespace {

// form of the large trailing updates (BEM_TUNE_LU_UPDATE): 1 register-staged
// gemm_tc_kernel, 2 the TMA-fed persistent lu_tc_kernel (the default: measured
// 12.1 vs 13.4 ms for a 5120^2 complex factorisation, 39.9 vs 57.1 ms at 10240^2)
constexpr int LU_UPDATE_DEFAULT = 2;

PFN_cuTensorMapEncodeTiled_v12000 lt_encode() {
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

int lu_update_tma(bem_ctx* ctx, float* C, const float* A, const float* B, int64_t m, int64_t n, int64_t k,
                  int64_t ldf, bool cplx, cudaStream_t s) {
    PFN_cuTensorMapEncodeTiled_v12000 enc = lt_encode();
    if (!enc) return 1;
    const int64_t n_real = cplx ? 2 * n : n, k_real = cplx ? 2 * k : k;
    const int64_t Mp = (m + TC_BM - 1) / TC_BM * TC_BM, Np = (n_real + TC_BN - 1) / TC_BN * TC_BN;
    const int64_t Kp = (k_real + LT_BK - 1) / LT_BK * LT_BK;
    void* ws = nullptr;
    if (int rc = bem_big_ws(ctx, sizeof(float) * 2 * (size_t)(Mp + Np) * (size_t)Kp, &ws)) return rc;
    float* ahi = static_cast<float*>(ws);
    float* alo = ahi + Mp * Kp;
    float* bhi = alo + Mp * Kp;
    float* blo = bhi + Np * Kp;
    {
        const int64_t ta = Mp * Kp, tb = Np * Kp;
        lu_split_a_kernel<<<(unsigned)((ta + 255) / 256), 256, 0, s>>>(A, ldf, (int)m, (int)k_real, ahi, alo,
                                                                       (int)Kp, ta);
        lu_split_b_kernel<<<(unsigned)((tb + 255) / 256), 256, 0, s>>>(B, ldf, (int)k, (int)n, cplx ? 1 : 0, bhi,
                                                                       blo, (int)Kp, tb);
        ctx->launches += 2;
        if (int rc = bem_check_cuda(ctx, cudaGetLastError(), "lu_split kernels")) return rc;
    }
    CUtensorMap tm[4];
    float* srcs[4] = {ahi, alo, bhi, blo};
    for (int h = 0; h < 4; ++h) {
        cuuint64_t gdim[2] = {(cuuint64_t)Kp, (cuuint64_t)(h < 2 ? Mp : Np)};
        cuuint64_t gstride[1] = {(cuuint64_t)Kp * sizeof(float)};
        cuuint32_t box[2] = {(cuuint32_t)LT_BK, (cuuint32_t)TC_BM};
        cuuint32_t estr[2] = {1, 1};
        CUresult r = enc(&tm[h], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, srcs[h], gdim, gstride, box, estr,
                         CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) return bem_fail(ctx, BEM_ERR_CUDA, "lu update: cuTensorMapEncodeTiled failed");
    }
    const int tiles_m = (int)(Mp / TC_BM);
    const int64_t ntiles = (int64_t)tiles_m * (Np / TC_BN);
    if (int rc = bem_check_cuda(ctx, cudaFuncSetAttribute(lu_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                          (int)LT_SMEM),
                                "lu_tc_kernel smem"))
        return rc;
    const unsigned grid = (unsigned)std::min<int64_t>(ntiles, ctx->num_sms);
    lu_tc_kernel<<<grid, LT_THREADS, LT_SMEM, s>>>(tm[0], tm[1], tm[2], tm[3], (int)(Kp / LT_BK), tiles_m,
                                                   (int)ntiles, C, ldf, (int)m, (int)n_real, ctx->flags + 4);
    ctx->launches++;
    return bem_check_cuda(ctx, cudaGetLastError(), "lu_tc_kernel");
}

}  // namespace

int bem_gemm_tc_update(bem_ctx* ctx, float* C, const float* A, const float* B, int64_t m, int64_t n, int64_t k,
                       int64_t lda, bool cplx, cudaStream_t s) {
    if (!tc_enabled()) return 1;
    if (m <= 0 || n <= 0 || k <= 0) return BEM_OK;
    const int64_t ldf = cplx ? 2 * lda : lda;
    const int64_t n_real = cplx ? 2 * n : n, k_real = cplx ? 2 * k : k;
    if (m > (int64_t)65535 * TC_BM || n_real > (int64_t)1 << 30) return 1;
    const size_t smem = (size_t)TC_STAGES * TC_STAGE_BYTES;
    cudaFuncSetAttribute(gemm_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    dim3 grid((unsigned)((n_real + TC_BN - 1) / TC_BN), (unsigned)((m + TC_BM - 1) / TC_BM));
    // Skinny updates (the LU's tile-column and tile-row strips) fill few
    // CTAs: split K over up to four CTAs per C tile, each adding its partial
    // product atomically, until the grid covers the SMs.
    const int nchunks = (int)((k_real + TC_KC - 1) / TC_KC);
    const int64_t tiles = (int64_t)grid.x * grid.y;
    const int form = ctx->tune[BEM_TUNE_LU_UPDATE] > 0 ? ctx->tune[BEM_TUNE_LU_UPDATE] : LU_UPDATE_DEFAULT;
    if (form == 2 && tiles >= ctx->num_sms) {
        // large updates: the TMA-fed persistent kernel (skinny ones keep split K below)
        const int rc = lu_update_tma(ctx, C, A, B, m, n, k, ldf, cplx, s);
        if (rc <= 0) return rc;
    }
    int splits = 1;
    if (tiles < ctx->num_sms && nchunks >= 4)
        splits = (int)std::min<int64_t>(std::min<int64_t>(4, nchunks / 2), std::max<int64_t>(1, ctx->num_sms / tiles));
    const int per = (nchunks + splits - 1) / splits;
    grid.z = (unsigned)((nchunks + per - 1) / per);
    gemm_tc_kernel<<<grid, TC_THREADS, smem, s>>>(C, A, B, (int)m, (int)n_real, (int)k_real, ldf, cplx ? 1 : 0, per,
                                                  ctx->flags + 4);
    ctx->launches++;
    return bem_check_cuda(ctx, cudaGetLastError(), "gemm_tc_kernel");
}
