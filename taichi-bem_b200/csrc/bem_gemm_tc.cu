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
#include <algorithm>
#include <cstdlib>

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

bool tc_enabled() {
    static int state = -1;
    if (state < 0) {
        const char* e = std::getenv("BEM_DISABLE_TENSOR_CORES");
        state = (e && e[0] == '1') ? 0 : 1;
    }
    return state == 1;
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
