// Post-processing of the driver's per-vertex results into headless device
// buffers.  The reference ends BEMManager.run with two Taichi kernels that
// prepare its GGUI window (src/managers/BEM_manager.py:1028-1029):
//
//   compute_color      (BEM_manager.py:527-587)  shifts the solved Dirichlet
//                      traces onto the mean of the exact ones and maps the
//                      solved, exact and difference values to RGB colours;
//   set_mesh_instances (BEM_manager.py:589-606)  copies the vertices into
//                      three position buffers, the exact one moved by -2.2
//                      and the difference one by +2.2 along x.
//
// There is no window here: the colour and position buffers are plain device
// arrays [nv*3] float that a caller can write to a file or draw itself.  Both
// passes are tiny (O(nv)); they are launch-latency bound, not HBM bound.

#include <algorithm>

#include "bem_internal.cuh"

namespace {

constexpr int COLOR_THREADS = 1024;
constexpr int VT_DIRICHLET = 1;  // VertAttachType.DIRICHLET_TOBESOLVED (utils/types.py)
constexpr int NACC = 7;          // max_N, max_D, count_D, sum solved (re, im), sum exact (re, im)

// |v| of a 1- or 2-vector as ti.Vector.norm computes it: sqrt of the sum of
// squares, rounded per operation (no FMA contraction).
__device__ __forceinline__ double vnorm(double re, double im) {
    return sqrt(__dadd_rn(__dmul_rn(re, re), __dmul_rn(im, im)));
}

// One CTA: the reference's pass is a reduction over all vertices (maxima of
// the exact values per vertex class, mean of the solved and exact Dirichlet
// traces) followed by an elementwise pass that depends on its result, so a
// single block does both with one barrier between them.
//   n = 1 (real) or 2 (complex, interleaved) doubles per vertex;
//   show = the BEMManager._show value (-1, 0 Neumann, 1 Dirichlet).
__global__ void __launch_bounds__(COLOR_THREADS)
compute_color_kernel(int nv, int n, double* __restrict__ solved, const double* __restrict__ exact,
                     const int32_t* __restrict__ vtype, int show, float* __restrict__ solved_color,
                     float* __restrict__ exact_color, float* __restrict__ diff_color) {
    __shared__ double part[COLOR_THREADS / 32][NACC];
    __shared__ double tot[NACC];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

    // (1) per-class maxima and the Dirichlet sums (BEM_manager.py:543-553)
    double acc[NACC] = {-5e11, -5e11, 0.0, 0.0, 0.0, 0.0, 0.0};
    for (int i = tid; i < nv; i += COLOR_THREADS) {
        const double ar = exact[(int64_t)i * n], ai = n == 2 ? exact[(int64_t)i * n + 1] : 0.0;
        const double na = vnorm(ar, ai);
        if (vtype[i] != VT_DIRICHLET) {
            acc[0] = fmax(acc[0], na);
        } else {
            acc[1] = fmax(acc[1], na);
            acc[2] += 1.0;
            acc[3] += solved[(int64_t)i * n];
            acc[4] += n == 2 ? solved[(int64_t)i * n + 1] : 0.0;
            acc[5] += ar;
            acc[6] += ai;
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        acc[0] = fmax(acc[0], __shfl_down_sync(0xffffffffu, acc[0], off));
        acc[1] = fmax(acc[1], __shfl_down_sync(0xffffffffu, acc[1], off));
#pragma unroll
        for (int c = 2; c < NACC; ++c) acc[c] += __shfl_down_sync(0xffffffffu, acc[c], off);
    }
    if (lane == 0)
#pragma unroll
        for (int c = 0; c < NACC; ++c) part[warp][c] = acc[c];
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int c = 0; c < NACC; ++c) acc[c] = part[lane][c];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            acc[0] = fmax(acc[0], __shfl_down_sync(0xffffffffu, acc[0], off));
            acc[1] = fmax(acc[1], __shfl_down_sync(0xffffffffu, acc[1], off));
#pragma unroll
            for (int c = 2; c < NACC; ++c) acc[c] += __shfl_down_sync(0xffffffffu, acc[c], off);
        }
        if (lane == 0)
#pragma unroll
            for (int c = 0; c < NACC; ++c) tot[c] = acc[c];
    }
    __syncthreads();

    const double max_n = tot[0], max_d = tot[1], cnt = tot[2];
    double mean_s_re = tot[3], mean_s_im = tot[4], mean_a_re = tot[5], mean_a_im = tot[6];
    if (cnt > 0.0) {  // BEM_manager.py:554-556
        mean_s_re /= cnt;
        mean_s_im /= cnt;
        mean_a_re /= cnt;
        mean_a_im /= cnt;
    }
    const double shift_re = mean_a_re - mean_s_re, shift_im = mean_a_im - mean_s_im;

    // (2) shift, then colour (BEM_manager.py:558-587)
    for (int i = tid; i < nv; i += COLOR_THREADS) {
        const int t = vtype[i];
        double sr = solved[(int64_t)i * n], si = n == 2 ? solved[(int64_t)i * n + 1] : 0.0;
        if (t == VT_DIRICHLET || show == VT_DIRICHLET) {
            sr += shift_re;
            si += shift_im;
            solved[(int64_t)i * n] = sr;
            if (n == 2) solved[(int64_t)i * n + 1] = si;
        }
        const double ar = exact[(int64_t)i * n], ai = n == 2 ? exact[(int64_t)i * n + 1] : 0.0;
        const double m = (t != VT_DIRICHLET && show != VT_DIRICHLET) ? max_n : max_d;
        const float ca = (float)(vnorm(ar, ai) / m), cs = (float)(vnorm(sr, si) / m);
        const float acx = ar > 0.0 ? ca : 0.0f, acz = ar > 0.0 ? 0.0f : ca;
        const float scx = sr > 0.0 ? cs : 0.0f, scz = sr > 0.0 ? 0.0f : cs;
        // |s.x - a.x - s.z + a.z| in the colour buffers' float, left to right
        const float dy = fabsf(__fadd_rn(__fsub_rn(__fsub_rn(scx, acx), scz), acz));
        float* sc = solved_color + (int64_t)i * 3;
        float* ac = exact_color + (int64_t)i * 3;
        float* dc = diff_color + (int64_t)i * 3;
        sc[0] = scx, sc[1] = 0.0f, sc[2] = scz;
        ac[0] = acx, ac[1] = 0.0f, ac[2] = acz;
        dc[0] = 0.0f, dc[1] = dy, dc[2] = 0.0f;
    }
}

// set_mesh_instances: the first `dim` coordinates of every vertex in float
// (a 2D mesh leaves z = 0), the exact copy at x - 2.2 and the difference copy
// at x + 2.2, in float as the reference's f32 fields compute it.
__global__ void mesh_instances_kernel(int nv, int dim, const double* __restrict__ verts, float* __restrict__ solved_v,
                                      float* __restrict__ exact_v, float* __restrict__ diff_v) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nv; i += gridDim.x * blockDim.x) {
        float p[3] = {0.0f, 0.0f, 0.0f};
        for (int c = 0; c < dim; ++c) p[c] = (float)verts[(int64_t)i * dim + c];
        const int64_t o = (int64_t)i * 3;
        solved_v[o] = p[0], solved_v[o + 1] = p[1], solved_v[o + 2] = p[2];
        exact_v[o] = __fsub_rn(p[0], 2.2f), exact_v[o + 1] = p[1], exact_v[o + 2] = p[2];
        diff_v[o] = __fadd_rn(p[0], 2.2f), diff_v[o + 1] = p[1], diff_v[o + 2] = p[2];
    }
}

}  // namespace

extern "C" {

int bem_compute_color(bem_ctx* ctx, int n, double* solved, const double* exact, const int32_t* vert_types, int show,
                      float* solved_color, float* exact_color, float* diff_color, void* stream) {
    if (!ctx) return BEM_ERR_INVALID;
    if (ctx->nv == 0) return bem_fail(ctx, BEM_ERR_NOMESH, "no mesh set");
    if (n != 1 && n != 2) return bem_fail(ctx, BEM_ERR_INVALID, "n must be 1 (real) or 2 (complex)");
    if (show < -1 || show > 2) return bem_fail(ctx, BEM_ERR_INVALID, "show must be -1, 0, 1 or 2");
    if (!solved || !exact || !vert_types || !solved_color || !exact_color || !diff_color)
        return bem_fail(ctx, BEM_ERR_INVALID, "null buffer");
    cudaStream_t s = (cudaStream_t)stream;
    compute_color_kernel<<<1, COLOR_THREADS, 0, s>>>(ctx->nv, n, solved, exact, vert_types, show, solved_color,
                                                     exact_color, diff_color);
    ctx->launches++;
    return bem_check_cuda(ctx, cudaGetLastError(), "compute_color_kernel launch");
}

int bem_set_mesh_instances(bem_ctx* ctx, float* solved_vertices, float* exact_vertices, float* diff_vertices,
                           void* stream) {
    if (!ctx) return BEM_ERR_INVALID;
    if (ctx->nv == 0) return bem_fail(ctx, BEM_ERR_NOMESH, "no mesh set");
    if (!solved_vertices || !exact_vertices || !diff_vertices) return bem_fail(ctx, BEM_ERR_INVALID, "null buffer");
    cudaStream_t s = (cudaStream_t)stream;
    const int threads = 256;
    const int blocks = (int)std::min<int64_t>((ctx->nv + threads - 1) / threads, (int64_t)ctx->num_sms * 8);
    mesh_instances_kernel<<<blocks, threads, 0, s>>>(ctx->nv, ctx->dim, ctx->verts, solved_vertices, exact_vertices,
                                                     diff_vertices);
    ctx->launches++;
    return bem_check_cuda(ctx, cudaGetLastError(), "mesh_instances_kernel launch");
}

}  // extern "C"
