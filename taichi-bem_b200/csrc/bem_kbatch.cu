// k-batched dense assembly (bem_assemble_batch): one operator at several
// Helmholtz wavenumbers, every separate panel pair's geometry evaluated once.
//
// The reference assembles an operator once per wavenumber: its wavenumber
// sweep (demo/demo_3d_plot_Sio.py:63-82) calls get_mat_A1_inv_norm /
// get_augment_mat_A1_inv_norm (src/managers/BEM_manager.py:922-988) per k,
// and each call runs matrix_layer_forward (BEM_manager.py:829-844) at the
// exterior and at the interior wavenumber, one Taichi kernel per operator
// and wavenumber.  Here one launch takes up to KB_MAX wavenumbers: at each
// point pair the k-independent part of the integrand (r, 1/r, d.n / r^3,
// the split phase argument, the basis weights) is formed once and only
// e^{ikr} and the accumulation run per wavenumber.  The layout follows the
// single-wavenumber far kernel (bem_assembly.cu): one thread per (test
// panel, trial panel) pair, 128 trial panels per CTA, FAR_TI test panels'
// points in shared memory, FP32 sums over the test points and FP64 sums over
// the trial points in mixed precision (pair frame, bem_farfield.cuh), FP64
// throughout on the plain path.  Coincident / edge / vertex pairs take the
// FP64 Sauter-Schwab kernel once per wavenumber (bem_launch_assemble_parts).
#include <cmath>

#include "bem_farfield.cuh"

namespace {

constexpr int KB_MAX = 4;  // wavenumbers per far launch

struct KbArgs {
    int n_test, n_trial;
    const int32_t* test_panels;
    const int32_t* test_dof;
    const int32_t* trial_panels;
    const int32_t* trial_dof;
    const int32_t* tris;
    const double* centroid;
    const double* normal;
    const double* curl;
    const double* area;
    double wcorr;
    int small_phase;
    const void* pts;
    const void* phi;
    const double* phi64;
    int Q2;
    int dk;  // 1: the kernel's k-derivative at fixed k2 (as bem_assemble's deriv_k)
    int64_t ld;
    double k[KB_MAX], k2[KB_MAX], scale[KB_MAX], scale_t[KB_MAX];
    double* out[KB_MAX];    // nullptr: padding slot, evaluated but not written
    double* out_t[KB_MAX];  // nullptr: no transposed copy
};

// Helmholtz kernel value (without 1/(4 pi)) at one wavenumber from the
// k-independent quantities of a point pair: rinv = 1/r, t = d.n / r^3 (K, K'),
// ph = the phase argument (r - R in the FP32 pair frame, r in FP64).  With
// dk the kernel's k-derivative: i e^{ikr} for V and W, k (d.n) e^{ikr} / r
// for K and K' (d.n / r = t r^2).
template <int OP, typename T>
__device__ __forceinline__ void kb_value(T rinv, T r, T t, T ph, T k, bool small, bool dk, T& re, T& im) {
    T s, c;
    if constexpr (sizeof(T) == 4)
        dev_sincos_phase(k * ph, small, &s, &c);
    else
        dev_sincos(k * ph, &s, &c);
    if (OP == BEM_OP_V || OP == BEM_OP_W) {
        re = dk ? -s : rinv * c;
        im = dk ? c : rinv * s;
    } else if (dk) {
        const T f = t * k * r * r;
        re = f * c;
        im = f * s;
    } else {
        const T kr = k * r;
        re = t * fma(kr, s, c);
        im = t * fma(-kr, c, s);
    }
}

template <int OP, int NBX, int NBY, typename T, int NKB>
__global__ void __launch_bounds__(FAR_THREADS) far_kbatch_kernel(KbArgs a) {
    using V4 = typename V4T<T>::type;
    constexpr bool SPLIT = sizeof(T) == 4;
    constexpr bool W_OP = (OP == BEM_OP_W);

    extern __shared__ __align__(16) unsigned char smem_raw[];
    V4* sx = reinterpret_cast<V4*>(smem_raw);             // [FAR_TI][Q2]
    T* sphi = reinterpret_cast<T*>(sx + FAR_TI * a.Q2);  // [Q2*3]
    __shared__ int s_gi[FAR_TI];
    __shared__ int s_tri[FAR_TI][3];
    __shared__ double s_cen[FAR_TI][3];
    __shared__ double s_nrm[FAR_TI][3];

    const int Q2 = a.Q2;
    const int lj = blockIdx.x * FAR_THREADS + threadIdx.x;
    const int li0 = blockIdx.y * FAR_TI;
    const V4* pts = reinterpret_cast<const V4*>(a.pts);

    for (int idx = threadIdx.x; idx < FAR_TI * Q2; idx += FAR_THREADS) {
        const int t = idx / Q2, q = idx - t * Q2;
        const int li = li0 + t;
        if (li < a.n_test) sx[idx] = pts[(size_t)a.test_panels[li] * Q2 + q];
    }
    if (NBX == 3 || NBY == 3) {
        const T* phi = reinterpret_cast<const T*>(a.phi);
        for (int idx = threadIdx.x; idx < Q2 * 3; idx += FAR_THREADS) sphi[idx] = phi[idx];
    }
    if (threadIdx.x < FAR_TI) {
        const int li = li0 + threadIdx.x;
        const int gi = li < a.n_test ? a.test_panels[li] : -1;
        s_gi[threadIdx.x] = gi;
        for (int c = 0; c < 3; ++c) {
            s_tri[threadIdx.x][c] = gi >= 0 ? a.tris[3 * gi + c] : -1;
            s_cen[threadIdx.x][c] = gi >= 0 ? a.centroid[3 * gi + c] : 0.0;
            s_nrm[threadIdx.x][c] = gi >= 0 ? a.normal[3 * gi + c] : 0.0;
        }
    }
    __syncthreads();

    const bool valid_j = lj < a.n_trial;
    const int gj = valid_j ? a.trial_panels[lj] : 0;
    int tri_j[3];
    double cen_j[3], nrm_j[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        tri_j[c] = a.tris[3 * gj + c];
        cen_j[c] = a.centroid[3 * gj + c];
        nrm_j[c] = a.normal[3 * gj + c];
    }
    const V4* ptsj = pts + (size_t)gj * Q2;
    T kk[NKB];
#pragma unroll
    for (int w = 0; w < NKB; ++w) kk[w] = T(a.k[w]);
    const bool small = a.small_phase != 0;
    const bool dk = a.dk != 0;

    for (int t = 0; t < FAR_TI; ++t) {
        const int li = li0 + t;
        if (li >= a.n_test) break;  // uniform across the CTA
        const int gi = s_gi[t];
        const bool sep = valid_j && (bem_relation(s_tri[t], tri_j, gi == gj) == REL_SEPARATE);

        double acc_re[NKB][NBX][NBY], acc_im[NKB][NBX][NBY];
        double c0_re[NKB], c0_im[NKB];  // W: curl-curl moment (sum of weights * kernel)
        double pf = 1.0, cR[NKB], sR[NKB];
#pragma unroll
        for (int w = 0; w < NKB; ++w) {
            c0_re[w] = c0_im[w] = 0.0;
            cR[w] = 1.0;
            sR[w] = 0.0;
#pragma unroll
            for (int bx = 0; bx < NBX; ++bx)
#pragma unroll
                for (int by = 0; by < NBY; ++by) acc_re[w][bx][by] = acc_im[w][bx][by] = 0.0;
        }

        if (sep) {
            const double dcx64 = s_cen[t][0] - cen_j[0], dcy64 = s_cen[t][1] - cen_j[1],
                         dcz64 = s_cen[t][2] - cen_j[2];
            const T dcx = T(dcx64), dcy = T(dcy64), dcz = T(dcz64);
            const T dlx = T(dcx64 - double(dcx)), dly = T(dcy64 - double(dcy)), dlz = T(dcz64 - double(dcz));
            // pair frame (FP32): 2D, R^2, R and e^{i k_w R} per wavenumber in FP64
            T ux = T(0), uy = T(0), uz = T(0), R2 = T(0), Rf = T(0);
            if (SPLIT) {
                pf = 4.0 * a.area[gi] * a.area[gj] * a.wcorr;
                ux = T(2.0 * dcx64);
                uy = T(2.0 * dcy64);
                uz = T(2.0 * dcz64);
                const double R2d = dcx64 * dcx64 + dcy64 * dcy64 + dcz64 * dcz64;
                R2 = T(R2d);
                const double R = sqrt(R2d);
                Rf = T(R);
#pragma unroll
                for (int w = 0; w < NKB; ++w) sincos(a.k[w] * R, &sR[w], &cR[w]);
            }
            const double n0 = (OP == BEM_OP_KP) ? s_nrm[t][0] : nrm_j[0];
            const double n1 = (OP == BEM_OP_KP) ? s_nrm[t][1] : nrm_j[1];
            const double n2 = (OP == BEM_OP_KP) ? s_nrm[t][2] : nrm_j[2];
            const T nx = T(n0), ny = T(n1), nz = T(n2);
            const T Dn = T(dcx64 * n0 + dcy64 * n1 + dcz64 * n2);
            const T mx = T(nrm_j[0] - s_nrm[t][0]), my = T(nrm_j[1] - s_nrm[t][1]), mz = T(nrm_j[2] - s_nrm[t][2]);
            const V4* sxt = sx + t * Q2;
            for (int b = 0; b < Q2; ++b) {
                const V4 yb = ptsj[b];
                const T ex = (dcx - yb.x) + dlx, ey = (dcy - yb.y) + dly, ez = (dcz - yb.z) + dlz;
                const T wx = ux - yb.x, wy = uy - yb.y, wz = uz - yb.z;
                const T dnb = -(Dn + (yb.x * mx + yb.y * my + yb.z * mz));
                T s_re[NKB][NBX], s_im[NKB][NBX], c_re[NKB], c_im[NKB];
#pragma unroll
                for (int w = 0; w < NKB; ++w) {
                    c_re[w] = c_im[w] = T(0);
#pragma unroll
                    for (int bx = 0; bx < NBX; ++bx) s_re[w][bx] = s_im[w][bx] = T(0);
                }
#pragma unroll 5
                for (int q = 0; q < Q2; ++q) {
                    const V4 xa = sxt[q];
                    T r, rinv, ph, tt = T(0);
                    if constexpr (SPLIT) {
                        const T e_x = xa.x - yb.x, e_y = xa.y - yb.y, e_z = xa.z - yb.z;
                        const T sq = e_x * (xa.x + wx) + e_y * (xa.y + wy) + e_z * (xa.z + wz);
                        dev_r_rinv(R2 + sq, r, rinv);
                        ph = __fdividef(sq, r + Rf);
                        if (OP == BEM_OP_K || OP == BEM_OP_KP) {
                            const T dn = (OP == BEM_OP_K) ? fma(xa.x, mx, fma(xa.y, my, fma(xa.z, mz, Dn))) : dnb;
                            tt = dn * rinv * rinv * rinv;
                        }
                    } else {
                        const T dx = xa.x + ex, dy = xa.y + ey, dz = xa.z + ez;
                        dev_r_rinv(dx * dx + dy * dy + dz * dz, r, rinv);
                        ph = r;
                        if (OP == BEM_OP_K || OP == BEM_OP_KP) {
                            T dn = dx * nx + dy * ny + dz * nz;
                            if (OP == BEM_OP_KP) dn = -dn;
                            tt = dn * rinv * rinv * rinv;
                        }
                    }
                    T wp[NBX];
#pragma unroll
                    for (int bx = 0; bx < NBX; ++bx) wp[bx] = NBX == 1 ? xa.w : xa.w * sphi[3 * q + bx];
#pragma unroll
                    for (int w = 0; w < NKB; ++w) {
                        T re, im;
                        kb_value<OP, T>(rinv, r, tt, ph, kk[w], small, dk, re, im);
                        if (W_OP) {
                            c_re[w] += xa.w * re;
                            c_im[w] += xa.w * im;
                        }
#pragma unroll
                        for (int bx = 0; bx < NBX; ++bx) {
                            s_re[w][bx] += wp[bx] * re;
                            s_im[w][bx] += wp[bx] * im;
                        }
                    }
                }
                const double wb = double(yb.w);
#pragma unroll
                for (int by = 0; by < NBY; ++by) {
                    const double wpb = (NBY == 1) ? wb : wb * a.phi64[3 * b + by];
#pragma unroll
                    for (int w = 0; w < NKB; ++w)
#pragma unroll
                        for (int bx = 0; bx < NBX; ++bx) {
                            acc_re[w][bx][by] += wpb * double(s_re[w][bx]);
                            acc_im[w][bx][by] += wpb * double(s_im[w][bx]);
                        }
                }
                if (W_OP) {
#pragma unroll
                    for (int w = 0; w < NKB; ++w) {
                        c0_re[w] += wb * double(c_re[w]);
                        c0_im[w] += wb * double(c_im[w]);
                    }
                }
            }
        }
        if (!sep) continue;

        // ---- epilogue per wavenumber ----
        const double nd = s_nrm[t][0] * nrm_j[0] + s_nrm[t][1] * nrm_j[1] + s_nrm[t][2] * nrm_j[2];
        constexpr bool ATOMIC = (NBX == 3 || NBY == 3);
#pragma unroll
        for (int w = 0; w < NKB; ++w) {
            double* out = a.out[w];
            if (out == nullptr) continue;
            double* out_t = a.out_t[w];
            // pf e^{i k_w R} / (4 pi)
            const double fr = pf * cR[w] * BEM_INV4PI, fi = pf * sR[w] * BEM_INV4PI;
#pragma unroll
            for (int bx = 0; bx < NBX; ++bx) {
                const int row = a.test_dof[li * NBX + bx];
                if (row < 0) continue;
#pragma unroll
                for (int by = 0; by < NBY; ++by) {
                    const int col = a.trial_dof[lj * NBY + by];
                    if (col < 0) continue;
                    double vr, vi;
                    if (W_OP) {
                        // W = G curl.curl - k2 (n_x.n_y) G phi_x phi_y (hypersingular_layer_3d.py:206-211)
                        double cd = 0.0;
                        if (NBX == 3 && NBY == 3) {
                            const double* cx = a.curl + 9 * gi + 3 * bx;
                            const double* cy = a.curl + 9 * gj + 3 * by;
                            cd = cx[0] * cy[0] + cx[1] * cy[1] + cx[2] * cy[2];
                        }
                        vr = c0_re[w] * cd - a.k2[w] * nd * acc_re[w][bx][by];
                        vi = c0_im[w] * cd - a.k2[w] * nd * acc_im[w][bx][by];
                    } else {
                        vr = acc_re[w][bx][by];
                        vi = acc_im[w][bx][by];
                    }
                    const double er = vr * fr - vi * fi, ei = vr * fi + vi * fr;
                    add_entry<true>(out, (int64_t)row * a.ld + col, a.scale[w] * er, a.scale[w] * ei, ATOMIC);
                    if (out_t)
                        add_entry<true>(out_t, (int64_t)col * a.ld + row, a.scale_t[w] * er, a.scale_t[w] * ei, true);
                }
            }
        }
    }
}

template <int OP, int NBX, int NBY, typename T, int NKB>
int launch_kb(bem_ctx* ctx, const KbArgs& a, cudaStream_t s) {
    using V4 = typename V4T<T>::type;
    dim3 grid((a.n_trial + FAR_THREADS - 1) / FAR_THREADS, (a.n_test + FAR_TI - 1) / FAR_TI);
    if (grid.y > 65535) return bem_fail(ctx, BEM_ERR_INVALID, "too many test panels for one launch");
    const size_t smem = FAR_TI * a.Q2 * sizeof(V4) + a.Q2 * 3 * sizeof(T);
    far_kbatch_kernel<OP, NBX, NBY, T, NKB><<<grid, FAR_THREADS, smem, s>>>(a);
    ctx->launches++;
    return bem_check_cuda(ctx, cudaGetLastError(), "far_kbatch_kernel launch");
}

// Four wavenumbers per launch only where the FP64 accumulators fit the
// register file: the P1 x P1 blocks (9 complex moments per wavenumber) take
// two (four spill at the 255-register limit).
template <int OP, int NBX, int NBY>
int dispatch_kb_t(bem_ctx* ctx, const KbArgs& a, bool fp32, int nkb, cudaStream_t s) {
    if constexpr (NBX * NBY == 9) {
        if (nkb != 2) return bem_fail(ctx, BEM_ERR_INVALID, "P1 x P1 blocks take two wavenumbers per launch");
        return fp32 ? launch_kb<OP, 3, 3, float, 2>(ctx, a, s) : launch_kb<OP, 3, 3, double, 2>(ctx, a, s);
    }
    if (fp32)
        return nkb == 4 ? launch_kb<OP, NBX, NBY, float, 4>(ctx, a, s) : launch_kb<OP, NBX, NBY, float, 2>(ctx, a, s);
    return nkb == 4 ? launch_kb<OP, NBX, NBY, double, 4>(ctx, a, s) : launch_kb<OP, NBX, NBY, double, 2>(ctx, a, s);
}

template <int OP>
int dispatch_kb(bem_ctx* ctx, const KbArgs& a, int nbx, int nby, bool fp32, int nkb, cudaStream_t s) {
    if (nbx == 1 && nby == 1) return dispatch_kb_t<OP, 1, 1>(ctx, a, fp32, nkb, s);
    if (nbx == 1 && nby == 3) return dispatch_kb_t<OP, 1, 3>(ctx, a, fp32, nkb, s);
    if (nbx == 3 && nby == 1) return dispatch_kb_t<OP, 3, 1>(ctx, a, fp32, nkb, s);
    if (nbx == 3 && nby == 3) return dispatch_kb_t<OP, 3, 3>(ctx, a, fp32, nkb, s);
    return bem_fail(ctx, BEM_ERR_INVALID, "nb must be 1 (P0) or 3 (P1)");
}

}  // namespace

// nk wavenumbers of one operator (validated by bem_assemble_batch): far
// pairs in groups of 2 or 4 wavenumbers per launch (BEM_TUNE_KBATCH_GROUP;
// always 2 for P1 x P1 blocks; a short last group is padded with slots that
// are not written), near pairs per wavenumber on the FP64 Sauter-Schwab
// kernel.
int bem_launch_assemble_batch(bem_ctx* ctx, const bem_op_desc* op, const bem_space* test, const bem_space* trial,
                              int nk, const double* k, const double* k2, void* const* out, int64_t ld,
                              const double* scale, void* const* out_t, const double* scale_t, cudaStream_t s) {
    const bool fp32 = op->precision == BEM_PREC_MIXED;
    const int tuned = ctx->tune[BEM_TUNE_KBATCH_GROUP];
    const int group = test->nb * trial->nb == 9 ? 2 : (tuned == 2 || tuned == 4 ? tuned : (fp32 ? 4 : 2));
    double kmax = 0.0;
    for (int w = 0; w < nk; ++w) kmax = fmax(kmax, fabs(k[w]));
    KbArgs a{};
    a.n_test = test->n_panels;
    a.n_trial = trial->n_panels;
    a.test_panels = test->panels;
    a.test_dof = test->dof;
    a.trial_panels = trial->panels;
    a.trial_dof = trial->dof;
    a.tris = ctx->tris;
    a.centroid = ctx->centroid;
    a.normal = ctx->normal;
    a.curl = ctx->curl;
    a.area = ctx->area;
    a.wcorr = ctx->wcorr32;
    a.small_phase = fp32 ? bem_phase_class(kmax * 2.0 * ctx->rho_max) : 0;
    a.pts = fp32 ? (const void*)ctx->pts32 : (const void*)ctx->pts64;
    a.phi = fp32 ? (const void*)ctx->phi32 : (const void*)ctx->phi64;
    a.phi64 = ctx->phi64;
    a.Q2 = ctx->Q2;
    a.dk = op->deriv_k ? 1 : 0;
    a.ld = ld;
    if (a.n_test > 0 && a.n_trial > 0) {
        for (int w0 = 0; w0 < nk; w0 += group) {
            const int m = nk - w0 < group ? nk - w0 : group;
            const int nkb = m > 2 ? 4 : 2;
            for (int w = 0; w < KB_MAX; ++w) {
                const bool live = w < m;
                const int src = live ? w0 + w : w0;  // padding repeats the group's first wavenumber
                a.k[w] = k[src];
                a.k2[w] = k2[src];
                a.scale[w] = live ? scale[src] : 0.0;
                a.scale_t[w] = live && scale_t ? scale_t[src] : 0.0;
                a.out[w] = live ? (double*)out[src] : nullptr;
                a.out_t[w] = live && out_t ? (double*)out_t[src] : nullptr;
            }
            int rc = BEM_OK;
            switch (op->op) {
                case BEM_OP_V: rc = dispatch_kb<BEM_OP_V>(ctx, a, test->nb, trial->nb, fp32, nkb, s); break;
                case BEM_OP_K: rc = dispatch_kb<BEM_OP_K>(ctx, a, test->nb, trial->nb, fp32, nkb, s); break;
                case BEM_OP_KP: rc = dispatch_kb<BEM_OP_KP>(ctx, a, test->nb, trial->nb, fp32, nkb, s); break;
                case BEM_OP_W: rc = dispatch_kb<BEM_OP_W>(ctx, a, test->nb, trial->nb, fp32, nkb, s); break;
                default: rc = bem_fail(ctx, BEM_ERR_INVALID, "unknown operator");
            }
            if (rc) return rc;
        }
    }
    for (int w = 0; w < nk; ++w) {
        bem_op_desc ow = *op;
        ow.k = k[w];
        ow.k2 = k2[w];
        void* ot = out_t ? out_t[w] : nullptr;
        if (int rc = bem_launch_assemble_parts(ctx, &ow, test, trial, 0, out[w], ld, scale[w], ot,
                                               ot ? scale_t[w] : 0.0, nullptr, nullptr, 0, s, true))
            return rc;
    }
    return BEM_OK;
}
