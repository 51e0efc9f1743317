// Galerkin BEM operator assembly on sm_100a.
//
// The reference evaluates every operator with one Taichi thread per test
// panel that loops serially over trial panels x basis pairs x GaussQR^4
// points and recomputes the integrand per basis pair
// (src/BEM_functions/single_layer/single_layer_3d.py:371-433 and its double /
// adjoint / hypersingular twins).  Here:
//
//  * separate pairs (the O(nt^2) bulk) run in `far_kernel`: one thread per
//    (test panel, trial panel) pair, 128 trial panels per CTA and TI test
//    panels staged in shared memory.  The separate-pair rule factorises into
//    Q^2 points per panel (x(xsi, eta1) on the test panel, y(eta2, eta3) on the
//    trial panel), so each thread loops over its trial points (registers) and
//    the test points (shared-memory broadcast), and ONE kernel evaluation
//    serves every basis pair (P0/P1 test x P0/P1 trial).  Coordinates are
//    stored relative to the panel centroid and the centroid difference is
//    formed in FP64, so the FP32 variant (mixed precision) keeps its relative
//    accuracy for close pairs.
//  * coincident / edge / vertex pairs (about 13 per panel on an icosphere)
//    run in `near_kernel` in FP64: one warp per pair, lanes split the
//    GaussQR^4 Sauter-Schwab points, warp-shuffle reduction.
//  * P0 rows/columns are written in place (each entry has one writer); P1
//    entries receive contributions from several panel pairs and use FP64
//    atomics, as the reference's Taichi `+=` does (hypersingular_layer_3d.py:500).
#include <cuda_runtime.h>

#include "bem_internal.cuh"
#include "bem_quadrature.cuh"
#include "bem_farfield.cuh"

namespace {


// ----------------------------------------------------------------------------
// geometry: areas/normals/centroids/curls and the separate-rule points
// (mesh_manager.py:114-125, hypersingular_layer_3d.py:55-64,163-169,
//  single_layer_3d.py:143-177)
// ----------------------------------------------------------------------------
__global__ void geometry_kernel(int nt, int Q, const double* __restrict__ verts, const int32_t* __restrict__ tris,
                                const double* __restrict__ gp, const double* __restrict__ gw, double* area,
                                double* normal, double* centroid, double* curl, double4* pts64, float4* pts32,
                                int32_t* flags) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= nt) return;
    double v[3][3];
    for (int a = 0; a < 3; ++a)
        for (int c = 0; c < 3; ++c) v[a][c] = verts[3 * tris[3 * p + a] + c];
    double e1[3], e2[3];
    for (int c = 0; c < 3; ++c) {
        e1[c] = v[1][c] - v[0][c];
        e2[c] = v[2][c] - v[1][c];
    }
    double cr[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
    double nrm = sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
    if (!(nrm > 0.0) || !isfinite(nrm)) {
        atomicExch(&flags[0], 1 + p);  // degenerate or non-finite panel
        nrm = 1.0;
    }
    double A = 0.5 * nrm;
    double n[3] = {cr[0] / nrm, cr[1] / nrm, cr[2] / nrm};
    area[p] = A;
    double cen[3];
    for (int c = 0; c < 3; ++c) {
        normal[3 * p + c] = n[c];
        cen[c] = (v[0][c] + v[1][c] + v[2][c]) / 3.0;
        centroid[3 * p + c] = cen[c];
    }
    // curl of the hat of vertex b: n x ((n x edge_opposite_b) / (2A))
    const double* opp[3][2] = {{v[2], v[1]}, {v[0], v[2]}, {v[1], v[0]}};
    for (int b = 0; b < 3; ++b) {
        double d[3] = {opp[b][0][0] - opp[b][1][0], opp[b][0][1] - opp[b][1][1], opp[b][0][2] - opp[b][1][2]};
        double g[3] = {(n[1] * d[2] - n[2] * d[1]) / (2.0 * A), (n[2] * d[0] - n[0] * d[2]) / (2.0 * A),
                       (n[0] * d[1] - n[1] * d[0]) / (2.0 * A)};
        curl[9 * p + 3 * b + 0] = n[1] * g[2] - n[2] * g[1];
        curl[9 * p + 3 * b + 1] = n[2] * g[0] - n[0] * g[2];
        curl[9 * p + 3 * b + 2] = n[0] * g[1] - n[1] * g[0];
    }
    int Q2 = Q * Q;
    for (int ix = 0; ix < Q; ++ix)
        for (int iy = 0; iy < Q; ++iy) {
            double r1 = gp[ix], r2 = gp[iy] * r1;
            // reference-triangle weight; FP64 points carry the Jacobian 2A,
            // FP32 points the panel-independent weight (the pair's 4 A_i A_j
            // is applied in FP64, so the FP32 rounding of a weight is the same
            // for every panel)
            const double wref = (gw[ix] * gw[iy]) * r1;
            double o[3];
            for (int c = 0; c < 3; ++c) o[c] = ((1.0 - r1) * v[0][c] + (r1 - r2) * v[1][c] + r2 * v[2][c]) - cen[c];
            pts64[(size_t)p * Q2 + ix * Q + iy] = make_double4(o[0], o[1], o[2], wref * (A * 2.0));
            pts32[(size_t)p * Q2 + ix * Q + iy] = make_float4((float)o[0], (float)o[1], (float)o[2], (float)wref);
        }
}

__global__ void scatter_local_kernel(int n, const int32_t* __restrict__ panels, int32_t* local_of_global, int nt,
                                     int32_t* flags) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int g = panels[i];
    if (g < 0 || g >= nt) {
        atomicExch(&flags[1], 1 + i);
        return;
    }
    local_of_global[g] = i;
}

// ----------------------------------------------------------------------------
// kernel functions
// ----------------------------------------------------------------------------
// Kernel value at d = x - y (without the 1/(4 pi) factor):
//   V, W: e^{ikr}/r                           (G, BEM_manager.py:474-483)
//   K:    (d.n_y)/r^3 (1 - ikr) e^{ikr}       (grad_G_y, BEM_manager.py:510-523)
//   KP:   (-d.n_x)/r^3 (1 - ikr) e^{ikr}      (grad_G_y with x,y swapped and n_x)
// and with dk (Helmholtz) their derivatives in k:
//   V, W: i e^{ikr}  (= i r G)                K, KP: k (d.n)/r e^{ikr}
template <int OP, bool HELM, typename T>
__device__ __forceinline__ void kval(T dx, T dy, T dz, T nx, T ny, T nz, T k, T& re, T& im, bool dk = false) {
    const T r2 = dx * dx + dy * dy + dz * dz;
    T r, rinv;
    dev_r_rinv(r2, r, rinv);
    if (OP == BEM_OP_V || OP == BEM_OP_W) {
        if (!HELM) {
            re = rinv;
            im = T(0);
        } else {
            T s, c;
            dev_sincos(k * r, &s, &c);
            re = dk ? -s : rinv * c;
            im = dk ? c : rinv * s;
        }
    } else {
        T dn = dx * nx + dy * ny + dz * nz;
        if (OP == BEM_OP_KP) dn = -dn;
        T t = dn * rinv * rinv * rinv;
        if (!HELM) {
            re = t;
            im = T(0);
        } else {
            T kr = k * r;
            T s, c;
            dev_sincos(kr, &s, &c);
            if (dk) {
                const T f = dn * k * rinv;
                re = f * c;
                im = f * s;
            } else {
                re = t * (c + kr * s);
                im = t * (s - kr * c);
            }
        }
    }
}

// The same values in a pair frame (FP32): r2 = R^2 + s, dn = d.n (-d.n_x for
// K'), Rf = R; the result lacks the pair's factor e^{ikR} (Frame::rotate).
template <int OP, bool HELM>
__device__ __forceinline__ void kval_split(float r2, float s, float dn, float k, float Rf, bool small, float& re,
                                           float& im, bool dk = false) {
    float r, rinv;
    dev_r_rinv(r2, r, rinv);
    if (OP == BEM_OP_V || OP == BEM_OP_W) {
        if (!HELM) {
            re = rinv;
            im = 0.0f;
        } else {
            float sn, cs;
            dev_sincos_phase(k * __fdividef(s, r + Rf), small, &sn, &cs);
            re = dk ? -sn : rinv * cs;
            im = dk ? cs : rinv * sn;
        }
    } else {
        const float t = dn * rinv * rinv * rinv;
        if (!HELM) {
            re = t;
            im = 0.0f;
        } else {
            const float kr = k * r;
            float sn, cs;
            dev_sincos_phase(k * __fdividef(s, r + Rf), small, &sn, &cs);
            if (dk) {
                const float f = dn * k * rinv;
                re = f * cs;
                im = f * sn;
            } else {
                re = t * fmaf(kr, sn, cs);
                im = t * fmaf(-kr, cs, sn);
            }
        }
    }
}

struct FarArgs {
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
    double wcorr;     // (exact / FP32 weight sum)^2 of the FP32 separate rule
    int small_phase;  // FP32 split phase bounded by pi/4 (1) or by 0.3 (2): sine/cosine without reduction
    const void* pts;
    const void* phi;
    const double* phi64;  // [Q2*3] P1 basis at the separate-rule points, FP64
    int Q2;
    double k, k2;
    int mode;
    double* out;
    int64_t ld;
    double scale;
    double* out_t;
    double scale_t;
    const double* x;
    double* y;
    int conj_x;
    int skip_far;  // 1: launch only the near-pair kernel (bem_launch_assemble_parts)
    int dk = 0;    // 1: the kernel's k-derivative (kval)
};


template <int OP, bool HELM, int NBX, int NBY, typename T>
__global__ void __launch_bounds__(FAR_THREADS) far_kernel(FarArgs a) {
    using V4 = typename V4T<T>::type;
    constexpr bool W_OP = (OP == BEM_OP_W);
    // accumulate phi-weighted moments for every op except Laplace W, whose
    // only term is the curl-curl one (k2 = 0)
    constexpr bool NEED_PHI = !(W_OP && !HELM);
    constexpr int AX = NEED_PHI ? NBX : 1;
    constexpr int AY = NEED_PHI ? NBY : 1;

    extern __shared__ __align__(16) unsigned char smem_raw[];
    V4* sx = reinterpret_cast<V4*>(smem_raw);                 // [FAR_TI][Q2]
    T* sphi = reinterpret_cast<T*>(sx + FAR_TI * a.Q2);      // [Q2*3]
    __shared__ int s_gi[FAR_TI];
    __shared__ int s_tri[FAR_TI][3];
    __shared__ double s_cen[FAR_TI][3];
    __shared__ double s_nrm[FAR_TI][3];

    const int Q2 = a.Q2;
    const int lj = blockIdx.x * FAR_THREADS + threadIdx.x;
    const int li0 = blockIdx.y * FAR_TI;
    const V4* pts = reinterpret_cast<const V4*>(a.pts);

    for (int idx = threadIdx.x; idx < FAR_TI * Q2; idx += FAR_THREADS) {
        int t = idx / Q2, q = idx - t * Q2;
        int li = li0 + t;
        if (li < a.n_test) sx[idx] = pts[(size_t)a.test_panels[li] * Q2 + q];
    }
    if (NBX == 3 || NBY == 3) {
        const T* phi = reinterpret_cast<const T*>(a.phi);
        for (int idx = threadIdx.x; idx < Q2 * 3; idx += FAR_THREADS) sphi[idx] = phi[idx];
    }
    if (threadIdx.x < FAR_TI) {
        int li = li0 + threadIdx.x;
        int gi = li < a.n_test ? a.test_panels[li] : -1;
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
    const T kk = T(a.k);
    const int lane = threadIdx.x & 31;

    for (int t = 0; t < FAR_TI; ++t) {
        const int li = li0 + t;
        if (li >= a.n_test) break;  // uniform across the CTA
        const int gi = s_gi[t];
        const bool sep = valid_j && (bem_relation(s_tri[t], tri_j, gi == gj) == REL_SEPARATE);

        double acc_re[AX][AY], acc_im[AX][AY];
        double acc0_re = 0.0, acc0_im = 0.0;  // W curl-curl moment (sum of weights * kernel)
        Frame<T, HELM> fr;
#pragma unroll
        for (int bx = 0; bx < AX; ++bx)
#pragma unroll
            for (int by = 0; by < AY; ++by) acc_re[bx][by] = acc_im[bx][by] = 0.0;

        if (sep) {
            // centroid difference as an unevaluated pair hi + lo: in FP32 a
            // single rounding of it would be one systematic error shared by
            // all GaussQR^4 terms of the pair
            const double dcx64 = s_cen[t][0] - cen_j[0], dcy64 = s_cen[t][1] - cen_j[1],
                         dcz64 = s_cen[t][2] - cen_j[2];
            const T dcx = T(dcx64), dcy = T(dcy64), dcz = T(dcz64);
            const T dlx = T(dcx64 - double(dcx)), dly = T(dcy64 - double(dcy)), dlz = T(dcz64 - double(dcz));
            fr.init(dcx64, dcy64, dcz64, a.k, a.area[gi], a.area[gj], a.wcorr);
            // normal of K (trial panel) or K' (test panel), and D.n in FP64
            const double n0 = (OP == BEM_OP_KP) ? s_nrm[t][0] : nrm_j[0];
            const double n1 = (OP == BEM_OP_KP) ? s_nrm[t][1] : nrm_j[1];
            const double n2 = (OP == BEM_OP_KP) ? s_nrm[t][2] : nrm_j[2];
            const T nx = T(n0), ny = T(n1), nz = T(n2);
            const T Dn = T(dcx64 * n0 + dcy64 * n1 + dcz64 * n2);
            // n_j - n_i: x_a.n_j = x_a.(n_j - n_i) and y_b.n_i = -y_b.(n_j - n_i), exact for
            // points in their panel's plane, and small for nearly coplanar close pairs
            const T mx = T(nrm_j[0] - s_nrm[t][0]), my = T(nrm_j[1] - s_nrm[t][1]), mz = T(nrm_j[2] - s_nrm[t][2]);
            const V4* sxt = sx + t * Q2;
            for (int b = 0; b < Q2; ++b) {
                const V4 yb = ptsj[b];
                const T ex = (dcx - yb.x) + dlx, ey = (dcy - yb.y) + dly, ez = (dcz - yb.z) + dlz;
                // frame: 2D - y_b, and -d.n_x = -(D.n_x - y_b.n_x) for K' (x_a lies in the plane of panel i)
                const T wx = fr.ux - yb.x, wy = fr.uy - yb.y, wz = fr.uz - yb.z;
                const T dnb = -(Dn + (yb.x * mx + yb.y * my + yb.z * mz));
                T s_re[AX], s_im[AX];
                T c_re = T(0), c_im = T(0);
#pragma unroll
                for (int bx = 0; bx < AX; ++bx) s_re[bx] = s_im[bx] = T(0);
#pragma unroll 5
                for (int q = 0; q < Q2; ++q) {
                    const V4 xa = sxt[q];
                    T re, im;
                    if constexpr (Frame<T, HELM>::SPLIT) {
                        const T e_x = xa.x - yb.x, e_y = xa.y - yb.y, e_z = xa.z - yb.z;
                        const T sq = e_x * (xa.x + wx) + e_y * (xa.y + wy) + e_z * (xa.z + wz);
                        // K: d.n_y = D.n_y + x_a.n_y (y_b lies in the plane of panel j)
                        const T dn = (OP == BEM_OP_K) ? fma(xa.x, mx, fma(xa.y, my, fma(xa.z, mz, Dn))) : dnb;
                        kval_split<OP, HELM>(fr.R2 + sq, sq, dn, kk, fr.Rf, a.small_phase != 0, re, im, a.dk != 0);
                    } else {
                        kval<OP, HELM, T>(xa.x + ex, xa.y + ey, xa.z + ez, nx, ny, nz, kk, re, im, a.dk != 0);
                    }
                    if (W_OP) {
                        c_re += xa.w * re;
                        if (HELM) c_im += xa.w * im;
                    }
                    if (NEED_PHI) {
                        if (AX == 1) {
                            s_re[0] += xa.w * re;
                            if (HELM) s_im[0] += xa.w * im;
                        } else {
#pragma unroll
                            for (int bx = 0; bx < AX; ++bx) {
                                T wp = xa.w * sphi[3 * q + bx];
                                s_re[bx] += wp * re;
                                if (HELM) s_im[bx] += wp * im;
                            }
                        }
                    }
                }
                const double wb = double(yb.w);
                if (W_OP) {
                    acc0_re += wb * double(c_re);
                    acc0_im += wb * double(c_im);
                }
                if (NEED_PHI) {
#pragma unroll
                    for (int by = 0; by < AY; ++by) {
                        // trial basis in FP64: an exact partition of unity for the trial side
                        double wpb = (AY == 1) ? wb : wb * a.phi64[3 * b + by];
#pragma unroll
                        for (int bx = 0; bx < AX; ++bx) {
                            acc_re[bx][by] += wpb * double(s_re[bx]);
                            acc_im[bx][by] += wpb * double(s_im[bx]);
                        }
                    }
                }
            }
        }

        // ---- epilogue: values of all basis pairs ----
        double val_re[NBX][NBY], val_im[NBX][NBY];
#pragma unroll
        for (int bx = 0; bx < NBX; ++bx)
#pragma unroll
            for (int by = 0; by < NBY; ++by) {
                double vr, vi;
                if (W_OP) {
                    // W = G curl.curl - k2 (n_x.n_y) G phi_x phi_y (hypersingular_layer_3d.py:206-211)
                    double cd = 0.0;
                    if (NBX == 3 && NBY == 3 && sep) {
                        const double* cx = a.curl + 9 * gi + 3 * bx;
                        const double* cy = a.curl + 9 * gj + 3 * by;
                        cd = cx[0] * cy[0] + cx[1] * cy[1] + cx[2] * cy[2];
                    }
                    vr = acc0_re * cd;
                    vi = acc0_im * cd;
                    if (NEED_PHI) {
                        double nd = s_nrm[t][0] * nrm_j[0] + s_nrm[t][1] * nrm_j[1] + s_nrm[t][2] * nrm_j[2];
                        int ix = AX == 1 ? 0 : bx, iy = AY == 1 ? 0 : by;
                        vr -= a.k2 * nd * acc_re[ix][iy];
                        vi -= a.k2 * nd * acc_im[ix][iy];
                    }
                } else {
                    int ix = AX == 1 ? 0 : bx, iy = AY == 1 ? 0 : by;
                    vr = acc_re[ix][iy];
                    vi = acc_im[ix][iy];
                }
                fr.rotate(vr, vi);
                val_re[bx][by] = vr * BEM_INV4PI;
                val_im[bx][by] = vi * BEM_INV4PI;
            }

        if (a.mode == 0) {
            if (sep) {
                constexpr bool ATOMIC = (NBX == 3 || NBY == 3);
#pragma unroll
                for (int bx = 0; bx < NBX; ++bx) {
                    const int row = a.test_dof[li * NBX + bx];
                    if (row < 0) continue;
#pragma unroll
                    for (int by = 0; by < NBY; ++by) {
                        const int col = a.trial_dof[lj * NBY + by];
                        if (col < 0) continue;
                        add_entry<HELM>(a.out, (int64_t)row * a.ld + col, a.scale * val_re[bx][by],
                                        a.scale * val_im[bx][by], ATOMIC);
                        if (a.out_t)
                            add_entry<HELM>(a.out_t, (int64_t)col * a.ld + row, a.scale_t * val_re[bx][by],
                                            a.scale_t * val_im[bx][by], true);
                    }
                }
            }
        } else {
            // apply: y[row] += scale * sum_col val * x[col]
#pragma unroll
            for (int bx = 0; bx < NBX; ++bx) {
                double cr = 0.0, ci = 0.0;
                if (sep) {
#pragma unroll
                    for (int by = 0; by < NBY; ++by) {
                        const int col = a.trial_dof[lj * NBY + by];
                        if (col < 0) continue;
                        if (HELM) {
                            double xr = a.x[2 * col], xi = a.x[2 * col + 1];
                            if (a.conj_x) xi = -xi;
                            cr += val_re[bx][by] * xr - val_im[bx][by] * xi;
                            ci += val_re[bx][by] * xi + val_im[bx][by] * xr;
                        } else {
                            cr += val_re[bx][by] * a.x[col];
                        }
                    }
                }
                cr = warp_sum(cr);
                if (HELM) ci = warp_sum(ci);
                if (lane == 0) {
                    const int row = a.test_dof[li * NBX + bx];
                    if (row >= 0) {
                        if (HELM) {
                            atomicAdd(a.y + 2 * row, a.scale * cr);
                            atomicAdd(a.y + 2 * row + 1, a.scale * ci);
                        } else {
                            atomicAdd(a.y + row, a.scale * cr);
                        }
                    }
                }
            }
        }
    }
}

// ----------------------------------------------------------------------------
// near field: coincident / edge / vertex pairs in FP64 (Sauter-Schwab maps of
// single_layer_3d.py:178-367, identical in the other operators)
// ----------------------------------------------------------------------------
struct NearArgs {
    int64_t n_near;
    const int4* near;
    const int32_t* test_local;
    const int32_t* trial_local;
    const int32_t* test_dof;
    const int32_t* trial_dof;
    const int32_t* tris;
    const double* verts;
    const double* area;
    const double* normal;
    const double* curl;
    const double* gp;
    const double* gw;
    int Q;
    double k, k2;
    int quirk;
    int mode;
    double* out;
    int64_t ld;
    double scale;
    double* out_t;
    double scale_t;
    const double* x;
    double* y;
    int conj_x;
    int dk = 0;  // 1: the kernel's k-derivative (kval)
};

struct NearPanel {
    double x1[3], x2[3], x3[3];
    double n[3];
    double area;
    int slot[3];  // parameter slot of original vertex b
};

__device__ __forceinline__ void load_near_panel(NearPanel& P, const NearArgs& a, int g, int perm) {
    int pm[3] = {perm & 3, (perm >> 2) & 3, (perm >> 4) & 3};
    const int32_t* t = a.tris + 3 * g;
    for (int c = 0; c < 3; ++c) {
        P.x1[c] = a.verts[3 * t[pm[0]] + c];
        P.x2[c] = a.verts[3 * t[pm[1]] + c];
        P.x3[c] = a.verts[3 * t[pm[2]] + c];
        P.n[c] = a.normal[3 * g + c];
    }
    P.area = a.area[g];
    for (int s = 0; s < 3; ++s) P.slot[pm[s]] = s;
}

__device__ __forceinline__ double shape_slot(double r1, double r2, int s) {
    return s == 0 ? 1.0 - r1 : (s == 1 ? r1 - r2 : r2);
}

template <int OP, bool HELM, int NBX, int NBY>
__global__ void __launch_bounds__(128) near_kernel(NearArgs a) {
    constexpr bool W_OP = (OP == BEM_OP_W);
    constexpr bool NEED_PHI = !(W_OP && !HELM);
    const int lane = threadIdx.x & 31;
    const int64_t pid = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (pid >= a.n_near) return;
    const int4 e = a.near[pid];
    const int gi = e.x, gj = e.y, rel = e.z;
    const int li = a.test_local[gi], lj = a.trial_local[gj];
    if (li < 0 || lj < 0) return;  // warp-uniform
    const int permx = a.quirk ? (0 | (1 << 2) | (2 << 4)) : (e.w & 63);
    const int permy = a.quirk ? (0 | (1 << 2) | (2 << 4)) : ((e.w >> 6) & 63);
    NearPanel X, Y;
    load_near_panel(X, a, gi, permx);
    load_near_panel(Y, a, gj, permy);
    const double* nKx = X.n;  // normal used by KP
    const double* nKy = Y.n;  // normal used by K

    double acc_re[NBX][NBY], acc_im[NBX][NBY], acc0_re = 0.0, acc0_im = 0.0;
#pragma unroll
    for (int bx = 0; bx < NBX; ++bx)
#pragma unroll
        for (int by = 0; by < NBY; ++by) acc_re[bx][by] = acc_im[bx][by] = 0.0;

    int sx[NBX], sy[NBY];
#pragma unroll
    for (int bx = 0; bx < NBX; ++bx) sx[bx] = NBX == 1 ? -1 : X.slot[bx];
#pragma unroll
    for (int by = 0; by < NBY; ++by) sy[by] = NBY == 1 ? -1 : Y.slot[by];

    const int Q = a.Q;
    const int Q4 = Q * Q * Q * Q;
    // One kernel evaluation at parameters (r1x,r2x) on X and (r1y,r2y) on Y,
    // argument order `second` (the swapped coincide term), basis values taken
    // at (px1,px2) for the test side and (py1,py2) for the trial side.
    auto add = [&](double r1x, double r2x, double r1y, double r2y, double wj, bool second, double px1, double px2,
                   double py1, double py2) {
        double x[3], yv[3];
        for (int c = 0; c < 3; ++c) {
            x[c] = (1.0 - r1x) * X.x1[c] + (r1x - r2x) * X.x2[c] + r2x * X.x3[c];
            yv[c] = (1.0 - r1y) * Y.x1[c] + (r1y - r2y) * Y.x2[c] + r2y * Y.x3[c];
        }
        double dx = x[0] - yv[0], dy = x[1] - yv[1], dz = x[2] - yv[2];
        double re, im;
        if (OP == BEM_OP_K) {
            // first: grad_G_y(x, y, n_y); second: grad_G_y(y, x, n_y)
            double sgn = second ? -1.0 : 1.0;
            kval<BEM_OP_K, HELM, double>(sgn * dx, sgn * dy, sgn * dz, nKy[0], nKy[1], nKy[2], a.k, re, im, a.dk != 0);
        } else if (OP == BEM_OP_KP) {
            // first: grad_G_y(y, x, n_x); second: grad_G_y(x, y, n_x)
            double sgn = second ? -1.0 : 1.0;
            kval<BEM_OP_KP, HELM, double>(sgn * dx, sgn * dy, sgn * dz, nKx[0], nKx[1], nKx[2], a.k, re, im,
                                          a.dk != 0);
        } else {
            kval<BEM_OP_V, HELM, double>(dx, dy, dz, 0.0, 0.0, 0.0, a.k, re, im, a.dk != 0);
        }
        re *= wj;
        im *= wj;
        if (W_OP) {
            acc0_re += re;
            acc0_im += im;
        }
        if (NEED_PHI) {
#pragma unroll
            for (int bx = 0; bx < NBX; ++bx) {
                double phx = NBX == 1 ? 1.0 : shape_slot(px1, px2, sx[bx]);
#pragma unroll
                for (int by = 0; by < NBY; ++by) {
                    double phy = NBY == 1 ? 1.0 : shape_slot(py1, py2, sy[by]);
                    acc_re[bx][by] += re * phx * phy;
                    acc_im[bx][by] += im * phx * phy;
                }
            }
        }
    };

    for (int p = lane; p < Q4; p += 32) {
        int iw = p % Q, iz = (p / Q) % Q, iy = (p / (Q * Q)) % Q, ix = p / (Q * Q * Q);
        const double xsi = a.gp[ix], eta1 = a.gp[iy], eta2 = a.gp[iz], eta3 = a.gp[iw];
        const double weight = (a.gw[ix] * a.gw[iy] * (X.area * 2.0)) * (a.gw[iz] * a.gw[iw] * (Y.area * 2.0));
        near_points(rel, a.quirk != 0, xsi, eta1, eta2, eta3, weight, add);
    }

    // warp reduction of every moment
    acc0_re = warp_sum(acc0_re);
    acc0_im = warp_sum(acc0_im);
#pragma unroll
    for (int bx = 0; bx < NBX; ++bx)
#pragma unroll
        for (int by = 0; by < NBY; ++by) {
            acc_re[bx][by] = warp_sum(acc_re[bx][by]);
            acc_im[bx][by] = warp_sum(acc_im[bx][by]);
        }
    if (lane != 0) return;

    const double nd = X.n[0] * Y.n[0] + X.n[1] * Y.n[1] + X.n[2] * Y.n[2];
#pragma unroll
    for (int bx = 0; bx < NBX; ++bx) {
        const int row = a.test_dof[li * NBX + bx];
        if (row < 0) continue;
        double cr = 0.0, ci = 0.0;
#pragma unroll
        for (int by = 0; by < NBY; ++by) {
            const int col = a.trial_dof[lj * NBY + by];
            if (col < 0) continue;
            double vr, vi;
            if (W_OP) {
                double cd = 0.0;
                if (NBX == 3 && NBY == 3) {
                    const double* cx = a.curl + 9 * gi + 3 * bx;
                    const double* cy = a.curl + 9 * gj + 3 * by;
                    cd = cx[0] * cy[0] + cx[1] * cy[1] + cx[2] * cy[2];
                }
                vr = acc0_re * cd;
                vi = acc0_im * cd;
                if (NEED_PHI) {
                    vr -= a.k2 * nd * acc_re[bx][by];
                    vi -= a.k2 * nd * acc_im[bx][by];
                }
            } else {
                vr = acc_re[bx][by];
                vi = acc_im[bx][by];
            }
            vr *= BEM_INV4PI;
            vi *= BEM_INV4PI;
            if (a.mode == 0) {
                add_entry<HELM>(a.out, (int64_t)row * a.ld + col, a.scale * vr, a.scale * vi, true);
                if (a.out_t) add_entry<HELM>(a.out_t, (int64_t)col * a.ld + row, a.scale_t * vr, a.scale_t * vi, true);
            } else {
                if (HELM) {
                    double xr = a.x[2 * col], xi = a.x[2 * col + 1];
                    if (a.conj_x) xi = -xi;
                    cr += vr * xr - vi * xi;
                    ci += vr * xi + vi * xr;
                } else {
                    cr += vr * a.x[col];
                }
            }
        }
        if (a.mode != 0) {
            if (HELM) {
                atomicAdd(a.y + 2 * row, a.scale * cr);
                atomicAdd(a.y + 2 * row + 1, a.scale * ci);
            } else {
                atomicAdd(a.y + row, a.scale * cr);
            }
        }
    }
}

// ----------------------------------------------------------------------------
// mass (identity) block: Q^2 rule on one triangle (identity_layer_3d.py:45-146)
// ----------------------------------------------------------------------------
struct MassArgs {
    int n_panels;
    const int32_t* panels;
    int nbx, nby;
    const int32_t* test_dof;
    const int32_t* trial_dof;
    const double* area;
    const double* gp;
    const double* gw;
    int Q;
    int cplx;
    int mode;
    double* out;
    int64_t ld;
    double scale;
    double* out_t;
    double scale_t;
    const double* x;
    double* y;
    int conj_x;
};

__global__ void mass_kernel(MassArgs a) {
    int id = blockIdx.x * blockDim.x + threadIdx.x;
    int per = a.nbx * a.nby;
    if (id >= a.n_panels * per) return;
    int li = id / per, r = id - li * per, ii = r / a.nby, jj = r - ii * a.nby;
    int row = a.test_dof[li * a.nbx + ii], col = a.trial_dof[li * a.nby + jj];
    if (row < 0 || col < 0) return;
    int bx = a.nbx == 1 ? -1 : ii, by = a.nby == 1 ? -1 : jj;
    double A = a.area[a.panels[li]];
    double acc = 0.0;
    for (int ix = 0; ix < a.Q; ++ix)
        for (int iy = 0; iy < a.Q; ++iy) {
            double r1 = a.gp[ix], r2 = a.gp[iy] * r1;
            double w = a.gw[ix] * a.gw[iy] * (A * 2.0);
            double px = bx < 0 ? 1.0 : shape_slot(r1, r2, bx);
            double py = by < 0 ? 1.0 : shape_slot(r1, r2, by);
            acc += (px * py) * w * r1;
        }
    if (a.mode == 0) {
        if (a.cplx) {
            atomicAdd(a.out + 2 * ((int64_t)row * a.ld + col), a.scale * acc);
            if (a.out_t) atomicAdd(a.out_t + 2 * ((int64_t)col * a.ld + row), a.scale_t * acc);
        } else {
            atomicAdd(a.out + (int64_t)row * a.ld + col, a.scale * acc);
            if (a.out_t) atomicAdd(a.out_t + (int64_t)col * a.ld + row, a.scale_t * acc);
        }
    } else {
        if (a.cplx) {
            double xr = a.x[2 * col], xi = a.x[2 * col + 1];
            if (a.conj_x) xi = -xi;
            atomicAdd(a.y + 2 * row, a.scale * acc * xr);
            atomicAdd(a.y + 2 * row + 1, a.scale * acc * xi);
        } else {
            atomicAdd(a.y + row, a.scale * acc * a.x[col]);
        }
    }
}

// Fused near field of the Dirichlet pass: V (P0 x P0, dense, `v`) and the
// matrix-free K g (P0 rows, NBD data bases on the trial panel, `k`) of one
// near pair from the same Sauter-Schwab points.  Each point's r, 1/r and
// e^{ikr} serve both integrands; the values and their accumulation are those
// of near_kernel<BEM_OP_V, HELM, 1, 1> and near_kernel<BEM_OP_K, HELM, 1, NBD>
// (the swapped coincide term takes K's kernel with -d, as there).  One warp
// per near pair.
template <bool HELM, int NBD>
__global__ void __launch_bounds__(128) near_vkg_kernel(NearArgs v, NearArgs k) {
    const int lane = threadIdx.x & 31;
    const int64_t pid = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (pid >= v.n_near) return;
    const int4 e = v.near[pid];
    const int gi = e.x, gj = e.y, rel = e.z;
    const int li = v.test_local[gi], lj = v.trial_local[gj];
    if (li < 0 || lj < 0) return;  // warp-uniform
    const int permx = v.quirk ? (0 | (1 << 2) | (2 << 4)) : (e.w & 63);
    const int permy = v.quirk ? (0 | (1 << 2) | (2 << 4)) : ((e.w >> 6) & 63);
    NearPanel X, Y;
    load_near_panel(X, v, gi, permx);
    load_near_panel(Y, v, gj, permy);
    int sy[NBD];
#pragma unroll
    for (int b = 0; b < NBD; ++b) sy[b] = NBD == 1 ? -1 : Y.slot[b];
    double av_re = 0.0, av_im = 0.0, ak_re[NBD], ak_im[NBD];
#pragma unroll
    for (int b = 0; b < NBD; ++b) ak_re[b] = ak_im[b] = 0.0;
    const double kk = v.k;
    auto add = [&](double r1x, double r2x, double r1y, double r2y, double wj, bool second, double px1, double px2,
                   double py1, double py2) {
        double x[3], yv[3];
        for (int c = 0; c < 3; ++c) {
            x[c] = (1.0 - r1x) * X.x1[c] + (r1x - r2x) * X.x2[c] + r2x * X.x3[c];
            yv[c] = (1.0 - r1y) * Y.x1[c] + (r1y - r2y) * Y.x2[c] + r2y * Y.x3[c];
        }
        const double dx = x[0] - yv[0], dy = x[1] - yv[1], dz = x[2] - yv[2];
        const double r2 = dx * dx + dy * dy + dz * dz;
        double r, rinv;
        dev_r_rinv(r2, r, rinv);
        // K: grad_G_y(x, y, n_y); the swapped coincide term grad_G_y(y, x, n_y)
        const double dn = (second ? -1.0 : 1.0) * (dx * Y.n[0] + dy * Y.n[1] + dz * Y.n[2]);
        const double t = dn * rinv * rinv * rinv;
        double vre, vim, kre, kim;
        if (HELM) {
            const double kr = kk * r;
            double sn, cs;
            dev_sincos(kr, &sn, &cs);
            vre = rinv * cs;
            vim = rinv * sn;
            kre = t * (cs + kr * sn);
            kim = t * (sn - kr * cs);
        } else {
            vre = rinv;
            vim = 0.0;
            kre = t;
            kim = 0.0;
        }
        av_re += vre * wj;
        av_im += vim * wj;
        (void)px1;
        (void)px2;
#pragma unroll
        for (int b = 0; b < NBD; ++b) {
            const double phy = NBD == 1 ? 1.0 : shape_slot(py1, py2, sy[b]);
            ak_re[b] += (kre * wj) * phy;
            ak_im[b] += (kim * wj) * phy;
        }
    };
    const int Q = v.Q;
    const int Q4 = Q * Q * Q * Q;
    for (int p = lane; p < Q4; p += 32) {
        int iw = p % Q, iz = (p / Q) % Q, iy = (p / (Q * Q)) % Q, ix = p / (Q * Q * Q);
        const double xsi = v.gp[ix], eta1 = v.gp[iy], eta2 = v.gp[iz], eta3 = v.gp[iw];
        const double weight = (v.gw[ix] * v.gw[iy] * (X.area * 2.0)) * (v.gw[iz] * v.gw[iw] * (Y.area * 2.0));
        near_points(rel, v.quirk != 0, xsi, eta1, eta2, eta3, weight, add);
    }
    av_re = warp_sum(av_re);
    av_im = warp_sum(av_im);
#pragma unroll
    for (int b = 0; b < NBD; ++b) {
        ak_re[b] = warp_sum(ak_re[b]);
        ak_im[b] = warp_sum(ak_im[b]);
    }
    if (lane != 0) return;
    {
        const int row = v.test_dof[li], col = v.trial_dof[lj];
        if (row >= 0 && col >= 0)
            add_entry<HELM>(v.out, (int64_t)row * v.ld + col, v.scale * BEM_INV4PI * av_re,
                            v.scale * BEM_INV4PI * av_im, true);
    }
    const int row = k.test_dof[li];
    if (row < 0) return;
    double cr = 0.0, ci = 0.0;
#pragma unroll
    for (int b = 0; b < NBD; ++b) {
        const int col = k.trial_dof[lj * NBD + b];
        if (col < 0) continue;
        const double vr = ak_re[b] * BEM_INV4PI, vi = ak_im[b] * BEM_INV4PI;
        if (HELM) {
            double xr = k.x[2 * col], xi = k.x[2 * col + 1];
            if (k.conj_x) xi = -xi;
            cr += vr * xr - vi * xi;
            ci += vr * xi + vi * xr;
        } else {
            cr += vr * k.x[col];
        }
    }
    if (HELM) {
        atomicAdd(k.y + 2 * row, k.scale * cr);
        atomicAdd(k.y + 2 * row + 1, k.scale * ci);
    } else {
        atomicAdd(k.y + row, k.scale * cr);
    }
}

// ----------------------------------------------------------------------------
// Fused Dirichlet-system pass: V (P0 x P0, dense) and the matrix-free K g
// (P0 test rows, g interpolated from P1 vertex data) over the same separate
// panel pairs.  Both integrands share the points, r, 1/r and e^{ikr}; the
// reference computes them in two sweeps (SingleLayer3d.forward,
// single_layer_3d.py:371-433, and DoubleLayer3d.apply_K_dot_D_boundary,
// double_layer_3d.py:440-501).
// ----------------------------------------------------------------------------
struct VkgArgs {
    const double* g;      // boundary data (real or complex interleaved)
    const int32_t* gdof;  // [n_trial * gnb] data index per trial panel basis
    int gnb;              // 1 (P0 data) or 3 (P1 data)
    const int32_t* rows;  // [n_test] rhs row of each test panel, <0 = skipped
    double* y;
    double scale;
    int conj;
};

// Boundary data on one panel, interpolated as g0 + phi1 (g1 - g0) + phi2 (g2 - g0)
// (P0 data: g0).  Constants are reproduced exactly whatever the FP32 rounding
// of the basis values: phi0 + phi1 + phi2 differs from 1 after rounding with the
// same pattern on every panel, which in the form sum_b phi_b g_b would act as a
// uniform weight error of the far field against the FP64 identity term.
template <bool HELM, typename T>
struct PanelData {
    T g0r = T(0), g0i = T(0), d1r = T(0), d1i = T(0), d2r = T(0), d2i = T(0);
    __device__ __forceinline__ void load(const VkgArgs& v, int l) {
        double gr[3] = {0.0, 0.0, 0.0}, gi[3] = {0.0, 0.0, 0.0};
        for (int b = 0; b < v.gnb; ++b) {
            const int d = v.gdof[l * v.gnb + b];
            if (d < 0) continue;
            gr[b] = HELM ? v.g[2 * d] : v.g[d];
            gi[b] = HELM ? (v.conj ? -v.g[2 * d + 1] : v.g[2 * d + 1]) : 0.0;
        }
        if (v.gnb != 3) {
            gr[1] = gr[2] = gr[0];
            gi[1] = gi[2] = gi[0];
        }
        g0r = T(gr[0]);
        g0i = T(gi[0]);
        d1r = T(gr[1] - gr[0]);
        d1i = T(gi[1] - gi[0]);
        d2r = T(gr[2] - gr[0]);
        d2i = T(gi[2] - gi[0]);
    }
    __device__ __forceinline__ void at(T p1, T p2, T& re, T& im) const {
        re = fma(p2, d2r, fma(p1, d1r, g0r));
        im = HELM ? fma(p2, d2i, fma(p1, d1i, g0i)) : T(0);
    }
};

template <bool HELM, typename T>
__global__ void __launch_bounds__(FAR_THREADS) far_vkg_kernel(FarArgs a, VkgArgs v) {
    using V4 = typename V4T<T>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V4* sx = reinterpret_cast<V4*>(smem_raw);
    T* sphi = reinterpret_cast<T*>(sx + FAR_TI * a.Q2);
    __shared__ int s_gi[FAR_TI];
    __shared__ int s_tri[FAR_TI][3];
    __shared__ double s_cen[FAR_TI][3];
    __shared__ double s_nrm[FAR_TI][3];

    const int Q2 = a.Q2;
    const int lj = blockIdx.x * FAR_THREADS + threadIdx.x;
    const int li0 = blockIdx.y * FAR_TI;
    const V4* pts = reinterpret_cast<const V4*>(a.pts);
    for (int idx = threadIdx.x; idx < FAR_TI * Q2; idx += FAR_THREADS) {
        int t = idx / Q2, q = idx - t * Q2;
        int li = li0 + t;
        if (li < a.n_test) sx[idx] = pts[(size_t)a.test_panels[li] * Q2 + q];
    }
    {
        const T* phi = reinterpret_cast<const T*>(a.phi);
        for (int idx = threadIdx.x; idx < Q2 * 3; idx += FAR_THREADS) sphi[idx] = phi[idx];
    }
    if (threadIdx.x < FAR_TI) {
        int li = li0 + threadIdx.x;
        int gi = li < a.n_test ? a.test_panels[li] : -1;
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
    double cen_j[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        tri_j[c] = a.tris[3 * gj + c];
        cen_j[c] = a.centroid[3 * gj + c];
    }
    const double nj64[3] = {a.normal[3 * gj + 0], a.normal[3 * gj + 1], a.normal[3 * gj + 2]};
    const T nx = T(nj64[0]), ny = T(nj64[1]), nz = T(nj64[2]);
    // trial data at the trial panel's basis functions (conjugated when asked)
    PanelData<HELM, T> gj_data;
    if (valid_j) gj_data.load(v, lj);
    const V4* ptsj = pts + (size_t)gj * Q2;
    const T kk = T(a.k);
    const int lane = threadIdx.x & 31;

    for (int t = 0; t < FAR_TI; ++t) {
        const int li = li0 + t;
        if (li >= a.n_test) break;
        const int gi = s_gi[t];
        const bool sep = valid_j && (bem_relation(s_tri[t], tri_j, gi == gj) == REL_SEPARATE);
        double av_re = 0.0, av_im = 0.0, ak_re = 0.0, ak_im = 0.0;
        if (sep) {
            // centroid difference as an unevaluated pair hi + lo: in FP32 a
            // single rounding of it would be one systematic error shared by
            // all GaussQR^4 terms of the pair
            const double dcx64 = s_cen[t][0] - cen_j[0], dcy64 = s_cen[t][1] - cen_j[1],
                         dcz64 = s_cen[t][2] - cen_j[2];
            const T dcx = T(dcx64), dcy = T(dcy64), dcz = T(dcz64);
            const T dlx = T(dcx64 - double(dcx)), dly = T(dcy64 - double(dcy)), dlz = T(dcz64 - double(dcz));
            Frame<T, HELM> fr;
            fr.init(dcx64, dcy64, dcz64, a.k, a.area[gi], a.area[gj], a.wcorr);
            const T Dn = T(dcx64 * nj64[0] + dcy64 * nj64[1] + dcz64 * nj64[2]);
            // x_a.n_j = x_a.(n_j - n_i) (x_a lies in the plane of panel i)
            const T mx = T(nj64[0] - s_nrm[t][0]), my = T(nj64[1] - s_nrm[t][1]), mz = T(nj64[2] - s_nrm[t][2]);
            const V4* sxt = sx + t * Q2;
            for (int b = 0; b < Q2; ++b) {
                const V4 yb = ptsj[b];
                const T ex = (dcx - yb.x) + dlx, ey = (dcy - yb.y) + dly, ez = (dcz - yb.z) + dlz;
                const T wx = fr.ux - yb.x, wy = fr.uy - yb.y, wz = fr.uz - yb.z;
                T sv_re = T(0), sv_im = T(0), sk_re = T(0), sk_im = T(0);
#pragma unroll 5
                for (int q = 0; q < Q2; ++q) {
                    const V4 xa = sxt[q];
                    T r, rinv, dn, phase;
                    if constexpr (Frame<T, HELM>::SPLIT) {
                        const T e_x = xa.x - yb.x, e_y = xa.y - yb.y, e_z = xa.z - yb.z;
                        const T sq = e_x * (xa.x + wx) + e_y * (xa.y + wy) + e_z * (xa.z + wz);
                        dev_r_rinv(fr.R2 + sq, r, rinv);
                        dn = fma(xa.x, mx, fma(xa.y, my, fma(xa.z, mz, Dn)));
                        phase = HELM ? kk * __fdividef(sq, r + fr.Rf) : T(0);
                    } else {
                        const T dx = xa.x + ex, dy = xa.y + ey, dz = xa.z + ez;
                        dev_r_rinv(dx * dx + dy * dy + dz * dz, r, rinv);
                        dn = dx * nx + dy * ny + dz * nz;
                        phase = kk * r;
                    }
                    const T wr = xa.w * rinv;
                    const T tk = xa.w * dn * rinv * rinv * rinv;
                    if (HELM) {
                        const T kr = kk * r;
                        T sn, cs;
                        if constexpr (Frame<T, HELM>::SPLIT)
                            dev_sincos_phase(phase, a.small_phase != 0, &sn, &cs);
                        else
                            dev_sincos(phase, &sn, &cs);
                        sv_re += wr * cs;
                        sv_im += wr * sn;
                        sk_re += tk * fma(kr, sn, cs);
                        sk_im += tk * fma(-kr, cs, sn);
                    } else {
                        sv_re += wr;
                        sk_re += tk;
                    }
                }
                const double wb = double(yb.w);
                av_re += wb * double(sv_re);
                av_im += wb * double(sv_im);
                // g interpolated at trial point b
                T gb_re, gb_im;
                gj_data.at(sphi[3 * b + 1], sphi[3 * b + 2], gb_re, gb_im);
                ak_re += wb * (double(sk_re) * double(gb_re) - double(sk_im) * double(gb_im));
                ak_im += wb * (double(sk_re) * double(gb_im) + double(sk_im) * double(gb_re));
            }
            fr.rotate(av_re, av_im);
            fr.rotate(ak_re, ak_im);
            const int row = a.test_dof[li];
            const int col = a.trial_dof[lj];
            if (row >= 0 && col >= 0)
                add_entry<HELM>(a.out, (int64_t)row * a.ld + col, a.scale * BEM_INV4PI * av_re,
                                a.scale * BEM_INV4PI * av_im, false);
        }
        ak_re = warp_sum(ak_re);
        if (HELM) ak_im = warp_sum(ak_im);
        if (lane == 0) {
            const int row = v.rows[li];
            if (row >= 0) {
                if (HELM) {
                    atomicAdd(v.y + 2 * row, v.scale * BEM_INV4PI * ak_re);
                    atomicAdd(v.y + 2 * row + 1, v.scale * BEM_INV4PI * ak_im);
                } else {
                    atomicAdd(v.y + row, v.scale * BEM_INV4PI * ak_re);
                }
            }
        }
    }
}

// ----------------------------------------------------------------------------
// Symmetric fused Dirichlet pass: the test and trial sides run over the same
// panel list, and the separate-pair rule places the same Q^2 points on a
// panel whether it is the test or the trial panel, so for i < j one
// evaluation at (x_a in i, y_b in j) gives
//   V_ij = V_ji          += w_a w_b e^{ikr}/r
//   (K g)_i              += w_a w_b ( d.n_j)/r^3 (1-ikr) e^{ikr} g_j(y_b)
//   (K g)_j              += w_a w_b (-d.n_i)/r^3 (1-ikr) e^{ikr} g_i(x_a)
// (d = x_a - y_b, g interpolated from the P1 vertex data).  Only tiles on or
// above the diagonal are launched; rows i are reduced across the warp, rows j
// accumulate per thread over the CTA's test panels.
// ----------------------------------------------------------------------------
template <bool HELM, typename T>
__global__ void __launch_bounds__(FAR_THREADS) far_vkg_sym_kernel(FarArgs a, VkgArgs v) {
    using V4 = typename V4T<T>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V4* sx = reinterpret_cast<V4*>(smem_raw);                        // [FAR_TI][Q2] test points
    T* sgx = reinterpret_cast<T*>(sx + FAR_TI * a.Q2);                // [FAR_TI][Q2][2] g at test points
    T* sphi = sgx + FAR_TI * a.Q2 * 2;                                // [Q2*3]
    __shared__ int s_gi[FAR_TI];
    __shared__ int s_tri[FAR_TI][3];
    __shared__ double s_cen[FAR_TI][3];
    __shared__ double s_nrm[FAR_TI][3];

    const int Q2 = a.Q2;
    const int n = a.n_test;  // == n_trial
    // tile (bx = trial tile of FAR_THREADS panels, by = test tile of FAR_TI panels);
    // skip tiles strictly below the diagonal
    const int j0 = blockIdx.x * FAR_THREADS;
    const int li0 = blockIdx.y * FAR_TI;
    if (j0 + FAR_THREADS - 1 <= li0) return;
    const int lj = j0 + threadIdx.x;
    const V4* pts = reinterpret_cast<const V4*>(a.pts);
    {
        const T* phi = reinterpret_cast<const T*>(a.phi);
        for (int idx = threadIdx.x; idx < Q2 * 3; idx += FAR_THREADS) sphi[idx] = phi[idx];
    }
    if (threadIdx.x < FAR_TI) {
        int li = li0 + threadIdx.x;
        int gi = li < n ? a.test_panels[li] : -1;
        s_gi[threadIdx.x] = gi;
        for (int c = 0; c < 3; ++c) {
            s_tri[threadIdx.x][c] = gi >= 0 ? a.tris[3 * gi + c] : -1;
            s_cen[threadIdx.x][c] = gi >= 0 ? a.centroid[3 * gi + c] : 0.0;
            s_nrm[threadIdx.x][c] = gi >= 0 ? a.normal[3 * gi + c] : 0.0;
        }
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < FAR_TI * Q2; idx += FAR_THREADS) {
        int t = idx / Q2, q = idx - t * Q2;
        int li = li0 + t;
        T gre = T(0), gim = T(0);
        if (li < n) {
            sx[idx] = pts[(size_t)s_gi[t] * Q2 + q];
            PanelData<HELM, T> gd;
            gd.load(v, li);
            gd.at(sphi[3 * q + 1], sphi[3 * q + 2], gre, gim);
        }
        sgx[2 * idx] = gre;
        sgx[2 * idx + 1] = gim;
    }
    __syncthreads();

    const bool valid_j = lj < n;
    const int gj = valid_j ? a.trial_panels[lj] : 0;
    int tri_j[3];
    double cen_j[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        tri_j[c] = a.tris[3 * gj + c];
        cen_j[c] = a.centroid[3 * gj + c];
    }
    const double nj64[3] = {a.normal[3 * gj + 0], a.normal[3 * gj + 1], a.normal[3 * gj + 2]};
    const T njx = T(nj64[0]), njy = T(nj64[1]), njz = T(nj64[2]);
    PanelData<HELM, T> gj_data;
    if (valid_j) gj_data.load(v, lj);
    const V4* ptsj = pts + (size_t)gj * Q2;
    const T kk = T(a.k);
    const int lane = threadIdx.x & 31;
    double rj_re = 0.0, rj_im = 0.0;  // this thread's contribution to row j

    for (int t = 0; t < FAR_TI; ++t) {
        const int li = li0 + t;
        if (li >= n) break;
        const int gi = s_gi[t];
        const bool sep = valid_j && li < lj && (bem_relation(s_tri[t], tri_j, gi == gj) == REL_SEPARATE);
        double av_re = 0.0, av_im = 0.0, ak_re = 0.0, ak_im = 0.0;
        if (sep) {
            // centroid difference as an unevaluated pair hi + lo: in FP32 a
            // single rounding of it would be one systematic error shared by
            // all GaussQR^4 terms of the pair
            const double dcx64 = s_cen[t][0] - cen_j[0], dcy64 = s_cen[t][1] - cen_j[1],
                         dcz64 = s_cen[t][2] - cen_j[2];
            const T dcx = T(dcx64), dcy = T(dcy64), dcz = T(dcz64);
            const T dlx = T(dcx64 - double(dcx)), dly = T(dcy64 - double(dcy)), dlz = T(dcz64 - double(dcz));
            const T nix = T(s_nrm[t][0]), niy = T(s_nrm[t][1]), niz = T(s_nrm[t][2]);
            Frame<T, HELM> fr;
            fr.init(dcx64, dcy64, dcz64, a.k, a.area[gi], a.area[gj], a.wcorr);
            const T Dnj = T(dcx64 * nj64[0] + dcy64 * nj64[1] + dcz64 * nj64[2]);
            const T Dni = T(dcx64 * s_nrm[t][0] + dcy64 * s_nrm[t][1] + dcz64 * s_nrm[t][2]);
            // n_j - n_i: x_a.n_j = x_a.(n_j - n_i), y_b.n_i = -y_b.(n_j - n_i) (points lie in their
            // panel's plane); small for the nearly coplanar close pairs
            const T mx = T(nj64[0] - s_nrm[t][0]), my = T(nj64[1] - s_nrm[t][1]), mz = T(nj64[2] - s_nrm[t][2]);
            double pj_re = 0.0, pj_im = 0.0;  // this pair's contribution to row j
            const V4* sxt = sx + t * Q2;
            const T* sgt = sgx + 2 * t * Q2;
            for (int b = 0; b < Q2; ++b) {
                const V4 yb = ptsj[b];
                const T ex = (dcx - yb.x) + dlx, ey = (dcy - yb.y) + dly, ez = (dcz - yb.z) + dlz;
                const T wx = fr.ux - yb.x, wy = fr.uy - yb.y, wz = fr.uz - yb.z;
                // d.n_i = D.n_i - y_b.n_i (x_a lies in the plane of panel i)
                const T dni = Dni + (yb.x * mx + yb.y * my + yb.z * mz);
                // two independent accumulator sets (even / odd test points):
                // shorter FP32 summation chains and more independent work
                T acc[2][6];
#pragma unroll
                for (int u = 0; u < 2; ++u)
#pragma unroll
                    for (int w = 0; w < 6; ++w) acc[u][w] = T(0);
                auto term = [&](int q, T* A) {
                    const V4 xa = sxt[q];
                    T r, rinv, dnj, dnx, phase;
                    if constexpr (Frame<T, HELM>::SPLIT) {
                        const T e_x = xa.x - yb.x, e_y = xa.y - yb.y, e_z = xa.z - yb.z;
                        const T sq = e_x * (xa.x + wx) + e_y * (xa.y + wy) + e_z * (xa.z + wz);
                        dev_r_rinv(fr.R2 + sq, r, rinv);
                        // d.n_j = D.n_j + x_a.n_j (y_b lies in the plane of panel j)
                        dnj = fma(xa.x, mx, fma(xa.y, my, fma(xa.z, mz, Dnj)));
                        dnx = dni;
                        phase = HELM ? kk * __fdividef(sq, r + fr.Rf) : T(0);
                    } else {
                        const T dx = xa.x + ex, dy = xa.y + ey, dz = xa.z + ez;
                        dev_r_rinv(dx * dx + dy * dy + dz * dz, r, rinv);
                        dnj = dx * njx + dy * njy + dz * njz;
                        dnx = dx * nix + dy * niy + dz * niz;
                        phase = kk * r;
                    }
                    const T wr = xa.w * rinv;
                    const T wr3 = wr * (rinv * rinv);
                    const T tj = wr3 * dnj;
                    const T ti = -wr3 * dnx;
                    if (HELM) {
                        const T kr = kk * r;
                        T sn, cs;
                        if constexpr (Frame<T, HELM>::SPLIT)
                            dev_sincos_phase(phase, a.small_phase != 0, &sn, &cs);
                        else
                            dev_sincos(phase, &sn, &cs);
                        const T f_re = fma(kr, sn, cs), f_im = fma(-kr, cs, sn);
                        A[0] = fma(wr, cs, A[0]);
                        A[1] = fma(wr, sn, A[1]);
                        A[2] = fma(tj, f_re, A[2]);
                        A[3] = fma(tj, f_im, A[3]);
                        const T h_re = ti * f_re, h_im = ti * f_im;
                        const T gre = sgt[2 * q], gimv = sgt[2 * q + 1];
                        A[4] += h_re * gre - h_im * gimv;
                        A[5] += h_re * gimv + h_im * gre;
                    } else {
                        A[0] += wr;
                        A[2] += tj;
                        A[4] = fma(ti, sgt[2 * q], A[4]);
                    }
                };
                int q = 0;
#pragma unroll 2
                for (; q + 1 < Q2; q += 2) {
                    term(q, acc[0]);
                    term(q + 1, acc[1]);
                }
                if (q < Q2) term(q, acc[0]);
                const T sv_re = acc[0][0] + acc[1][0], sv_im = acc[0][1] + acc[1][1];
                const T sk_re = acc[0][2] + acc[1][2], sk_im = acc[0][3] + acc[1][3];
                const T s2_re = acc[0][4] + acc[1][4], s2_im = acc[0][5] + acc[1][5];
                const double wb = double(yb.w);
                av_re += wb * double(sv_re);
                av_im += wb * double(sv_im);
                T gb_re, gb_im;
                gj_data.at(sphi[3 * b + 1], sphi[3 * b + 2], gb_re, gb_im);
                ak_re += wb * (double(sk_re) * double(gb_re) - double(sk_im) * double(gb_im));
                ak_im += wb * (double(sk_re) * double(gb_im) + double(sk_im) * double(gb_re));
                pj_re += wb * double(s2_re);
                pj_im += wb * double(s2_im);
            }
            fr.rotate(av_re, av_im);
            fr.rotate(ak_re, ak_im);
            fr.rotate(pj_re, pj_im);
            rj_re += pj_re;
            rj_im += pj_im;
            const int row = a.test_dof[li];
            const int col = a.trial_dof[lj];
            if (row >= 0 && col >= 0) {
                const double vr = a.scale * BEM_INV4PI * av_re, vi = a.scale * BEM_INV4PI * av_im;
                add_entry<HELM>(a.out, (int64_t)row * a.ld + col, vr, vi, false);
                add_entry<HELM>(a.out, (int64_t)col * a.ld + row, vr, vi, false);
            }
        }
        ak_re = warp_sum(ak_re);
        if (HELM) ak_im = warp_sum(ak_im);
        if (lane == 0) {
            const int row = v.rows[li];
            if (row >= 0) {
                if (HELM) {
                    atomicAdd(v.y + 2 * row, v.scale * BEM_INV4PI * ak_re);
                    atomicAdd(v.y + 2 * row + 1, v.scale * BEM_INV4PI * ak_im);
                } else {
                    atomicAdd(v.y + row, v.scale * BEM_INV4PI * ak_re);
                }
            }
        }
    }
    if (valid_j) {
        const int row = v.rows[lj];
        if (row >= 0 && (rj_re != 0.0 || rj_im != 0.0)) {
            if (HELM) {
                atomicAdd(v.y + 2 * row, v.scale * BEM_INV4PI * rj_re);
                atomicAdd(v.y + 2 * row + 1, v.scale * BEM_INV4PI * rj_im);
            } else {
                atomicAdd(v.y + row, v.scale * BEM_INV4PI * rj_re);
            }
        }
    }
}

// ----------------------------------------------------------------------------
// FP32 symmetric fused Dirichlet pass on packed FP32x2 arithmetic: the sweep
// of far_vkg_sym_kernel<HELM, float> with two test points (q, q+1) in the two
// lanes of every FFMA2/FMUL2/FADD2 (the lanes are the even/odd accumulator
// sets, so the order of summation over q is that of the scalar kernel).  A
// packed instruction does two FMAs in one issue slot at the per-lane FMA
// rate; the scalar kernel is bound by instruction issue.  The per-point work
// is also reduced, each step exact algebra on the scalar kernel's terms:
//   s = e.(2D + e) = |x_a|^2 + x_a.U_b + C_b,  U_b = 2D - 2y_b,
//                                              C_b = -y_b.(2D - y_b)
//     (|x_a|^2 once per point, U_b and C_b once per trial point; the absolute
//     FP32 error stays of order eps |D| |e|, as in the product form);
//   d.n_j = D.n_j + x_a.(n_j - n_i) depends on the pair and the test point
//     only: it is formed once per pair and kept in shared memory per thread;
//   -d.n_i = -(D.n_i - y_b.(n_j - n_i)) is constant over the test points of a
//     trial point and multiplies the (K g)_j sum after the loop over q;
//   the sine/cosine polynomials drop their last term when the host has
//     bounded the phase by 0.3 (small_phase == 2; truncation below 6e-11).
// Shared memory holds the test points pairwise as structure-of-arrays:
// (x0 x1 y0 y1), (z0 z1 w0 w1), g (re0 re1 im0 im1) and |x|^2 (xx0 xx1); an
// odd Q^2 is padded by a copy of the last point with weight 0 and g = 0.
// ----------------------------------------------------------------------------

// One trial point y_b against all test-point pairs of panel t: accumulates
// the V sum (A0, A1), the (K g)_i kernel sum (A2, A3) and the (K g)_j sum
// without its -d.n_i factor (A4 - A6, A5).
template <bool HELM, int PH>
__device__ __forceinline__ void x2_trial_point(int P2, const float4* __restrict__ sxyt,
                                               const float4* __restrict__ szwt, const float4* __restrict__ sgt,
                                               const float2* __restrict__ sxxt, const float2* __restrict__ sdn,
                                               float2 U0, float2 U1, float2 U2, float2 CB, float2 R2, float2 RF,
                                               float2 KK, float2 NKK, float2& A0, float2& A1, float2& A2,
                                               float2& A3, float2& A4, float2& A5, float2& A6) {
#pragma unroll 4
    for (int p = 0; p < P2; ++p) {
        const float4 xy = sxyt[p], zw = szwt[p];
        const float2 X = make_float2(xy.x, xy.y), Y = make_float2(xy.z, xy.w);
        const float2 Z = make_float2(zw.x, zw.y), W = make_float2(zw.z, zw.w);
        const float2 sq = ffma2(X, U0, ffma2(Y, U1, ffma2(Z, U2, fadd2(sxxt[p], CB))));
        float2 r, rinv;
        dev_r_rinv2(fadd2(R2, sq), r, rinv);
        const float2 dnj = sdn[p * FAR_THREADS];
        const float2 wr = fmul2(W, rinv);
        const float2 wr3 = fmul2(wr, fmul2(rinv, rinv));
        if (HELM) {
            const float2 rr = fadd2(r, RF);
            const float2 inv = make_float2(__fdividef(1.0f, rr.x), __fdividef(1.0f, rr.y));
            const float2 phase = fmul2(KK, fmul2(sq, inv));
            float2 sn, cs;
            if (PH == 2) {
                dev_sincos_poly2<true>(phase, sn, cs);
            } else if (PH == 1) {
                dev_sincos_poly2<false>(phase, sn, cs);
            } else {
                dev_sincos(phase.x, &sn.x, &cs.x);
                dev_sincos(phase.y, &sn.y, &cs.y);
            }
            const float2 kr = fmul2(KK, r), nkr = fmul2(NKK, r);
            // u = wr3 (1 - ikr) e^{ik(r-R)}
            const float2 u_re = fmul2(wr3, ffma2(kr, sn, cs)), u_im = fmul2(wr3, ffma2(nkr, cs, sn));
            A0 = ffma2(wr, cs, A0);
            A1 = ffma2(wr, sn, A1);
            A2 = ffma2(dnj, u_re, A2);
            A3 = ffma2(dnj, u_im, A3);
            const float4 g = sgt[p];
            const float2 GR = make_float2(g.x, g.y), GI = make_float2(g.z, g.w);
            A4 = ffma2(u_re, GR, A4);
            A6 = ffma2(u_im, GI, A6);
            A5 = ffma2(u_re, GI, A5);
            A5 = ffma2(u_im, GR, A5);
        } else {
            A0 = fadd2(A0, wr);
            A2 = ffma2(dnj, wr3, A2);
            const float4 g = sgt[p];
            A4 = ffma2(wr3, make_float2(g.x, g.y), A4);
        }
    }
}

template <bool HELM, int PH>
__global__ void __launch_bounds__(FAR_THREADS, 5) far_vkg_sym_x2_kernel(FarArgs a, VkgArgs v) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int Q2 = a.Q2;
    const int P2 = (Q2 + 1) / 2;                                    // point pairs per panel
    float4* sxy = reinterpret_cast<float4*>(smem_raw);              // [FAR_TI][P2] (x0 x1 y0 y1)
    float4* szw = sxy + FAR_TI * P2;                                // [FAR_TI][P2] (z0 z1 w0 w1)
    float4* sg = szw + FAR_TI * P2;                                 // [FAR_TI][P2] (re0 re1 im0 im1)
    float2* sxx = reinterpret_cast<float2*>(sg + FAR_TI * P2);      // [FAR_TI][P2] (|x0|^2 |x1|^2)
    float2* sdn = sxx + FAR_TI * P2;                                // [P2][FAR_THREADS] d.n_j of this thread's pair
    float* sphi = reinterpret_cast<float*>(sdn + P2 * FAR_THREADS);  // [Q2*3]
    __shared__ int s_gi[FAR_TI];
    __shared__ int s_tri[FAR_TI][3];
    __shared__ double s_cen[FAR_TI][3];
    __shared__ double s_nrm[FAR_TI][3];

    const int n = a.n_test;  // == n_trial
    const int j0 = blockIdx.x * FAR_THREADS;
    const int li0 = blockIdx.y * FAR_TI;
    if (j0 + FAR_THREADS - 1 <= li0) return;
    const int lj = j0 + threadIdx.x;
    const float4* pts = reinterpret_cast<const float4*>(a.pts);
    {
        const float* phi = reinterpret_cast<const float*>(a.phi);
        for (int idx = threadIdx.x; idx < Q2 * 3; idx += FAR_THREADS) sphi[idx] = phi[idx];
    }
    if (threadIdx.x < FAR_TI) {
        int li = li0 + threadIdx.x;
        int gi = li < n ? a.test_panels[li] : -1;
        s_gi[threadIdx.x] = gi;
        for (int c = 0; c < 3; ++c) {
            s_tri[threadIdx.x][c] = gi >= 0 ? a.tris[3 * gi + c] : -1;
            s_cen[threadIdx.x][c] = gi >= 0 ? a.centroid[3 * gi + c] : 0.0;
            s_nrm[threadIdx.x][c] = gi >= 0 ? a.normal[3 * gi + c] : 0.0;
        }
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < FAR_TI * P2; idx += FAR_THREADS) {
        const int t = idx / P2, p = idx - t * P2;
        const int li = li0 + t;
        const int q0 = 2 * p, q1 = 2 * p + 1 < Q2 ? 2 * p + 1 : Q2 - 1;
        float4 x0 = make_float4(0.f, 0.f, 0.f, 0.f), x1 = x0;
        float g0r = 0.f, g0i = 0.f, g1r = 0.f, g1i = 0.f;
        if (li < n) {
            x0 = pts[(size_t)s_gi[t] * Q2 + q0];
            x1 = pts[(size_t)s_gi[t] * Q2 + q1];
            PanelData<HELM, float> gd;
            gd.load(v, li);
            gd.at(sphi[3 * q0 + 1], sphi[3 * q0 + 2], g0r, g0i);
            gd.at(sphi[3 * q1 + 1], sphi[3 * q1 + 2], g1r, g1i);
            if (2 * p + 1 >= Q2) {  // padding point: weight 0, data 0
                x1.w = 0.f;
                g1r = g1i = 0.f;
            }
        }
        sxy[idx] = make_float4(x0.x, x1.x, x0.y, x1.y);
        szw[idx] = make_float4(x0.z, x1.z, x0.w, x1.w);
        sg[idx] = make_float4(g0r, g1r, g0i, g1i);
        sxx[idx] = make_float2(fmaf(x0.x, x0.x, fmaf(x0.y, x0.y, x0.z * x0.z)),
                               fmaf(x1.x, x1.x, fmaf(x1.y, x1.y, x1.z * x1.z)));
    }
    __syncthreads();

    const bool valid_j = lj < n;
    const int gj = valid_j ? a.trial_panels[lj] : 0;
    int tri_j[3];
    double cen_j[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        tri_j[c] = a.tris[3 * gj + c];
        cen_j[c] = a.centroid[3 * gj + c];
    }
    const double nj64[3] = {a.normal[3 * gj + 0], a.normal[3 * gj + 1], a.normal[3 * gj + 2]};
    PanelData<HELM, float> gj_data;
    if (valid_j) gj_data.load(v, lj);
    const float4* ptsj = pts + (size_t)gj * Q2;
    const float2 KK = f2(float(a.k)), NKK = f2(-float(a.k));
    const int lane = threadIdx.x & 31;
    float2* sdn_me = sdn + threadIdx.x;
    double rj_re = 0.0, rj_im = 0.0;

    for (int t = 0; t < FAR_TI; ++t) {
        const int li = li0 + t;
        if (li >= n) break;
        const int gi = s_gi[t];
        const bool sep = valid_j && li < lj && (bem_relation(s_tri[t], tri_j, gi == gj) == REL_SEPARATE);
        double av_re = 0.0, av_im = 0.0, ak_re = 0.0, ak_im = 0.0;
        if (sep) {
            const double dcx64 = s_cen[t][0] - cen_j[0], dcy64 = s_cen[t][1] - cen_j[1],
                         dcz64 = s_cen[t][2] - cen_j[2];
            Frame<float, HELM> fr;
            fr.init(dcx64, dcy64, dcz64, a.k, a.area[gi], a.area[gj], a.wcorr);
            const float Dnj = float(dcx64 * nj64[0] + dcy64 * nj64[1] + dcz64 * nj64[2]);
            const float Dni = float(dcx64 * s_nrm[t][0] + dcy64 * s_nrm[t][1] + dcz64 * s_nrm[t][2]);
            const float mx = float(nj64[0] - s_nrm[t][0]), my = float(nj64[1] - s_nrm[t][1]),
                        mz = float(nj64[2] - s_nrm[t][2]);
            const float4* sxyt = sxy + t * P2;
            const float4* szwt = szw + t * P2;
            const float4* sgt = sg + t * P2;
            const float2* sxxt = sxx + t * P2;
            {
                // d.n_j = D.n_j + x_a.(n_j - n_i) of this pair's test points
                const float2 MX = f2(mx), MY = f2(my), MZ = f2(mz), DNJ = f2(Dnj);
                for (int p = 0; p < P2; ++p) {
                    const float4 xy = sxyt[p], zw = szwt[p];
                    sdn_me[p * FAR_THREADS] = ffma2(make_float2(xy.x, xy.y), MX,
                                                    ffma2(make_float2(xy.z, xy.w), MY,
                                                          ffma2(make_float2(zw.x, zw.y), MZ, DNJ)));
                }
            }
            const float2 R2 = f2(fr.R2), RF = f2(fr.Rf);
            double pj_re = 0.0, pj_im = 0.0;
            for (int b = 0; b < Q2; ++b) {
                const float4 yb = ptsj[b];
                const float wx = fr.ux - yb.x, wy = fr.uy - yb.y, wz = fr.uz - yb.z;
                const float2 U0 = f2(wx - yb.x), U1 = f2(wy - yb.y), U2 = f2(wz - yb.z);
                const float2 CB = f2(-fmaf(yb.x, wx, fmaf(yb.y, wy, yb.z * wz)));
                // -d.n_i = -(D.n_i - y_b.(n_j - n_i)), constant over the test points
                const float ndni = -(Dni + (yb.x * mx + yb.y * my + yb.z * mz));
                float2 A0 = f2(0.f), A1 = f2(0.f), A2 = f2(0.f), A3 = f2(0.f), A4 = f2(0.f), A5 = f2(0.f),
                       A6 = f2(0.f);
                x2_trial_point<HELM, PH>(P2, sxyt, szwt, sgt, sxxt, sdn_me, U0, U1, U2, CB, R2, RF, KK, NKK, A0, A1,
                                         A2, A3, A4, A5, A6);
                const float sv_re = A0.x + A0.y, sv_im = A1.x + A1.y;
                const float sk_re = A2.x + A2.y, sk_im = A3.x + A3.y;
                const float s2_re = ndni * ((A4.x + A4.y) - (A6.x + A6.y)), s2_im = ndni * (A5.x + A5.y);
                const double wb = double(yb.w);
                av_re += wb * double(sv_re);
                av_im += wb * double(sv_im);
                float gb_re, gb_im;
                gj_data.at(sphi[3 * b + 1], sphi[3 * b + 2], gb_re, gb_im);
                ak_re += wb * (double(sk_re) * double(gb_re) - double(sk_im) * double(gb_im));
                ak_im += wb * (double(sk_re) * double(gb_im) + double(sk_im) * double(gb_re));
                pj_re += wb * double(s2_re);
                pj_im += wb * double(s2_im);
            }
            fr.rotate(av_re, av_im);
            fr.rotate(ak_re, ak_im);
            fr.rotate(pj_re, pj_im);
            rj_re += pj_re;
            rj_im += pj_im;
            const int row = a.test_dof[li];
            const int col = a.trial_dof[lj];
            if (row >= 0 && col >= 0) {
                const double vr = a.scale * BEM_INV4PI * av_re, vi = a.scale * BEM_INV4PI * av_im;
                add_entry<HELM>(a.out, (int64_t)row * a.ld + col, vr, vi, false);
                add_entry<HELM>(a.out, (int64_t)col * a.ld + row, vr, vi, false);
            }
        }
        ak_re = warp_sum(ak_re);
        if (HELM) ak_im = warp_sum(ak_im);
        if (lane == 0) {
            const int row = v.rows[li];
            if (row >= 0) {
                if (HELM) {
                    atomicAdd(v.y + 2 * row, v.scale * BEM_INV4PI * ak_re);
                    atomicAdd(v.y + 2 * row + 1, v.scale * BEM_INV4PI * ak_im);
                } else {
                    atomicAdd(v.y + row, v.scale * BEM_INV4PI * ak_re);
                }
            }
        }
    }
    if (valid_j) {
        const int row = v.rows[lj];
        if (row >= 0 && (rj_re != 0.0 || rj_im != 0.0)) {
            if (HELM) {
                atomicAdd(v.y + 2 * row, v.scale * BEM_INV4PI * rj_re);
                atomicAdd(v.y + 2 * row + 1, v.scale * BEM_INV4PI * rj_im);
            } else {
                atomicAdd(v.y + row, v.scale * BEM_INV4PI * rj_re);
            }
        }
    }
}

template <int OP, bool HELM, int NBX, int NBY>
int launch_op(bem_ctx* ctx, const FarArgs& fa, const NearArgs& na, bool fp32, cudaStream_t s) {
    dim3 grid((fa.n_trial + FAR_THREADS - 1) / FAR_THREADS, (fa.n_test + FAR_TI - 1) / FAR_TI);
    if (grid.y > 65535) return bem_fail(ctx, BEM_ERR_INVALID, "too many test panels for one launch");
    if (fa.n_test > 0 && fa.n_trial > 0 && !fa.skip_far) {
        size_t smem;
        if (fp32) {
            smem = FAR_TI * fa.Q2 * sizeof(float4) + fa.Q2 * 3 * sizeof(float);
            far_kernel<OP, HELM, NBX, NBY, float><<<grid, FAR_THREADS, smem, s>>>(fa);
        } else {
            smem = FAR_TI * fa.Q2 * sizeof(double4) + fa.Q2 * 3 * sizeof(double);
            far_kernel<OP, HELM, NBX, NBY, double><<<grid, FAR_THREADS, smem, s>>>(fa);
        }
        ctx->launches++;
        if (int rc = bem_check_cuda(ctx, cudaGetLastError(), "far_kernel launch")) return rc;
    }
    if (na.n_near > 0) {
        int warps = 4;
        int64_t blocks = (na.n_near + warps - 1) / warps;
        near_kernel<OP, HELM, NBX, NBY><<<(unsigned)blocks, 32 * warps, 0, s>>>(na);
        ctx->launches++;
        if (int rc = bem_check_cuda(ctx, cudaGetLastError(), "near_kernel launch")) return rc;
    }
    return BEM_OK;
}

template <int OP, bool HELM>
int dispatch_nb(bem_ctx* ctx, int nbx, int nby, const FarArgs& fa, const NearArgs& na, bool fp32, cudaStream_t s) {
    if (nbx == 1 && nby == 1) return launch_op<OP, HELM, 1, 1>(ctx, fa, na, fp32, s);
    if (nbx == 1 && nby == 3) return launch_op<OP, HELM, 1, 3>(ctx, fa, na, fp32, s);
    if (nbx == 3 && nby == 1) return launch_op<OP, HELM, 3, 1>(ctx, fa, na, fp32, s);
    if (nbx == 3 && nby == 3) return launch_op<OP, HELM, 3, 3>(ctx, fa, na, fp32, s);
    return bem_fail(ctx, BEM_ERR_INVALID, "nb must be 1 (P0) or 3 (P1)");
}

template <int OP>
int dispatch_helm(bem_ctx* ctx, bool helm, int nbx, int nby, const FarArgs& fa, const NearArgs& na, bool fp32,
                  cudaStream_t s) {
    return helm ? dispatch_nb<OP, true>(ctx, nbx, nby, fa, na, fp32, s)
                : dispatch_nb<OP, false>(ctx, nbx, nby, fa, na, fp32, s);
}

}  // namespace

int bem_launch_geometry(bem_ctx* ctx, cudaStream_t s) {
    int threads = 128;
    int blocks = (ctx->nt + threads - 1) / threads;
    geometry_kernel<<<blocks, threads, 0, s>>>(ctx->nt, ctx->Q, ctx->verts, ctx->tris, ctx->gp, ctx->gw, ctx->area,
                                                ctx->normal, ctx->centroid, ctx->curl, ctx->pts64, ctx->pts32,
                                                ctx->flags);
    ctx->launches++;
    return bem_check_cuda(ctx, cudaGetLastError(), "geometry_kernel launch");
}

// Class of the bound on the FP32 split phase |k (r - R)| <= k (rho_i + rho_j):
// 2 when <= 0.3 (short polynomials), 1 when <= 0.78 < pi/4 (no reduction), 0 otherwise
int bem_phase_class(double bound) { return bound <= 0.3 ? 2 : (bound <= 0.78 ? 1 : 0); }

int bem_fill_local_map(bem_ctx* ctx, const bem_space* sp, int32_t* map, cudaStream_t s) {
    if (int rc = bem_check_cuda(ctx, cudaMemsetAsync(map, 0xff, sizeof(int32_t) * ctx->nt, s), "memset")) return rc;
    if (sp->n_panels > 0) {
        scatter_local_kernel<<<(sp->n_panels + 127) / 128, 128, 0, s>>>(sp->n_panels, sp->panels, map, ctx->nt,
                                                                        ctx->flags);
        ctx->launches++;
        return bem_check_cuda(ctx, cudaGetLastError(), "scatter_local_kernel launch");
    }
    return BEM_OK;
}

int bem_launch_assemble(bem_ctx* ctx, const bem_op_desc* op, const bem_space* test, const bem_space* trial,
                        int mode, void* out, int64_t ld, double scale, void* out_t, double scale_t, const void* x,
                        void* y, int conj_x, cudaStream_t s) {
    return bem_launch_assemble_parts(ctx, op, test, trial, mode, out, ld, scale, out_t, scale_t, x, y, conj_x, s,
                                     false);
}

int bem_launch_assemble_parts(bem_ctx* ctx, const bem_op_desc* op, const bem_space* test, const bem_space* trial,
                              int mode, void* out, int64_t ld, double scale, void* out_t, double scale_t,
                              const void* x, void* y, int conj_x, cudaStream_t s, bool near_only) {
    if (int rc = bem_fill_local_map(ctx, test, ctx->test_local, s)) return rc;
    if (int rc = bem_fill_local_map(ctx, trial, ctx->trial_local, s)) return rc;
    bool fp32 = op->precision == BEM_PREC_MIXED;
    FarArgs fa{};
    fa.skip_far = near_only ? 1 : 0;
    fa.n_test = test->n_panels;
    fa.n_trial = trial->n_panels;
    fa.test_panels = test->panels;
    fa.test_dof = test->dof;
    fa.trial_panels = trial->panels;
    fa.trial_dof = trial->dof;
    fa.tris = ctx->tris;
    fa.centroid = ctx->centroid;
    fa.normal = ctx->normal;
    fa.curl = ctx->curl;
    fa.area = ctx->area;
    fa.wcorr = ctx->wcorr32;
    fa.small_phase = fp32 && op->kernel == BEM_KERNEL_HELMHOLTZ ? bem_phase_class(op->k * 2.0 * ctx->rho_max) : 0;
    fa.pts = fp32 ? (const void*)ctx->pts32 : (const void*)ctx->pts64;
    fa.phi = fp32 ? (const void*)ctx->phi32 : (const void*)ctx->phi64;
    fa.phi64 = ctx->phi64;
    fa.Q2 = ctx->Q2;
    fa.k = op->k;
    fa.k2 = op->k2;
    fa.dk = op->deriv_k ? 1 : 0;
    fa.mode = mode;
    fa.out = (double*)out;
    fa.ld = ld;
    fa.scale = scale;
    fa.out_t = (double*)out_t;
    fa.scale_t = scale_t;
    fa.x = (const double*)x;
    fa.y = (double*)y;
    fa.conj_x = conj_x;

    NearArgs na;
    na.n_near = ctx->n_near;
    na.near = ctx->near;
    na.test_local = ctx->test_local;
    na.trial_local = ctx->trial_local;
    na.test_dof = test->dof;
    na.trial_dof = trial->dof;
    na.tris = ctx->tris;
    na.verts = ctx->verts;
    na.area = ctx->area;
    na.normal = ctx->normal;
    na.curl = ctx->curl;
    na.gp = ctx->gp;
    na.gw = ctx->gw;
    na.Q = ctx->Q;
    na.k = op->k;
    na.k2 = op->k2;
    na.dk = op->deriv_k ? 1 : 0;
    na.quirk = op->quirk;
    na.mode = mode;
    na.out = (double*)out;
    na.ld = ld;
    na.scale = scale;
    na.out_t = (double*)out_t;
    na.scale_t = scale_t;
    na.x = (const double*)x;
    na.y = (double*)y;
    na.conj_x = conj_x;

    bool helm = op->kernel == BEM_KERNEL_HELMHOLTZ;
    switch (op->op) {
        case BEM_OP_V: return dispatch_helm<BEM_OP_V>(ctx, helm, test->nb, trial->nb, fa, na, fp32, s);
        case BEM_OP_K: return dispatch_helm<BEM_OP_K>(ctx, helm, test->nb, trial->nb, fa, na, fp32, s);
        case BEM_OP_KP: return dispatch_helm<BEM_OP_KP>(ctx, helm, test->nb, trial->nb, fa, na, fp32, s);
        case BEM_OP_W: return dispatch_helm<BEM_OP_W>(ctx, helm, test->nb, trial->nb, fa, na, fp32, s);
        default: return bem_fail(ctx, BEM_ERR_INVALID, "unknown operator");
    }
}

int bem_launch_dirichlet(bem_ctx* ctx, const bem_op_desc* op, const bem_space* test, const bem_space* trial,
                         void* out, int64_t ld, double scale, const bem_space* rows, const bem_space* data,
                         const void* g, void* y, double scale_k, int conj_g, cudaStream_t s) {
    if (int rc = bem_fill_local_map(ctx, test, ctx->test_local, s)) return rc;
    if (int rc = bem_fill_local_map(ctx, trial, ctx->trial_local, s)) return rc;
    // the FP64 near-pair kernels run on the side stream, concurrently with the
    // FP32 far sweep (different pipes; they write other V entries and add to
    // the right-hand side atomically); the caller's stream waits for both
    if (int rc = bem_lookahead_stream(ctx)) return rc;
    const bool side = ctx->n_near > 0;
    if (side) {
        cudaEventRecord(ctx->ev_next, s);
        cudaStreamWaitEvent(ctx->aux, ctx->ev_next, 0);
    }
    const cudaStream_t sn = side ? ctx->aux : s;
    const bool fp32 = op->precision == BEM_PREC_MIXED;
    const bool helm = op->kernel == BEM_KERNEL_HELMHOLTZ;
    FarArgs fa{};
    fa.n_test = test->n_panels;
    fa.n_trial = trial->n_panels;
    fa.test_panels = test->panels;
    fa.test_dof = test->dof;
    fa.trial_panels = trial->panels;
    fa.trial_dof = trial->dof;
    fa.tris = ctx->tris;
    fa.centroid = ctx->centroid;
    fa.normal = ctx->normal;
    fa.curl = ctx->curl;
    fa.area = ctx->area;
    fa.wcorr = ctx->wcorr32;
    fa.small_phase = fp32 && op->kernel == BEM_KERNEL_HELMHOLTZ ? bem_phase_class(op->k * 2.0 * ctx->rho_max) : 0;
    fa.pts = fp32 ? (const void*)ctx->pts32 : (const void*)ctx->pts64;
    fa.phi = fp32 ? (const void*)ctx->phi32 : (const void*)ctx->phi64;
    fa.phi64 = ctx->phi64;
    fa.Q2 = ctx->Q2;
    fa.k = op->k;
    fa.k2 = op->k2;
    fa.mode = 0;
    fa.out = (double*)out;
    fa.ld = ld;
    fa.scale = scale;
    VkgArgs va{(const double*)g, data->dof, data->nb, rows->dof, (double*)y, scale_k, conj_g};
    dim3 grid((fa.n_trial + FAR_THREADS - 1) / FAR_THREADS, (fa.n_test + FAR_TI - 1) / FAR_TI);
    if (grid.y > 65535) return bem_fail(ctx, BEM_ERR_INVALID, "too many test panels for one launch");
    // same panels and dofs on both sides: the symmetric sweep over i < j
    const bool sym = test->n_panels == trial->n_panels && test->panels == trial->panels &&
                     test->dof == trial->dof && rows->n_panels == test->n_panels;
    if (fa.n_test > 0 && fa.n_trial > 0 && sym) {
        if (fp32) {
            const int P2 = (fa.Q2 + 1) / 2;
            size_t smem = 3 * FAR_TI * P2 * sizeof(float4) + FAR_TI * P2 * sizeof(float2) +
                          P2 * FAR_THREADS * sizeof(float2) + fa.Q2 * 3 * sizeof(float);
            if (!helm)
                far_vkg_sym_x2_kernel<false, 2><<<grid, FAR_THREADS, smem, s>>>(fa, va);
            else if (fa.small_phase == 2)
                far_vkg_sym_x2_kernel<true, 2><<<grid, FAR_THREADS, smem, s>>>(fa, va);
            else if (fa.small_phase == 1)
                far_vkg_sym_x2_kernel<true, 1><<<grid, FAR_THREADS, smem, s>>>(fa, va);
            else
                far_vkg_sym_x2_kernel<true, 0><<<grid, FAR_THREADS, smem, s>>>(fa, va);
        } else {
            size_t smem = FAR_TI * fa.Q2 * (sizeof(double4) + 2 * sizeof(double)) + fa.Q2 * 3 * sizeof(double);
            if (helm)
                far_vkg_sym_kernel<true, double><<<grid, FAR_THREADS, smem, s>>>(fa, va);
            else
                far_vkg_sym_kernel<false, double><<<grid, FAR_THREADS, smem, s>>>(fa, va);
        }
        ctx->launches++;
        if (int rc = bem_check_cuda(ctx, cudaGetLastError(), "far_vkg_sym_kernel launch")) return rc;
    } else if (fa.n_test > 0 && fa.n_trial > 0) {
        if (fp32) {
            size_t smem = FAR_TI * fa.Q2 * sizeof(float4) + fa.Q2 * 3 * sizeof(float);
            if (helm)
                far_vkg_kernel<true, float><<<grid, FAR_THREADS, smem, s>>>(fa, va);
            else
                far_vkg_kernel<false, float><<<grid, FAR_THREADS, smem, s>>>(fa, va);
        } else {
            size_t smem = FAR_TI * fa.Q2 * sizeof(double4) + fa.Q2 * 3 * sizeof(double);
            if (helm)
                far_vkg_kernel<true, double><<<grid, FAR_THREADS, smem, s>>>(fa, va);
            else
                far_vkg_kernel<false, double><<<grid, FAR_THREADS, smem, s>>>(fa, va);
        }
        ctx->launches++;
        if (int rc = bem_check_cuda(ctx, cudaGetLastError(), "far_vkg_kernel launch")) return rc;
    }
    // near field: V dense and K g apply, FP64, with the operator's own kernels
    NearArgs na{};
    na.n_near = ctx->n_near;
    na.near = ctx->near;
    na.test_local = ctx->test_local;
    na.trial_local = ctx->trial_local;
    na.tris = ctx->tris;
    na.verts = ctx->verts;
    na.area = ctx->area;
    na.normal = ctx->normal;
    na.curl = ctx->curl;
    na.gp = ctx->gp;
    na.gw = ctx->gw;
    na.Q = ctx->Q;
    na.k = op->k;
    na.k2 = op->k2;
    na.quirk = op->quirk;
    if (na.n_near > 0) {
        const unsigned blocks = (unsigned)((na.n_near + 3) / 4);
        NearArgs nv = na;
        nv.test_dof = test->dof;
        nv.trial_dof = trial->dof;
        nv.mode = 0;
        nv.out = (double*)out;
        nv.ld = ld;
        nv.scale = scale;
        NearArgs nk = na;
        nk.test_dof = rows->dof;
        nk.trial_dof = data->dof;
        nk.mode = 1;
        nk.x = (const double*)g;
        nk.y = (double*)y;
        nk.scale = scale_k;
        nk.conj_x = conj_g;
        if (helm) {
            if (data->nb == 3)
                near_vkg_kernel<true, 3><<<blocks, 128, 0, sn>>>(nv, nk);
            else
                near_vkg_kernel<true, 1><<<blocks, 128, 0, sn>>>(nv, nk);
        } else {
            if (data->nb == 3)
                near_vkg_kernel<false, 3><<<blocks, 128, 0, sn>>>(nv, nk);
            else
                near_vkg_kernel<false, 1><<<blocks, 128, 0, sn>>>(nv, nk);
        }
        ctx->launches++;
        if (int rc = bem_check_cuda(ctx, cudaGetLastError(), "near_vkg_kernel launch")) return rc;
    }
    if (side) {
        cudaEventRecord(ctx->ev_diag, ctx->aux);
        cudaStreamWaitEvent(s, ctx->ev_diag, 0);
    }
    return bem_check_cuda(ctx, cudaGetLastError(), "near-field join");
}

int bem_launch_mass(bem_ctx* ctx, const bem_space* test, const bem_space* trial, int is_complex, int mode, void* out,
                    int64_t ld, double scale, void* out_t, double scale_t, const void* x, void* y, int conj_x,
                    cudaStream_t s) {
    MassArgs m;
    m.n_panels = test->n_panels;
    m.panels = test->panels;
    m.nbx = test->nb;
    m.nby = trial->nb;
    m.test_dof = test->dof;
    m.trial_dof = trial->dof;
    m.area = ctx->area;
    m.gp = ctx->gp;
    m.gw = ctx->gw;
    m.Q = ctx->Q;
    m.cplx = is_complex;
    m.mode = mode;
    m.out = (double*)out;
    m.ld = ld;
    m.scale = scale;
    m.out_t = (double*)out_t;
    m.scale_t = scale_t;
    m.x = (const double*)x;
    m.y = (double*)y;
    m.conj_x = conj_x;
    int total = m.n_panels * m.nbx * m.nby;
    if (total == 0) return BEM_OK;
    mass_kernel<<<(total + 127) / 128, 128, 0, s>>>(m);
    ctx->launches++;
    return bem_check_cuda(ctx, cudaGetLastError(), "mass_kernel launch");
}
