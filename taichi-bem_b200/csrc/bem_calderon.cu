// Fused Calderon-block assembly: the separate panel pairs of V, K, K^T and W
// for one or two wavenumbers in ONE sweep over unordered panel pairs, added
// straight into the block systems of the transmission problem.
//
// The reference assembles the transmission operator with one Taichi kernel
// per operator and scope (BEMManager.matrix_layer_forward, BEM_manager.py:829-844:
// SingleLayer3d.forward, DoubleLayer3d.forward, HypersingularLayer3d.forward
// at sqrt_no and again at sqrt_ni), each over ordered panel pairs, and then
// scatters the blocks into _mat_A (matA_add_M, BEM_manager.py:608-628).  Here,
// with P0 Neumann and P1 Dirichlet spaces over one panel list, one evaluation
// of the kernel at a point pair (x_a in panel i, y_b in panel j, i < j) serves
//   V_ij = V_ji                 sum w e^{ikr}/r
//   K_ij (trial hats of j)      sum w phi_b(y) ( d.n_j) F / r^3
//   K_ji (trial hats of i)      sum w phi_a(x) (-d.n_i) F / r^3
//   W_ij = W_ji^T               G curl_a.curl_b - k2 (n_i.n_j) sum w phi_a phi_b e^{ikr}/r
// with d = x_a - y_b, F = (1 - ikr) e^{ikr}, and the entries go into each
// output X_w with the reference's block placement for matA_add_M(c_w):
//   X_NN += -c V,  X_ND += c K,  X_DN += -c K^T,  X_DD += -c W.
// The hats are carried as (total, phi_1, phi_2) moments and phi_0 = 1 - phi_1
// - phi_2 is formed in FP64, so a constant is reproduced exactly.
//
// FP32 (mixed precision) evaluates in the pair frame of the other far-field
// kernels (bem_farfield.cuh): r^2 = R^2 + s, e^{ikr} = e^{ikR} e^{ik(r - R)}
// with e^{ikR} per pair and wavenumber in FP64, reference-triangle weights
// rescaled in FP64; the sums over the test points run in FP32, the sums over
// the trial points in FP64.  FP64 (plain path) evaluates d = x - y directly.
// Coincident / edge / vertex pairs are left to the FP64 Sauter-Schwab
// kernels (bem_launch_assemble_parts, near only), which run on the side
// stream while the sweep runs.
#include <cmath>

#include "bem_farfield.cuh"

namespace {

constexpr int CAL_MAXK = 2;

struct CalArgs {
    int n;                  // panels on every side (one list)
    const int32_t* panels;  // [n] global panel index
    const int32_t* ndof;    // [n] Neumann (P0) dof of each panel, <0 = skipped
    const int32_t* ddof;    // [n*3] Dirichlet (P1) dof of each panel vertex, <0 = skipped
    const int32_t* tris;
    const double* centroid;
    const double* normal;
    const double* curl;
    const double* area;
    double wcorr;
    int small_phase;
    const void* pts;
    const void* phi;      // [Q2*3] P1 hats at the separate-rule points (FP32 or FP64)
    const double* phi64;  // [Q2*3] FP64
    int Q2;
    double k[CAL_MAXK], k2[CAL_MAXK], coef[CAL_MAXK];
    double* out[CAL_MAXK];
    int64_t ld;
};

// (tot, phi_1, phi_2) moments -> values of the three hats
__device__ __forceinline__ void hats(const double* m, double* v) {
    v[0] = m[0] - m[1] - m[2];
    v[1] = m[1];
    v[2] = m[2];
}

// Entries of one unordered separate pair (i = li, j = lj) for wavenumber w
// from its FP64 moments Mr / Mi (layout of far_calderon_kernel), added to
// out[w] with the reference's block placement.  rotate: multiply by the pair
// frame's e^{ikR} (FP32 pair frame).
template <bool HELM>
__device__ __forceinline__ void calderon_epilogue(const CalArgs& a, int w, int li, int lj, int gi, int gj,
                                                  const double* ni64, const double* nj64, double pf, double Rd,
                                                  const double* Mr, const double* Mi, bool rotate) {
    const int nri = a.ndof[li], nrj = a.ndof[lj];
    int di[3], dj[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        di[c] = a.ddof[3 * li + c];
        dj[c] = a.ddof[3 * lj + c];
    }
    const double nd = ni64[0] * nj64[0] + ni64[1] * nj64[1] + ni64[2] * nj64[2];
    // pair factor and e^{ikR}, then 1/(4 pi)
    double fr_ = pf * BEM_INV4PI, fi_ = 0.0;
    if (rotate) {
        double sR, cR;
        sincos(a.k[w] * Rd, &sR, &cR);
        fi_ = fr_ * sR;
        fr_ = fr_ * cR;
    }
    double vr[15], vi[15];
#pragma unroll
    for (int m = 0; m < 15; ++m) {
        vr[m] = Mr[m] * fr_ - Mi[m] * fi_;
        vi[m] = Mr[m] * fi_ + Mi[m] * fr_;
    }
    double* X = a.out[w];
    const double c = a.coef[w];
    const int64_t ld = a.ld;
    // V (P0 x P0): one writer per entry
    if (nri >= 0 && nrj >= 0) {
        add_entry<HELM>(X, (int64_t)nri * ld + nrj, -c * vr[0], -c * vi[0], false);
        add_entry<HELM>(X, (int64_t)nrj * ld + nri, -c * vr[0], -c * vi[0], false);
    }
    // K_ij (row N_i, trial hats of j) and K_ji (row N_j, trial hats of i), with their -K^T
    double kyr[3], kyi[3], kxr[3], kxi[3];
    hats(vr + 1, kyr);
    hats(vi + 1, kyi);
    hats(vr + 4, kxr);
    hats(vi + 4, kxi);
#pragma unroll
    for (int h = 0; h < 3; ++h) {
        if (nri >= 0 && dj[h] >= 0) {
            add_entry<HELM>(X, (int64_t)nri * ld + dj[h], c * kyr[h], c * kyi[h], true);
            add_entry<HELM>(X, (int64_t)dj[h] * ld + nri, -c * kyr[h], -c * kyi[h], true);
        }
        if (nrj >= 0 && di[h] >= 0) {
            add_entry<HELM>(X, (int64_t)nrj * ld + di[h], c * kxr[h], c * kxi[h], true);
            add_entry<HELM>(X, (int64_t)di[h] * ld + nrj, -c * kxr[h], -c * kxi[h], true);
        }
    }
    // W (P1 x P1) and its transpose
    double pr[3][3], pim[3][3];
    if (HELM) {
        // moments (x-side in {tot,1,2}) x (y-side in {tot,1,2}) -> hat values
        const double tr[3][3] = {{vr[0], vr[7], vr[8]}, {vr[9], vr[10], vr[11]}, {vr[12], vr[13], vr[14]}};
        const double ti[3][3] = {{vi[0], vi[7], vi[8]}, {vi[9], vi[10], vi[11]}, {vi[12], vi[13], vi[14]}};
        double rr[3][3], ri[3][3];
#pragma unroll
        for (int x = 0; x < 3; ++x) {
            hats(tr[x], rr[x]);
            hats(ti[x], ri[x]);
        }
#pragma unroll
        for (int y = 0; y < 3; ++y) {
            const double cr[3] = {rr[0][y], rr[1][y], rr[2][y]}, ci[3] = {ri[0][y], ri[1][y], ri[2][y]};
            double hr[3], hi[3];
            hats(cr, hr);
            hats(ci, hi);
#pragma unroll
            for (int x = 0; x < 3; ++x) {
                pr[x][y] = hr[x];
                pim[x][y] = hi[x];
            }
        }
    }
#pragma unroll
    for (int x = 0; x < 3; ++x) {
        if (di[x] < 0) continue;
        const double* cx = a.curl + 9 * gi + 3 * x;
#pragma unroll
        for (int y = 0; y < 3; ++y) {
            if (dj[y] < 0) continue;
            const double* cy = a.curl + 9 * gj + 3 * y;
            const double cc = cx[0] * cy[0] + cx[1] * cy[1] + cx[2] * cy[2];  // curl_x(i) . curl_y(j)
            double wr_ = vr[0] * cc, wi_ = vi[0] * cc;
            if (HELM) {
                wr_ -= a.k2[w] * nd * pr[x][y];
                wi_ -= a.k2[w] * nd * pim[x][y];
            }
            add_entry<HELM>(X, (int64_t)di[x] * ld + dj[y], -c * wr_, -c * wi_, true);
            add_entry<HELM>(X, (int64_t)dj[y] * ld + di[x], -c * wr_, -c * wi_, true);
        }
    }
}

template <typename T, int NK, bool HELM, int PH>
__global__ void __launch_bounds__(FAR_THREADS) far_calderon_kernel(CalArgs a) {
    using V4 = typename V4T<T>::type;
    constexpr bool SPLIT = sizeof(T) == 4;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V4* sx = reinterpret_cast<V4*>(smem_raw);          // [FAR_TI][Q2] test points
    T* sp = reinterpret_cast<T*>(sx + FAR_TI * a.Q2);  // [Q2][2] phi_1, phi_2 at the points
    __shared__ int s_gi[FAR_TI];
    __shared__ int s_tri[FAR_TI][3];
    __shared__ double s_cen[FAR_TI][3];
    __shared__ double s_nrm[FAR_TI][3];

    const int Q2 = a.Q2;
    const int n = a.n;
    const int j0 = blockIdx.x * FAR_THREADS;
    const int li0 = blockIdx.y * FAR_TI;
    if (j0 + FAR_THREADS - 1 <= li0) return;  // tile strictly below the diagonal
    const int lj = j0 + threadIdx.x;
    const V4* pts = reinterpret_cast<const V4*>(a.pts);
    {
        const T* phi = reinterpret_cast<const T*>(a.phi);
        for (int q = threadIdx.x; q < Q2; q += FAR_THREADS) {
            sp[2 * q] = phi[3 * q + 1];
            sp[2 * q + 1] = phi[3 * q + 2];
        }
    }
    if (threadIdx.x < FAR_TI) {
        const int li = li0 + threadIdx.x;
        const int gi = li < n ? a.panels[li] : -1;
        s_gi[threadIdx.x] = gi;
        for (int c = 0; c < 3; ++c) {
            s_tri[threadIdx.x][c] = gi >= 0 ? a.tris[3 * gi + c] : -1;
            s_cen[threadIdx.x][c] = gi >= 0 ? a.centroid[3 * gi + c] : 0.0;
            s_nrm[threadIdx.x][c] = gi >= 0 ? a.normal[3 * gi + c] : 0.0;
        }
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < FAR_TI * Q2; idx += FAR_THREADS) {
        const int t = idx / Q2, q = idx - t * Q2;
        if (li0 + t < n) sx[idx] = pts[(size_t)s_gi[t] * Q2 + q];
    }
    __syncthreads();

    const bool valid_j = lj < n;
    const int gj = valid_j ? a.panels[lj] : 0;
    int tri_j[3];
    double cen_j[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        tri_j[c] = a.tris[3 * gj + c];
        cen_j[c] = a.centroid[3 * gj + c];
    }
    const double nj64[3] = {a.normal[3 * gj + 0], a.normal[3 * gj + 1], a.normal[3 * gj + 2]};
    const V4* ptsj = pts + (size_t)gj * Q2;
    T kk[NK];
#pragma unroll
    for (int w = 0; w < NK; ++w) kk[w] = T(a.k[w]);

    for (int t = 0; t < FAR_TI; ++t) {
        const int li = li0 + t;
        if (li >= n) break;  // uniform across the CTA
        const int gi = s_gi[t];
        const bool sep = valid_j && li < lj && (bem_relation(s_tri[t], tri_j, gi == gj) == REL_SEPARATE);
        if (!sep) continue;
        const double Dx = s_cen[t][0] - cen_j[0], Dy = s_cen[t][1] - cen_j[1], Dz = s_cen[t][2] - cen_j[2];
        const double ni64[3] = {s_nrm[t][0], s_nrm[t][1], s_nrm[t][2]};
        // pair frame (FP32): 2D, R^2, R and the pair factor; FP64 evaluates d directly
        const T dcx = T(Dx), dcy = T(Dy), dcz = T(Dz);
        const T dlx = T(Dx - double(dcx)), dly = T(Dy - double(dcy)), dlz = T(Dz - double(dcz));
        const T ux = T(2.0 * Dx), uy = T(2.0 * Dy), uz = T(2.0 * Dz);
        const double R2d = Dx * Dx + Dy * Dy + Dz * Dz;
        const T R2 = T(R2d);
        const double Rd = sqrt(R2d);
        const T Rf = T(Rd);
        const double pf = SPLIT ? 4.0 * a.area[gi] * a.area[gj] * a.wcorr : 1.0;
        const T Dnj = T(Dx * nj64[0] + Dy * nj64[1] + Dz * nj64[2]);
        const double Dni64 = Dx * ni64[0] + Dy * ni64[1] + Dz * ni64[2];
        // n_j - n_i: x_a.n_j = x_a.(n_j - n_i) (x_a lies in the plane of panel i)
        const T mx = T(nj64[0] - ni64[0]), my = T(nj64[1] - ni64[1]), mz = T(nj64[2] - ni64[2]);
        const T njx = T(nj64[0]), njy = T(nj64[1]), njz = T(nj64[2]);
        const V4* sxt = sx + t * Q2;

        // FP64 moments over the trial points, per wavenumber:
        // [0] V / W curl (sum w G), [1..3] K_ij (tot, phi1, phi2 of y), [4..6] K_ji (tot, phi1, phi2 of x),
        // [7..14] W mass phi(x) phi(y) (a,b) in {tot,1,2}^2 without (tot, tot)
        double Mr[NK][15], Mi[NK][15];
#pragma unroll
        for (int w = 0; w < NK; ++w)
#pragma unroll
            for (int m = 0; m < 15; ++m) Mr[w][m] = Mi[w][m] = 0.0;

        for (int b = 0; b < Q2; ++b) {
            const V4 yb = ptsj[b];
            const T ex = (dcx - yb.x) + dlx, ey = (dcy - yb.y) + dly, ez = (dcz - yb.z) + dlz;
            const T wx = ux - yb.x, wy = uy - yb.y, wz = uz - yb.z;
            // FP32 sums over the test points: [0] G, [1] phi1 G, [2] phi2 G, [3] d.n_j F/r^3,
            // [4] F/r^3, [5] phi1 F/r^3, [6] phi2 F/r^3 (times w_a)
            T sr[NK][7], si[NK][7];
#pragma unroll
            for (int w = 0; w < NK; ++w)
#pragma unroll
                for (int m = 0; m < 7; ++m) sr[w][m] = si[w][m] = T(0);
#pragma unroll 5
            for (int q = 0; q < Q2; ++q) {
                const V4 xa = sxt[q];
                const T p1 = sp[2 * q], p2 = sp[2 * q + 1];
                T r, rinv, dnj, ph;
                if constexpr (SPLIT) {
                    const T e_x = xa.x - yb.x, e_y = xa.y - yb.y, e_z = xa.z - yb.z;
                    const T sq = e_x * (xa.x + wx) + e_y * (xa.y + wy) + e_z * (xa.z + wz);
                    dev_r_rinv(R2 + sq, r, rinv);
                    dnj = fma(xa.x, mx, fma(xa.y, my, fma(xa.z, mz, Dnj)));
                    ph = HELM ? __fdividef(sq, r + Rf) : T(0);
                } else {
                    const T dx = xa.x + ex, dy = xa.y + ey, dz = xa.z + ez;
                    dev_r_rinv(dx * dx + dy * dy + dz * dz, r, rinv);
                    dnj = dx * njx + dy * njy + dz * njz;
                    ph = r;
                }
                const T wr = xa.w * rinv;
                const T wr3 = wr * (rinv * rinv);
                const T tj = wr3 * dnj;
#pragma unroll
                for (int w = 0; w < NK; ++w) {
                    T gr, gi_, fr, fi;
                    if (HELM) {
                        T sn, cs;
                        if constexpr (SPLIT)
                            dev_sincos_phase(kk[w] * ph, PH != 0, &sn, &cs);
                        else
                            dev_sincos(kk[w] * ph, &sn, &cs);
                        const T kr = kk[w] * r;
                        gr = wr * cs;
                        gi_ = wr * sn;
                        fr = fma(kr, sn, cs);
                        fi = fma(-kr, cs, sn);
                    } else {
                        gr = wr;
                        gi_ = T(0);
                        fr = T(1);
                        fi = T(0);
                    }
                    sr[w][0] += gr;
                    sr[w][1] = fma(p1, gr, sr[w][1]);
                    sr[w][2] = fma(p2, gr, sr[w][2]);
                    sr[w][3] = fma(tj, fr, sr[w][3]);
                    const T hr = wr3 * fr;
                    sr[w][4] += hr;
                    sr[w][5] = fma(p1, hr, sr[w][5]);
                    sr[w][6] = fma(p2, hr, sr[w][6]);
                    if (HELM) {
                        si[w][0] += gi_;
                        si[w][1] = fma(p1, gi_, si[w][1]);
                        si[w][2] = fma(p2, gi_, si[w][2]);
                        si[w][3] = fma(tj, fi, si[w][3]);
                        const T hi = wr3 * fi;
                        si[w][4] += hi;
                        si[w][5] = fma(p1, hi, si[w][5]);
                        si[w][6] = fma(p2, hi, si[w][6]);
                    }
                }
            }
            const double wb = double(yb.w);
            const double wb1 = wb * a.phi64[3 * b + 1], wb2 = wb * a.phi64[3 * b + 2];
            // -d.n_i = -(D.n_i - y_b.n_i), constant over the test points
            const double ndni =
                -(Dni64 - (double(yb.x) * ni64[0] + double(yb.y) * ni64[1] + double(yb.z) * ni64[2]));
            const double wbn = wb * ndni;
#pragma unroll
            for (int w = 0; w < NK; ++w) {
                const double g0r = sr[w][0], g0i = si[w][0], g1r = sr[w][1], g1i = si[w][1];
                const double g2r = sr[w][2], g2i = si[w][2];
                Mr[w][0] += wb * g0r;
                Mr[w][1] += wb * double(sr[w][3]);
                Mr[w][2] += wb1 * double(sr[w][3]);
                Mr[w][3] += wb2 * double(sr[w][3]);
                Mr[w][4] += wbn * double(sr[w][4]);
                Mr[w][5] += wbn * double(sr[w][5]);
                Mr[w][6] += wbn * double(sr[w][6]);
                if (HELM) {
                    Mi[w][0] += wb * g0i;
                    Mi[w][1] += wb * double(si[w][3]);
                    Mi[w][2] += wb1 * double(si[w][3]);
                    Mi[w][3] += wb2 * double(si[w][3]);
                    Mi[w][4] += wbn * double(si[w][4]);
                    Mi[w][5] += wbn * double(si[w][5]);
                    Mi[w][6] += wbn * double(si[w][6]);
                    // W mass moments (tot,1), (tot,2), (1,tot), (1,1), (1,2), (2,tot), (2,1), (2,2)
                    Mr[w][7] += wb1 * g0r;
                    Mi[w][7] += wb1 * g0i;
                    Mr[w][8] += wb2 * g0r;
                    Mi[w][8] += wb2 * g0i;
                    Mr[w][9] += wb * g1r;
                    Mi[w][9] += wb * g1i;
                    Mr[w][10] += wb1 * g1r;
                    Mi[w][10] += wb1 * g1i;
                    Mr[w][11] += wb2 * g1r;
                    Mi[w][11] += wb2 * g1i;
                    Mr[w][12] += wb * g2r;
                    Mi[w][12] += wb * g2i;
                    Mr[w][13] += wb1 * g2r;
                    Mi[w][13] += wb1 * g2i;
                    Mr[w][14] += wb2 * g2r;
                    Mi[w][14] += wb2 * g2i;
                }
            }
        }

        // ---- epilogue: entries of every block, per wavenumber ----
#pragma unroll
        for (int w = 0; w < NK; ++w)
            calderon_epilogue<HELM>(a, w, li, lj, gi, gj, ni64, nj64, pf, Rd, Mr[w], Mi[w], SPLIT && HELM);
    }
}

// ---------------------------------------------------------------------------
// Packed FP32x2 form of the Helmholtz sweep (mixed precision, one
// wavenumber per launch): two test points (q, q + 1) in the two lanes of every
// FFMA2 / FMUL2 / FADD2, as in the packed Dirichlet sweep, with the same
// pair-frame algebra as far_calderon_kernel<float, 1, true, PH>:
//   s = |x_a|^2 + x_a.U_b + C_b,  U_b = 2D - 2y_b,  C_b = -y_b.(2D - y_b)
//   d.n_j = D.n_j + x_a.(n_j - n_i).
// The lanes are summed after the loop over the test points; an odd Q^2 is
// padded by a copy of the last point with weight 0.  PH: 2 short polynomial
// (phase <= 0.3), 1 full polynomial (<= pi/4), 0 argument reduction.
// ---------------------------------------------------------------------------
template <int PH>
__global__ void __launch_bounds__(FAR_THREADS) far_calderon_x2_kernel(CalArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int Q2 = a.Q2;
    const int P2 = (Q2 + 1) / 2;
    float4* sxy = reinterpret_cast<float4*>(smem_raw);          // [FAR_TI][P2] (x0 x1 y0 y1)
    float4* szw = sxy + FAR_TI * P2;                             // [FAR_TI][P2] (z0 z1 w0 w1)
    float2* sxx = reinterpret_cast<float2*>(szw + FAR_TI * P2);  // [FAR_TI][P2] |x|^2
    float4* sph = reinterpret_cast<float4*>(sxx + FAR_TI * P2);  // [P2] (phi1_0 phi1_1 phi2_0 phi2_1)
    __shared__ int s_gi[FAR_TI];
    __shared__ int s_tri[FAR_TI][3];
    __shared__ double s_cen[FAR_TI][3];
    __shared__ double s_nrm[FAR_TI][3];

    const int n = a.n;
    const int j0 = blockIdx.x * FAR_THREADS;
    const int li0 = blockIdx.y * FAR_TI;
    if (j0 + FAR_THREADS - 1 <= li0) return;
    const int lj = j0 + threadIdx.x;
    const float4* pts = reinterpret_cast<const float4*>(a.pts);
    const float* phi = reinterpret_cast<const float*>(a.phi);
    if (threadIdx.x < FAR_TI) {
        const int li = li0 + threadIdx.x;
        const int gi = li < n ? a.panels[li] : -1;
        s_gi[threadIdx.x] = gi;
        for (int c = 0; c < 3; ++c) {
            s_tri[threadIdx.x][c] = gi >= 0 ? a.tris[3 * gi + c] : -1;
            s_cen[threadIdx.x][c] = gi >= 0 ? a.centroid[3 * gi + c] : 0.0;
            s_nrm[threadIdx.x][c] = gi >= 0 ? a.normal[3 * gi + c] : 0.0;
        }
    }
    for (int p = threadIdx.x; p < P2; p += FAR_THREADS) {
        const int q0 = 2 * p, q1 = 2 * p + 1 < Q2 ? 2 * p + 1 : Q2 - 1;
        const float pad = 2 * p + 1 < Q2 ? 1.f : 0.f;
        sph[p] = make_float4(phi[3 * q0 + 1], pad * phi[3 * q1 + 1], phi[3 * q0 + 2], pad * phi[3 * q1 + 2]);
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < FAR_TI * P2; idx += FAR_THREADS) {
        const int t = idx / P2, p = idx - t * P2;
        const int q0 = 2 * p, q1 = 2 * p + 1 < Q2 ? 2 * p + 1 : Q2 - 1;
        float4 x0 = make_float4(0.f, 0.f, 0.f, 0.f), x1 = x0;
        if (li0 + t < n) {
            x0 = pts[(size_t)s_gi[t] * Q2 + q0];
            x1 = pts[(size_t)s_gi[t] * Q2 + q1];
            if (2 * p + 1 >= Q2) x1.w = 0.f;  // padding point: weight 0
        }
        sxy[idx] = make_float4(x0.x, x1.x, x0.y, x1.y);
        szw[idx] = make_float4(x0.z, x1.z, x0.w, x1.w);
        sxx[idx] = make_float2(fmaf(x0.x, x0.x, fmaf(x0.y, x0.y, x0.z * x0.z)),
                               fmaf(x1.x, x1.x, fmaf(x1.y, x1.y, x1.z * x1.z)));
    }
    __syncthreads();

    const bool valid_j = lj < n;
    const int gj = valid_j ? a.panels[lj] : 0;
    int tri_j[3];
    double cen_j[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        tri_j[c] = a.tris[3 * gj + c];
        cen_j[c] = a.centroid[3 * gj + c];
    }
    const double nj64[3] = {a.normal[3 * gj + 0], a.normal[3 * gj + 1], a.normal[3 * gj + 2]};
    const float4* ptsj = pts + (size_t)gj * Q2;
    const float2 KK = f2((float)a.k[0]), NKK = f2(-(float)a.k[0]);

    for (int t = 0; t < FAR_TI; ++t) {
        const int li = li0 + t;
        if (li >= n) break;
        const int gi = s_gi[t];
        const bool sep = valid_j && li < lj && (bem_relation(s_tri[t], tri_j, gi == gj) == REL_SEPARATE);
        if (!sep) continue;
        const double Dx = s_cen[t][0] - cen_j[0], Dy = s_cen[t][1] - cen_j[1], Dz = s_cen[t][2] - cen_j[2];
        const double ni64[3] = {s_nrm[t][0], s_nrm[t][1], s_nrm[t][2]};
        const float ux = (float)(2.0 * Dx), uy = (float)(2.0 * Dy), uz = (float)(2.0 * Dz);
        const double R2d = Dx * Dx + Dy * Dy + Dz * Dz;
        const double Rd = sqrt(R2d);
        const float2 R2 = f2((float)R2d), RF = f2((float)Rd);
        const double pf = 4.0 * a.area[gi] * a.area[gj] * a.wcorr;
        const double Dni64 = Dx * ni64[0] + Dy * ni64[1] + Dz * ni64[2];
        const float2 DNJ = f2((float)(Dx * nj64[0] + Dy * nj64[1] + Dz * nj64[2]));
        const float2 MX = f2((float)(nj64[0] - ni64[0])), MY = f2((float)(nj64[1] - ni64[1])),
                     MZ = f2((float)(nj64[2] - ni64[2]));
        const float4* sxyt = sxy + t * P2;
        const float4* szwt = szw + t * P2;
        const float2* sxxt = sxx + t * P2;

        double Mr[15], Mi[15];
#pragma unroll
        for (int m = 0; m < 15; ++m) Mr[m] = Mi[m] = 0.0;

        for (int b = 0; b < Q2; ++b) {
            const float4 yb = ptsj[b];
            const float wx = ux - yb.x, wy = uy - yb.y, wz = uz - yb.z;
            const float2 U0 = f2(wx - yb.x), U1 = f2(wy - yb.y), U2 = f2(wz - yb.z);
            const float2 CB = f2(-fmaf(yb.x, wx, fmaf(yb.y, wy, yb.z * wz)));
            // [0] G, [1] phi1 G, [2] phi2 G, [3] d.n_j F/r^3, [4] F/r^3, [5] phi1 F/r^3, [6] phi2 F/r^3
            float2 Ar[7], Ai[7];
#pragma unroll
            for (int m = 0; m < 7; ++m) Ar[m] = Ai[m] = f2(0.f);
#pragma unroll 2
            for (int p = 0; p < P2; ++p) {
                const float4 xy = sxyt[p], zw = szwt[p], ph = sph[p];
                const float2 X = make_float2(xy.x, xy.y), Y = make_float2(xy.z, xy.w);
                const float2 Z = make_float2(zw.x, zw.y), Wt = make_float2(zw.z, zw.w);
                const float2 P1 = make_float2(ph.x, ph.y), P2v = make_float2(ph.z, ph.w);
                const float2 sq = ffma2(X, U0, ffma2(Y, U1, ffma2(Z, U2, fadd2(sxxt[p], CB))));
                float2 r, rinv;
                dev_r_rinv2(fadd2(R2, sq), r, rinv);
                const float2 dnj = ffma2(X, MX, ffma2(Y, MY, ffma2(Z, MZ, DNJ)));
                const float2 rr = fadd2(r, RF);
                const float2 phase = fmul2(KK, fmul2(sq, make_float2(__fdividef(1.0f, rr.x), __fdividef(1.0f, rr.y))));
                const float2 wr = fmul2(Wt, rinv);
                const float2 wr3 = fmul2(wr, fmul2(rinv, rinv));
                const float2 tj = fmul2(wr3, dnj);
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
                const float2 gr = fmul2(wr, cs), gi_ = fmul2(wr, sn);
                const float2 fr = ffma2(kr, sn, cs), fi = ffma2(nkr, cs, sn);
                Ar[0] = fadd2(Ar[0], gr);
                Ai[0] = fadd2(Ai[0], gi_);
                Ar[1] = ffma2(P1, gr, Ar[1]);
                Ai[1] = ffma2(P1, gi_, Ai[1]);
                Ar[2] = ffma2(P2v, gr, Ar[2]);
                Ai[2] = ffma2(P2v, gi_, Ai[2]);
                Ar[3] = ffma2(tj, fr, Ar[3]);
                Ai[3] = ffma2(tj, fi, Ai[3]);
                const float2 hr = fmul2(wr3, fr), hi = fmul2(wr3, fi);
                Ar[4] = fadd2(Ar[4], hr);
                Ai[4] = fadd2(Ai[4], hi);
                Ar[5] = ffma2(P1, hr, Ar[5]);
                Ai[5] = ffma2(P1, hi, Ai[5]);
                Ar[6] = ffma2(P2v, hr, Ar[6]);
                Ai[6] = ffma2(P2v, hi, Ai[6]);
            }
            float sr[7], si[7];
#pragma unroll
            for (int m = 0; m < 7; ++m) {
                sr[m] = Ar[m].x + Ar[m].y;
                si[m] = Ai[m].x + Ai[m].y;
            }
            const double wb = double(yb.w);
            const double wb1 = wb * a.phi64[3 * b + 1], wb2 = wb * a.phi64[3 * b + 2];
            const double ndni =
                -(Dni64 - (double(yb.x) * ni64[0] + double(yb.y) * ni64[1] + double(yb.z) * ni64[2]));
            const double wbn = wb * ndni;
            const double g0r = sr[0], g0i = si[0], g1r = sr[1], g1i = si[1], g2r = sr[2], g2i = si[2];
            Mr[0] += wb * g0r;
            Mi[0] += wb * g0i;
            Mr[1] += wb * double(sr[3]);
            Mi[1] += wb * double(si[3]);
            Mr[2] += wb1 * double(sr[3]);
            Mi[2] += wb1 * double(si[3]);
            Mr[3] += wb2 * double(sr[3]);
            Mi[3] += wb2 * double(si[3]);
            Mr[4] += wbn * double(sr[4]);
            Mi[4] += wbn * double(si[4]);
            Mr[5] += wbn * double(sr[5]);
            Mi[5] += wbn * double(si[5]);
            Mr[6] += wbn * double(sr[6]);
            Mi[6] += wbn * double(si[6]);
            Mr[7] += wb1 * g0r;
            Mi[7] += wb1 * g0i;
            Mr[8] += wb2 * g0r;
            Mi[8] += wb2 * g0i;
            Mr[9] += wb * g1r;
            Mi[9] += wb * g1i;
            Mr[10] += wb1 * g1r;
            Mi[10] += wb1 * g1i;
            Mr[11] += wb2 * g1r;
            Mi[11] += wb2 * g1i;
            Mr[12] += wb * g2r;
            Mi[12] += wb * g2i;
            Mr[13] += wb1 * g2r;
            Mi[13] += wb1 * g2i;
            Mr[14] += wb2 * g2r;
            Mi[14] += wb2 * g2i;
        }
        calderon_epilogue<true>(a, 0, li, lj, gi, gj, ni64, nj64, pf, Rd, Mr, Mi, true);
    }
}

// Both wavenumbers of the FP32 Helmholtz sweep packed into the two lanes of
// FP32x2 instructions (x: k[0], y: k[1]): the pair-frame geometry of a point
// pair (r, 1/r, the split phase, w/r, w/r^3, d.n_j) is formed once in scalar
// FP32, and the per-wavenumber part -- the phase k (r - R), its sine and
// cosine, (1 - ikr) e^{ikr} and the 14 sums over the test points -- runs on
// FFMA2 / FMUL2 / FADD2, one instruction for both wavenumbers.  Same
// algebra, summation order and FP64 moments as
// far_calderon_kernel<float, 2, true, PH>; the test points' phi_1, phi_2 are
// staged as broadcast pairs.  PH 2 / 1: the short / full sine and cosine
// polynomials without argument reduction; PH 0: the reduced scalar form per
// lane.
template <int PH, bool SM>
__global__ void __launch_bounds__(FAR_THREADS, SM ? 3 : 1) far_calderon_k2_kernel(CalArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float4* sx = reinterpret_cast<float4*>(smem_raw);     // [FAR_TI][Q2] test points
    float4* sp = reinterpret_cast<float4*>(sx + FAR_TI * a.Q2);  // [Q2] (phi_1, phi_1, phi_2, phi_2)
    // SM: the FP64 moments over the trial points live in shared memory,
    // [moment][thread] with moment (w * 15 + m) * 2 + (0 re, 1 im), so that
    // three CTAs fit an SM; otherwise in registers
    double* mom = reinterpret_cast<double*>(sp + a.Q2) + threadIdx.x;
    __shared__ int s_gi[FAR_TI];
    __shared__ int s_tri[FAR_TI][3];
    __shared__ double s_cen[FAR_TI][3];
    __shared__ double s_nrm[FAR_TI][3];

    const int Q2 = a.Q2;
    const int n = a.n;
    const int j0 = blockIdx.x * FAR_THREADS;
    const int li0 = blockIdx.y * FAR_TI;
    if (j0 + FAR_THREADS - 1 <= li0) return;  // tile strictly below the diagonal
    const int lj = j0 + threadIdx.x;
    const float4* pts = reinterpret_cast<const float4*>(a.pts);
    {
        const float* phi = reinterpret_cast<const float*>(a.phi);
        for (int q = threadIdx.x; q < Q2; q += FAR_THREADS) {
            const float p1 = phi[3 * q + 1], p2 = phi[3 * q + 2];
            sp[q] = make_float4(p1, p1, p2, p2);
        }
    }
    if (threadIdx.x < FAR_TI) {
        const int li = li0 + threadIdx.x;
        const int gi = li < n ? a.panels[li] : -1;
        s_gi[threadIdx.x] = gi;
        for (int c = 0; c < 3; ++c) {
            s_tri[threadIdx.x][c] = gi >= 0 ? a.tris[3 * gi + c] : -1;
            s_cen[threadIdx.x][c] = gi >= 0 ? a.centroid[3 * gi + c] : 0.0;
            s_nrm[threadIdx.x][c] = gi >= 0 ? a.normal[3 * gi + c] : 0.0;
        }
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < FAR_TI * Q2; idx += FAR_THREADS) {
        const int t = idx / Q2, q = idx - t * Q2;
        if (li0 + t < n) sx[idx] = pts[(size_t)s_gi[t] * Q2 + q];
    }
    __syncthreads();

    const bool valid_j = lj < n;
    const int gj = valid_j ? a.panels[lj] : 0;
    int tri_j[3];
    double cen_j[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        tri_j[c] = a.tris[3 * gj + c];
        cen_j[c] = a.centroid[3 * gj + c];
    }
    const double nj64[3] = {a.normal[3 * gj + 0], a.normal[3 * gj + 1], a.normal[3 * gj + 2]};
    const float4* ptsj = pts + (size_t)gj * Q2;
    const float2 kk = make_float2(float(a.k[0]), float(a.k[1]));
    const float2 nkk = make_float2(-float(a.k[0]), -float(a.k[1]));

    for (int t = 0; t < FAR_TI; ++t) {
        const int li = li0 + t;
        if (li >= n) break;  // uniform across the CTA
        const int gi = s_gi[t];
        const bool sep = valid_j && li < lj && (bem_relation(s_tri[t], tri_j, gi == gj) == REL_SEPARATE);
        if (!sep) continue;
        const double Dx = s_cen[t][0] - cen_j[0], Dy = s_cen[t][1] - cen_j[1], Dz = s_cen[t][2] - cen_j[2];
        const double ni64[3] = {s_nrm[t][0], s_nrm[t][1], s_nrm[t][2]};
        const float ux = float(2.0 * Dx), uy = float(2.0 * Dy), uz = float(2.0 * Dz);
        const double R2d = Dx * Dx + Dy * Dy + Dz * Dz;
        const float R2 = float(R2d);
        const double Rd = sqrt(R2d);
        const float Rf = float(Rd);
        const double pf = 4.0 * a.area[gi] * a.area[gj] * a.wcorr;
        const float Dnj = float(Dx * nj64[0] + Dy * nj64[1] + Dz * nj64[2]);
        const double Dni64 = Dx * ni64[0] + Dy * ni64[1] + Dz * ni64[2];
        const float mx = float(nj64[0] - ni64[0]), my = float(nj64[1] - ni64[1]), mz = float(nj64[2] - ni64[2]);
        const float4* sxt = sx + t * Q2;

        double Mr[2][15], Mi[2][15];
        if constexpr (SM) {
#pragma unroll
            for (int m = 0; m < 60; ++m) mom[m * FAR_THREADS] = 0.0;
        } else {
#pragma unroll
            for (int w = 0; w < 2; ++w)
#pragma unroll
                for (int m = 0; m < 15; ++m) Mr[w][m] = Mi[w][m] = 0.0;
        }
        auto acc = [&](int w, int m, double re, double im) {
            if constexpr (SM) {
                double* q = mom + ((w * 15 + m) * 2) * FAR_THREADS;
                q[0] += re;
                q[FAR_THREADS] += im;
            } else {
                Mr[w][m] += re;
                Mi[w][m] += im;
            }
        };

        for (int b = 0; b < Q2; ++b) {
            const float4 yb = ptsj[b];
            const float wx = ux - yb.x, wy = uy - yb.y, wz = uz - yb.z;
            // packed sums over the test points (lanes: the two wavenumbers), as in
            // far_calderon_kernel: [0] G, [1] phi1 G, [2] phi2 G, [3] d.n_j F/r^3,
            // [4] F/r^3, [5] phi1 F/r^3, [6] phi2 F/r^3
            float2 sr[7], si[7];
#pragma unroll
            for (int m = 0; m < 7; ++m) sr[m] = si[m] = make_float2(0.0f, 0.0f);
#pragma unroll 5
            for (int q = 0; q < Q2; ++q) {
                const float4 xa = sxt[q];
                const float4 pp = sp[q];
                const float2 p1 = make_float2(pp.x, pp.y), p2 = make_float2(pp.z, pp.w);
                float r, rinv;
                const float e_x = xa.x - yb.x, e_y = xa.y - yb.y, e_z = xa.z - yb.z;
                const float sq = e_x * (xa.x + wx) + e_y * (xa.y + wy) + e_z * (xa.z + wz);
                dev_r_rinv(R2 + sq, r, rinv);
                const float dnj = fmaf(xa.x, mx, fmaf(xa.y, my, fmaf(xa.z, mz, Dnj)));
                const float ph = __fdividef(sq, r + Rf);
                const float wr = xa.w * rinv;
                const float wr3 = wr * (rinv * rinv);
                const float tj = wr3 * dnj;
                const float2 y = fmul2(kk, f2(ph));
                float2 sn, cs;
                if (PH == 2) {
                    dev_sincos_poly2<true>(y, sn, cs);
                } else if (PH == 1) {
                    dev_sincos_poly2<false>(y, sn, cs);
                } else {
                    dev_sincos(y.x, &sn.x, &cs.x);
                    dev_sincos(y.y, &sn.y, &cs.y);
                }
                const float2 rr = f2(r);
                const float2 kr = fmul2(kk, rr), nkr = fmul2(nkk, rr);
                const float2 w2 = f2(wr), w32 = f2(wr3);
                const float2 gr = fmul2(w2, cs), gim = fmul2(w2, sn);
                const float2 fr = ffma2(kr, sn, cs);
                const float2 fi = ffma2(nkr, cs, sn);
                const float2 t2 = f2(tj);
                sr[0] = fadd2(sr[0], gr);
                sr[1] = ffma2(p1, gr, sr[1]);
                sr[2] = ffma2(p2, gr, sr[2]);
                sr[3] = ffma2(t2, fr, sr[3]);
                const float2 hr = fmul2(w32, fr);
                sr[4] = fadd2(sr[4], hr);
                sr[5] = ffma2(p1, hr, sr[5]);
                sr[6] = ffma2(p2, hr, sr[6]);
                si[0] = fadd2(si[0], gim);
                si[1] = ffma2(p1, gim, si[1]);
                si[2] = ffma2(p2, gim, si[2]);
                si[3] = ffma2(t2, fi, si[3]);
                const float2 hi = fmul2(w32, fi);
                si[4] = fadd2(si[4], hi);
                si[5] = ffma2(p1, hi, si[5]);
                si[6] = ffma2(p2, hi, si[6]);
            }
            const double wb = double(yb.w);
            const double wb1 = wb * a.phi64[3 * b + 1], wb2 = wb * a.phi64[3 * b + 2];
            const double ndni =
                -(Dni64 - (double(yb.x) * ni64[0] + double(yb.y) * ni64[1] + double(yb.z) * ni64[2]));
            const double wbn = wb * ndni;
#pragma unroll
            for (int w = 0; w < 2; ++w) {
                const double s3r = w ? sr[3].y : sr[3].x, s3i = w ? si[3].y : si[3].x;
                const double g0r = w ? sr[0].y : sr[0].x, g0i = w ? si[0].y : si[0].x;
                const double g1r = w ? sr[1].y : sr[1].x, g1i = w ? si[1].y : si[1].x;
                const double g2r = w ? sr[2].y : sr[2].x, g2i = w ? si[2].y : si[2].x;
                const double h0r = w ? sr[4].y : sr[4].x, h0i = w ? si[4].y : si[4].x;
                const double h1r = w ? sr[5].y : sr[5].x, h1i = w ? si[5].y : si[5].x;
                const double h2r = w ? sr[6].y : sr[6].x, h2i = w ? si[6].y : si[6].x;
                acc(w, 0, wb * g0r, wb * g0i);
                acc(w, 1, wb * s3r, wb * s3i);
                acc(w, 2, wb1 * s3r, wb1 * s3i);
                acc(w, 3, wb2 * s3r, wb2 * s3i);
                acc(w, 4, wbn * h0r, wbn * h0i);
                acc(w, 5, wbn * h1r, wbn * h1i);
                acc(w, 6, wbn * h2r, wbn * h2i);
                acc(w, 7, wb1 * g0r, wb1 * g0i);
                acc(w, 8, wb2 * g0r, wb2 * g0i);
                acc(w, 9, wb * g1r, wb * g1i);
                acc(w, 10, wb1 * g1r, wb1 * g1i);
                acc(w, 11, wb2 * g1r, wb2 * g1i);
                acc(w, 12, wb * g2r, wb * g2i);
                acc(w, 13, wb1 * g2r, wb1 * g2i);
                acc(w, 14, wb2 * g2r, wb2 * g2i);
            }
        }
#pragma unroll
        for (int w = 0; w < 2; ++w) {
            if constexpr (SM) {
#pragma unroll
                for (int m = 0; m < 15; ++m) {
                    Mr[w][m] = mom[((w * 15 + m) * 2) * FAR_THREADS];
                    Mi[w][m] = mom[((w * 15 + m) * 2 + 1) * FAR_THREADS];
                }
            }
            calderon_epilogue<true>(a, w, li, lj, gi, gj, ni64, nj64, pf, Rd, Mr[w], Mi[w], true);
        }
    }
}

template <int PH, bool SM>
int launch_calderon_k2(bem_ctx* ctx, const CalArgs& a, cudaStream_t s) {
    dim3 grid((a.n + FAR_THREADS - 1) / FAR_THREADS, (a.n + FAR_TI - 1) / FAR_TI);
    if (grid.y > 65535) return bem_fail(ctx, BEM_ERR_INVALID, "calderon: too many panels for one launch");
    const size_t smem = FAR_TI * a.Q2 * sizeof(float4) + a.Q2 * sizeof(float4) +
                        (SM ? 60 * FAR_THREADS * sizeof(double) : 0);
    if (int rc = bem_check_cuda(ctx, cudaFuncSetAttribute(far_calderon_k2_kernel<PH, SM>,
                                                          cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                                "far_calderon_k2_kernel smem"))
        return rc;
    far_calderon_k2_kernel<PH, SM><<<grid, FAR_THREADS, smem, s>>>(a);
    ctx->launches++;
    return bem_check_cuda(ctx, cudaGetLastError(), "far_calderon_k2_kernel launch");
}

template <typename T, int NK, bool HELM, int PH>
int launch_calderon(bem_ctx* ctx, const CalArgs& a, cudaStream_t s) {
    dim3 grid((a.n + FAR_THREADS - 1) / FAR_THREADS, (a.n + FAR_TI - 1) / FAR_TI);
    if (grid.y > 65535) return bem_fail(ctx, BEM_ERR_INVALID, "calderon: too many panels for one launch");
    const size_t smem = FAR_TI * a.Q2 * sizeof(typename V4T<T>::type) + 2 * a.Q2 * sizeof(T);
    far_calderon_kernel<T, NK, HELM, PH><<<grid, FAR_THREADS, smem, s>>>(a);
    ctx->launches++;
    return bem_check_cuda(ctx, cudaGetLastError(), "far_calderon_kernel launch");
}

template <int PH>
int launch_calderon_x2(bem_ctx* ctx, const CalArgs& a, cudaStream_t s) {
    dim3 grid((a.n + FAR_THREADS - 1) / FAR_THREADS, (a.n + FAR_TI - 1) / FAR_TI);
    if (grid.y > 65535) return bem_fail(ctx, BEM_ERR_INVALID, "calderon: too many panels for one launch");
    const int P2 = (a.Q2 + 1) / 2;
    const size_t smem = (size_t)FAR_TI * P2 * (2 * sizeof(float4) + sizeof(float2)) + (size_t)P2 * sizeof(float4);
    far_calderon_x2_kernel<PH><<<grid, FAR_THREADS, smem, s>>>(a);
    ctx->launches++;
    return bem_check_cuda(ctx, cudaGetLastError(), "far_calderon_x2_kernel launch");
}

template <int NK>
int dispatch_calderon(bem_ctx* ctx, const CalArgs& a, bool fp32, bool helm, cudaStream_t s) {
    if (!fp32)
        return helm ? launch_calderon<double, NK, true, 0>(ctx, a, s) : launch_calderon<double, NK, false, 0>(ctx, a, s);
    if (!helm) return launch_calderon<float, NK, false, 0>(ctx, a, s);
    if (a.small_phase != 0) return launch_calderon<float, NK, true, 1>(ctx, a, s);
    return launch_calderon<float, NK, true, 0>(ctx, a, s);
}

}  // namespace

extern "C" int bem_assemble_calderon(bem_ctx* ctx, const bem_op_desc* op, int nk, const double* k, const double* k2,
                                     const bem_space* neu, const bem_space* dir, void* const* out,
                                     const double* coef, int64_t ld, void* stream) {
    if (!ctx) return BEM_ERR_INVALID;
    if (!op || !k || !k2 || !neu || !dir || !out || !coef || nk < 1 || nk > CAL_MAXK || ld <= 0 || op->deriv_k)
        return bem_fail(ctx, BEM_ERR_INVALID, "assemble_calderon: bad arguments");
    if (ctx->nt <= 0 || ctx->dim != 3) return bem_fail(ctx, BEM_ERR_NOMESH, "assemble_calderon: no 3D mesh set");
    if (neu->nb != 1 || dir->nb != 3 || neu->n_panels != dir->n_panels || neu->n_panels <= 0)
        return bem_fail(ctx, BEM_ERR_INVALID,
                        "assemble_calderon: needs a P0 Neumann and a P1 Dirichlet space over one panel list");
    for (int w = 0; w < nk; ++w)
        if (!out[w]) return bem_fail(ctx, BEM_ERR_INVALID, "assemble_calderon: null output");
    cudaStream_t s = (cudaStream_t)stream;
    const bool fp32 = op->precision == BEM_PREC_MIXED;
    const bool helm = op->kernel == BEM_KERNEL_HELMHOLTZ;
    // near pairs: the FP64 Sauter-Schwab kernels of each operator, per
    // wavenumber, on the high-priority side stream, concurrently with the far
    // sweep (different pipes; they write other V entries, and every entry they
    // share with the sweep -- the P1 columns and rows -- is added atomically);
    // the caller's stream waits for both
    if (int rc = bem_lookahead_stream(ctx)) return rc;
    if (int rc = bem_check_cuda(ctx, cudaEventRecord(ctx->ev_next, s), "calderon fork")) return rc;
    if (int rc = bem_check_cuda(ctx, cudaStreamWaitEvent(ctx->aux, ctx->ev_next, 0), "calderon fork")) return rc;
    const cudaStream_t sn = ctx->aux;
    for (int w = 0; w < nk; ++w) {
        bem_op_desc d = *op;
        d.k = k[w];
        d.k2 = k2[w];
        const double c = coef[w];
        d.op = BEM_OP_V;
        if (int rc = bem_launch_assemble_parts(ctx, &d, neu, neu, 0, out[w], ld, -c, nullptr, 0.0, nullptr, nullptr, 0,
                                               sn, true))
            return rc;
        d.op = BEM_OP_K;
        if (int rc = bem_launch_assemble_parts(ctx, &d, neu, dir, 0, out[w], ld, c, out[w], -c, nullptr, nullptr, 0,
                                               sn, true))
            return rc;
        d.op = BEM_OP_W;
        if (int rc = bem_launch_assemble_parts(ctx, &d, dir, dir, 0, out[w], ld, -c, nullptr, 0.0, nullptr, nullptr, 0,
                                               sn, true))
            return rc;
    }
    CalArgs a{};
    a.n = neu->n_panels;
    a.panels = neu->panels;
    a.ndof = neu->dof;
    a.ddof = dir->dof;
    a.tris = ctx->tris;
    a.centroid = ctx->centroid;
    a.normal = ctx->normal;
    a.curl = ctx->curl;
    a.area = ctx->area;
    a.wcorr = ctx->wcorr32;
    double kmax = 0.0;
    for (int w = 0; w < nk; ++w) kmax = std::fmax(kmax, std::fabs(k[w]));
    // class of the bound on the phase k (r - R): 2 (<= 0.3: short polynomial), 1 (<= pi/4: no argument
    // reduction), 0 (reduction)
    const int phase_class = fp32 && helm ? bem_phase_class(kmax * 2.0 * ctx->rho_max) : 0;
    a.small_phase = phase_class != 0 ? 1 : 0;
    a.pts = fp32 ? (const void*)ctx->pts32 : (const void*)ctx->pts64;
    a.phi = fp32 ? (const void*)ctx->phi32 : (const void*)ctx->phi64;
    a.phi64 = ctx->phi64;
    a.Q2 = ctx->Q2;
    for (int w = 0; w < nk; ++w) {
        a.k[w] = k[w];
        a.k2[w] = k2[w];
        a.coef[w] = coef[w];
        a.out[w] = (double*)out[w];
    }
    a.ld = ld;
    // default with two wavenumbers: both in one scalar launch (measured on the
    // 20480-panel transmission problem: FP64 1602 vs 1736 ms for one launch
    // per wavenumber; mixed 656 ms, against 802 ms scalar and 750 ms packed
    // FP32x2 per wavenumber); with one wavenumber the packed sweep is the
    // mixed Helmholtz default
    int rc = BEM_OK;
    const int variant = ctx->tune[BEM_TUNE_CALDERON_GROUP];
    if (fp32 && helm && nk == 2 && variant == 4) {
        // both wavenumbers packed into the FP32x2 lanes, one launch, moments in registers
        rc = phase_class == 2 ? launch_calderon_k2<2, false>(ctx, a, s)
                              : (phase_class == 1 ? launch_calderon_k2<1, false>(ctx, a, s)
                                                  : launch_calderon_k2<0, false>(ctx, a, s));
    } else if (fp32 && helm && nk == 2 && variant == 5) {
        // the same with the moments in shared memory (three CTAs per SM)
        rc = phase_class == 2 ? launch_calderon_k2<2, true>(ctx, a, s)
                              : (phase_class == 1 ? launch_calderon_k2<1, true>(ctx, a, s)
                                                  : launch_calderon_k2<0, true>(ctx, a, s));
    } else if (fp32 && helm && (variant == 3 || (variant == 0 && nk == 1))) {
        // packed FP32x2, one wavenumber per launch
        for (int w = 0; w < nk && !rc; ++w) {
            CalArgs b = a;
            b.k[0] = a.k[w];
            b.k2[0] = a.k2[w];
            b.coef[0] = a.coef[w];
            b.out[0] = a.out[w];
            rc = phase_class == 2 ? launch_calderon_x2<2>(ctx, b, s)
                                  : (phase_class == 1 ? launch_calderon_x2<1>(ctx, b, s) : launch_calderon_x2<0>(ctx, b, s));
        }
    } else if (nk == 2 && variant != 1) {
        rc = dispatch_calderon<2>(ctx, a, fp32, helm, s);
    } else {
        for (int w = 0; w < nk && !rc; ++w) {
            CalArgs b = a;
            b.k[0] = a.k[w];
            b.k2[0] = a.k2[w];
            b.coef[0] = a.coef[w];
            b.out[0] = a.out[w];
            rc = dispatch_calderon<1>(ctx, b, fp32, helm, s);
        }
    }
    // join: the caller's stream waits for the near-pair kernels
    if (int e = bem_check_cuda(ctx, cudaEventRecord(ctx->ev_diag, sn), "calderon join")) return e;
    if (int e = bem_check_cuda(ctx, cudaStreamWaitEvent(s, ctx->ev_diag, 0), "calderon join")) return e;
    return rc;
}
