// Shape derivatives of Galerkin BEM bilinear forms (the adjoint of the
// assembly): for the Laplace single layer V (P0 x P0) and double layer K
// (P0 test x P1 trial)
//
//   grad[v] += d/dX_v  sum_{rows r, cols c} lam[r] A[r, c] u[c]
//
// with X the vertex positions.  Nothing is stored between the forward solve
// and this pass: every quadrature point of every pair is recomputed, with the
// same rules as the assembly (separate pairs: the GaussQR^2 x GaussQR^2 tensor
// rule; coincident / edge / vertex pairs: the Sauter-Schwab points of
// bem_quadrature.cuh).  Per point x = sum_a beta_a(xi) P_a on panel i,
// y = sum_b beta_b(eta) Q_b on panel j, weight w = w_xi w_eta J_i J_j
// (J = 2 x area), the integrand's dependence on the vertices is
//   * through d = x - y:   d/dP_a = beta_a(xi) d/dd,   d/dQ_b = -beta_b(eta) d/dd;
//   * through J_i (and J_j for V):  dJ/dP_a = n x (P_{a+2} - P_{a+1});
//   * for K through N_j = J_j n_j = (Q_1 - Q_0) x (Q_2 - Q_1), linear in each
//     trial vertex.
// The near-field integrands keep the singularity order of the assembled ones
// (d/dd G ~ 1/r^2 multiplies beta_a(xi) - beta_a(eta) ~ r at a shared
// vertex), so the same quadrature integrates them.  All in FP64.
#include <cuda_runtime.h>

#include "bem_internal.cuh"
#include "bem_quadrature.cuh"

namespace {

constexpr int ADJ_THREADS = 128;
constexpr int ADJ_TI = 8;

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// d(2A)/dP_a for the vertices v[3][3] in the panel's stored order, unit normal n
__device__ __forceinline__ void jac_grad(const double v[3][3], const double n[3], int a, double g[3]) {
    const double* p2 = v[(a + 2) % 3];
    const double* p1 = v[(a + 1) % 3];
    const double e[3] = {p2[0] - p1[0], p2[1] - p1[1], p2[2] - p1[2]};
    g[0] = n[1] * e[2] - n[2] * e[1];
    g[1] = n[2] * e[0] - n[0] * e[2];
    g[2] = n[0] * e[1] - n[1] * e[0];
}

__device__ __forceinline__ void cross3(const double a[3], const double b[3], double c[3]) {
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}

// d(w . N)/dQ_b with N = (Q1 - Q0) x (Q2 - Q1): Q0: w x (Q2 - Q1), Q1: (Q2 - Q0) x w, Q2: w x (Q1 - Q0)
__device__ __forceinline__ void normal_grad(const double q[3][3], const double w[3], int b, double g[3]) {
    double e[3];
    if (b == 0) {
        for (int c = 0; c < 3; ++c) e[c] = q[2][c] - q[1][c];
        cross3(w, e, g);
    } else if (b == 1) {
        for (int c = 0; c < 3; ++c) e[c] = q[2][c] - q[0][c];
        cross3(e, w, g);
    } else {
        for (int c = 0; c < 3; ++c) e[c] = q[1][c] - q[0][c];
        cross3(w, e, g);
    }
}

// Per-pair moments.  For V: k = 1/(4 pi r); for K: k = (d_e . n_j)/(4 pi r^3)
// times the trial density u(eta), d_e = sgn d.
struct PairMoments {
    double S0;        // sum w k
    double SX[3][3];  // sum w beta_a(xi) dk/dd        (test vertex a)
    double SY[3][3];  // sum w beta_b(eta) dk/dd       (trial vertex b, enters with -)
    double SN[3];     // K: sum (w / J_j) u d_e / (4 pi r^3)   (derivative with respect to N_j)
    __device__ __forceinline__ void zero() {
        S0 = 0.0;
        for (int a = 0; a < 3; ++a)
            for (int c = 0; c < 3; ++c) SX[a][c] = SY[a][c] = 0.0;
        SN[0] = SN[1] = SN[2] = 0.0;
    }
    __device__ __forceinline__ void reduce() {
        S0 = warp_sum_d(S0);
        for (int a = 0; a < 3; ++a)
            for (int c = 0; c < 3; ++c) {
                SX[a][c] = warp_sum_d(SX[a][c]);
                SY[a][c] = warp_sum_d(SY[a][c]);
            }
        for (int c = 0; c < 3; ++c) SN[c] = warp_sum_d(SN[c]);
    }
};

// one point: d = x - y, weight w (with J_i J_j), barycentric weights bx, by,
// trial density uy (K), argument sign sgn (the swapped coincide term of K),
// 1/J_j (K)
template <int OP>
__device__ __forceinline__ void adj_point(PairMoments& M, const double d[3], double w, const double bx[3],
                                          const double by[3], double uy, double sgn, const double nj[3],
                                          double invJj) {
    const double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
    const double rinv = rsqrt(r2);
    const double rinv2 = rinv * rinv;
    double g[3];
    if (OP == BEM_OP_V) {
        const double G = BEM_INV4PI * rinv;
        M.S0 += w * G;
        const double f = -G * rinv2;  // dG/dd = -d / (4 pi r^3)
        for (int c = 0; c < 3; ++c) g[c] = w * f * d[c];
    } else {
        const double de[3] = {sgn * d[0], sgn * d[1], sgn * d[2]};
        const double dn = de[0] * nj[0] + de[1] * nj[1] + de[2] * nj[2];
        const double g3 = BEM_INV4PI * rinv * rinv2;  // 1/(4 pi r^3)
        const double wu = w * uy;
        M.S0 += wu * dn * g3;
        // d/dd [(d_e . n) g3(r)] = sgn [n g3 - 3 (d_e . n) d_e / (4 pi r^5)]
        for (int c = 0; c < 3; ++c) g[c] = sgn * wu * (nj[c] * g3 - 3.0 * dn * de[c] * g3 * rinv2);
        for (int c = 0; c < 3; ++c) M.SN[c] += wu * invJj * de[c] * g3;
    }
    for (int a = 0; a < 3; ++a)
        for (int c = 0; c < 3; ++c) {
            M.SX[a][c] += bx[a] * g[c];
            M.SY[a][c] += by[a] * g[c];
        }
}

struct AdjArgs {
    int n_test, n_trial;
    const int32_t* test_panels;
    const int32_t* test_dof;
    const int32_t* trial_panels;
    const int32_t* trial_dof;
    int nby;  // 1 (V) or 3 (K)
    const int32_t* tris;
    const double* verts;
    const double* centroid;
    const double* normal;
    const double* area;
    const double4* pts;   // FP64 separate-rule points (offset, weight with 2A)
    const double* phi64;  // [Q2*3] barycentric weights of the separate-rule points
    int Q2;
    int64_t n_near;
    const int4* near;
    const int32_t* test_local;
    const int32_t* trial_local;
    const double* gp;
    const double* gw;
    int Q;
    int quirk;
    const double* lam;
    const double* u;
    double* grad;
};

__device__ __forceinline__ void load_tri(const AdjArgs& a, int g, double v[3][3], double n[3]) {
    for (int b = 0; b < 3; ++b)
        for (int c = 0; c < 3; ++c) v[b][c] = a.verts[3 * a.tris[3 * g + b] + c];
    for (int c = 0; c < 3; ++c) n[c] = a.normal[3 * g + c];
}

// contributions of one pair's moments (scaled by cw) to its six vertices:
// test vertex a: cw [(dJ_i/dP_a)/J_i S0 + SX[a]]
// trial vertex b: V: cw [(dJ_j/dQ_b)/J_j S0 - SY[b]];  K: cw [-SY[b] + d(SN . N_j)/dQ_b]
template <int OP>
__device__ __forceinline__ void pair_grads(const PairMoments& M, double cw, const double vi[3][3], const double ni[3],
                                           double Ji, const double vj[3][3], const double nj[3], double Jj,
                                           double gx[3][3], double gy[3][3]) {
    for (int a = 0; a < 3; ++a) {
        double jg[3];
        jac_grad(vi, ni, a, jg);
        for (int c = 0; c < 3; ++c) gx[a][c] = cw * (jg[c] / Ji * M.S0 + M.SX[a][c]);
    }
    for (int b = 0; b < 3; ++b) {
        double t[3];
        if (OP == BEM_OP_V) {
            jac_grad(vj, nj, b, t);
            for (int c = 0; c < 3; ++c) gy[b][c] = cw * (t[c] / Jj * M.S0 - M.SY[b][c]);
        } else {
            normal_grad(vj, M.SN, b, t);
            for (int c = 0; c < 3; ++c) gy[b][c] = cw * (t[c] - M.SY[b][c]);
        }
    }
}

// ---- separate pairs: CTA = ADJ_TI test panels (shared memory) x ADJ_THREADS trial panels ----
template <int OP>
__global__ void __launch_bounds__(ADJ_THREADS) adj_far_kernel(AdjArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double4* sx = reinterpret_cast<double4*>(smem_raw);   // [ADJ_TI][Q2]
    double* sphi = reinterpret_cast<double*>(sx + ADJ_TI * a.Q2);  // [Q2*3]
    __shared__ int s_gi[ADJ_TI];
    __shared__ int s_tri[ADJ_TI][3];
    __shared__ double s_lam[ADJ_TI];
    const int Q2 = a.Q2;
    const int lj = blockIdx.x * ADJ_THREADS + threadIdx.x;
    const int li0 = blockIdx.y * ADJ_TI;
    const int lane = threadIdx.x & 31;
    for (int idx = threadIdx.x; idx < Q2 * 3; idx += ADJ_THREADS) sphi[idx] = a.phi64[idx];
    if (threadIdx.x < ADJ_TI) {
        const int li = li0 + threadIdx.x;
        const int gi = li < a.n_test ? a.test_panels[li] : -1;
        s_gi[threadIdx.x] = gi;
        const int row = li < a.n_test ? a.test_dof[li] : -1;
        s_lam[threadIdx.x] = row >= 0 ? a.lam[row] : 0.0;
        for (int c = 0; c < 3; ++c) s_tri[threadIdx.x][c] = gi >= 0 ? a.tris[3 * gi + c] : -1;
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < ADJ_TI * Q2; idx += ADJ_THREADS) {
        const int t = idx / Q2, q = idx - t * Q2;
        if (s_gi[t] >= 0) sx[idx] = a.pts[(size_t)s_gi[t] * Q2 + q];
    }
    __syncthreads();

    const bool valid_j = lj < a.n_trial;
    const int gj = valid_j ? a.trial_panels[lj] : 0;
    int tri_j[3];
    for (int c = 0; c < 3; ++c) tri_j[c] = a.tris[3 * gj + c];
    double vj[3][3], nj[3];
    load_tri(a, gj, vj, nj);
    const double Jj = 2.0 * a.area[gj];
    double cj[3];
    for (int c = 0; c < 3; ++c) cj[c] = a.centroid[3 * gj + c];
    // trial coefficient (V) or nodal data of the trial panel (K)
    double uj[3] = {0.0, 0.0, 0.0};
    if (valid_j)
        for (int b = 0; b < a.nby; ++b) {
            const int col = a.trial_dof[lj * a.nby + b];
            uj[b] = col >= 0 ? a.u[col] : 0.0;
        }
    double gyacc[3][3] = {{0.0}};
    const double4* ptsj = a.pts + (size_t)gj * Q2;

    for (int t = 0; t < ADJ_TI; ++t) {
        const int gi = s_gi[t];
        if (gi < 0) break;
        const bool sep = valid_j && s_lam[t] != 0.0 && (bem_relation(s_tri[t], tri_j, gi == gj) == REL_SEPARATE);
        double gx[3][3] = {{0.0}};
        if (sep) {
            double vi[3][3], ni[3];
            load_tri(a, gi, vi, ni);
            const double Ji = 2.0 * a.area[gi];
            double D[3];
            for (int c = 0; c < 3; ++c) D[c] = a.centroid[3 * gi + c] - cj[c];
            PairMoments M;
            M.zero();
            for (int b = 0; b < Q2; ++b) {
                const double4 yb = ptsj[b];
                const double by[3] = {sphi[3 * b], sphi[3 * b + 1], sphi[3 * b + 2]};
                const double ub = OP == BEM_OP_V ? 1.0 : by[0] * uj[0] + by[1] * uj[1] + by[2] * uj[2];
                for (int q = 0; q < Q2; ++q) {
                    const double4 xa = sx[t * Q2 + q];
                    const double d[3] = {D[0] + xa.x - yb.x, D[1] + xa.y - yb.y, D[2] + xa.z - yb.z};
                    const double bx[3] = {sphi[3 * q], sphi[3 * q + 1], sphi[3 * q + 2]};
                    adj_point<OP>(M, d, xa.w * yb.w, bx, by, ub, 1.0, nj, 1.0 / Jj);
                }
            }
            const double cw = s_lam[t] * (OP == BEM_OP_V ? uj[0] : 1.0);
            double gy[3][3];
            pair_grads<OP>(M, cw, vi, ni, Ji, vj, nj, Jj, gx, gy);
            for (int b = 0; b < 3; ++b)
                for (int c = 0; c < 3; ++c) gyacc[b][c] += gy[b][c];
        }
        // test-vertex gradients: reduce over the warp's trial panels
        for (int b = 0; b < 3; ++b)
            for (int c = 0; c < 3; ++c) gx[b][c] = warp_sum_d(gx[b][c]);
        if (lane == 0)
            for (int b = 0; b < 3; ++b)
                for (int c = 0; c < 3; ++c)
                    if (gx[b][c] != 0.0) atomicAdd(a.grad + 3 * s_tri[t][b] + c, gx[b][c]);
    }
    if (valid_j)
        for (int b = 0; b < 3; ++b)
            for (int c = 0; c < 3; ++c)
                if (gyacc[b][c] != 0.0) atomicAdd(a.grad + 3 * tri_j[b] + c, gyacc[b][c]);
}

// ---- near pairs: one warp per ordered pair of the near list ----
template <int OP>
__global__ void __launch_bounds__(128) adj_near_kernel(AdjArgs a) {
    const int lane = threadIdx.x & 31;
    const int64_t pid = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (pid >= a.n_near) return;
    const int4 e = a.near[pid];
    const int gi = e.x, gj = e.y, rel = e.z;
    const int li = a.test_local[gi], lj = a.trial_local[gj];
    if (li < 0 || lj < 0) return;  // warp-uniform
    const int row = a.test_dof[li];
    if (row < 0) return;
    const double lam = a.lam[row];
    if (lam == 0.0) return;
    double uj[3] = {0.0, 0.0, 0.0};
    for (int b = 0; b < a.nby; ++b) {
        const int col = a.trial_dof[lj * a.nby + b];
        uj[b] = col >= 0 ? a.u[col] : 0.0;
    }
    // slot order of the Sauter-Schwab maps (as in the assembly's near kernel)
    const int permx = a.quirk ? (0 | (1 << 2) | (2 << 4)) : (e.w & 63);
    const int permy = a.quirk ? (0 | (1 << 2) | (2 << 4)) : ((e.w >> 6) & 63);
    const int pmx[3] = {permx & 3, (permx >> 2) & 3, (permx >> 4) & 3};
    const int pmy[3] = {permy & 3, (permy >> 2) & 3, (permy >> 4) & 3};
    double vi[3][3], ni[3], vj[3][3], nj[3];
    load_tri(a, gi, vi, ni);
    load_tri(a, gj, vj, nj);
    const double Ji = 2.0 * a.area[gi], Jj = 2.0 * a.area[gj];
    double X[3][3], Y[3][3];  // slot s = stored vertex pm[s]
    int slotx[3], sloty[3];   // slot of stored vertex b
    for (int s = 0; s < 3; ++s) {
        for (int c = 0; c < 3; ++c) {
            X[s][c] = vi[pmx[s]][c];
            Y[s][c] = vj[pmy[s]][c];
        }
        slotx[pmx[s]] = s;
        sloty[pmy[s]] = s;
    }
    PairMoments M;
    M.zero();
    auto add = [&](double r1x, double r2x, double r1y, double r2y, double wj, bool second, double px1, double px2,
                   double py1, double py2) {
        const double sx_[3] = {1.0 - r1x, r1x - r2x, r2x};
        const double sy_[3] = {1.0 - r1y, r1y - r2y, r2y};
        double d[3];
        for (int c = 0; c < 3; ++c)
            d[c] = (sx_[0] * X[0][c] + sx_[1] * X[1][c] + sx_[2] * X[2][c]) -
                   (sy_[0] * Y[0][c] + sy_[1] * Y[1][c] + sy_[2] * Y[2][c]);
        // barycentric weights per stored vertex
        const double bx[3] = {sx_[slotx[0]], sx_[slotx[1]], sx_[slotx[2]]};
        const double by[3] = {sy_[sloty[0]], sy_[sloty[1]], sy_[sloty[2]]};
        double ub = 1.0;
        if (OP == BEM_OP_K) {
            // P1 data at the basis parameters of the trial side
            const double pb[3] = {1.0 - py1, py1 - py2, py2};
            ub = pb[sloty[0]] * uj[0] + pb[sloty[1]] * uj[1] + pb[sloty[2]] * uj[2];
        }
        (void)px1;
        (void)px2;
        adj_point<OP>(M, d, wj, bx, by, ub, second ? -1.0 : 1.0, nj, 1.0 / Jj);
    };
    const int Q = a.Q, Q4 = Q * Q * Q * Q;
    for (int p = lane; p < Q4; p += 32) {
        const int iw = p % Q, iz = (p / Q) % Q, iy = (p / (Q * Q)) % Q, ix = p / (Q * Q * Q);
        const double weight = (a.gw[ix] * a.gw[iy] * Ji) * (a.gw[iz] * a.gw[iw] * Jj);
        near_points(rel, a.quirk != 0, a.gp[ix], a.gp[iy], a.gp[iz], a.gp[iw], weight, add);
    }
    M.reduce();
    if (lane != 0) return;
    double gx[3][3], gy[3][3];
    pair_grads<OP>(M, lam * (OP == BEM_OP_V ? uj[0] : 1.0), vi, ni, Ji, vj, nj, Jj, gx, gy);
    const int32_t* ti = a.tris + 3 * gi;
    const int32_t* tj = a.tris + 3 * gj;
    for (int b = 0; b < 3; ++b)
        for (int c = 0; c < 3; ++c) {
            atomicAdd(a.grad + 3 * ti[b] + c, gx[b][c]);
            atomicAdd(a.grad + 3 * tj[b] + c, gy[b][c]);
        }
}

}  // namespace

int bem_launch_adjoint(bem_ctx* ctx, const bem_op_desc* op, const bem_space* test, const bem_space* trial,
                       const double* lam, const double* u, double* grad, cudaStream_t s) {
    if (int rc = bem_fill_local_map(ctx, test, ctx->test_local, s)) return rc;
    if (int rc = bem_fill_local_map(ctx, trial, ctx->trial_local, s)) return rc;
    AdjArgs a;
    a.n_test = test->n_panels;
    a.n_trial = trial->n_panels;
    a.test_panels = test->panels;
    a.test_dof = test->dof;
    a.trial_panels = trial->panels;
    a.trial_dof = trial->dof;
    a.nby = trial->nb;
    a.tris = ctx->tris;
    a.verts = ctx->verts;
    a.centroid = ctx->centroid;
    a.normal = ctx->normal;
    a.area = ctx->area;
    a.pts = ctx->pts64;
    a.phi64 = ctx->phi64;
    a.Q2 = ctx->Q2;
    a.n_near = ctx->n_near;
    a.near = ctx->near;
    a.test_local = ctx->test_local;
    a.trial_local = ctx->trial_local;
    a.gp = ctx->gp;
    a.gw = ctx->gw;
    a.Q = ctx->Q;
    a.quirk = op->quirk;
    a.lam = lam;
    a.u = u;
    a.grad = grad;
    const size_t smem = sizeof(double4) * ADJ_TI * ctx->Q2 + sizeof(double) * 3 * ctx->Q2;
    const dim3 fgrid((unsigned)((a.n_trial + ADJ_THREADS - 1) / ADJ_THREADS), (unsigned)((a.n_test + ADJ_TI - 1) / ADJ_TI));
    const unsigned nblocks = (unsigned)((a.n_near + 3) / 4);
    if (a.n_test > 0 && a.n_trial > 0) {
        if (op->op == BEM_OP_V) {
            adj_far_kernel<BEM_OP_V><<<fgrid, ADJ_THREADS, smem, s>>>(a);
            if (nblocks) adj_near_kernel<BEM_OP_V><<<nblocks, 128, 0, s>>>(a);
        } else {
            adj_far_kernel<BEM_OP_K><<<fgrid, ADJ_THREADS, smem, s>>>(a);
            if (nblocks) adj_near_kernel<BEM_OP_K><<<nblocks, 128, 0, s>>>(a);
        }
        ctx->launches += nblocks ? 2 : 1;
    }
    return bem_check_cuda(ctx, cudaGetLastError(), "adjoint kernels launch");
}
