// Galerkin assembly of the 2D operators on line-segment panels (the
// reference's dim = 2 path): V, K, K', W for the Laplace and Helmholtz kernels,
// the mass (identity) blocks, dense and matrix-free.
//
// Operator integrands follow single_layer_2d.py:56-215 (and the double,
// adjoint-double and hypersingular variants), the kernels G and grad_G_y
// BEM_manager.py:451-525 (2D branches):
//   Laplace    G = -(1/2pi) log r,        dG/dn_y = (1/2pi) (x - y).n_y / r^2
//   Helmholtz  G = (i/4) H0(kr),          dG/dn_y = (i/4) k H1(kr) (x - y).n_y / r
// with H0 = J0 + i Y0 and H1 = J1 + i Y1 (the derivative H0' = -H1 that the
// reference takes through scipy's h1vp), evaluated with the CUDA math
// library's j0/y0/j1/y1.  K' is grad_G_y with the roles of x and y swapped
// (adj_double_layer_2d.py: grad_G_y(x=y, y=x, normal_y=normal_x)); W is
//   G curl(phi_x) curl(phi_y) - k^2 G phi_x phi_y n_x.n_y
// with curl(phi) = n.x dphi/dy - n.y dphi/dx = (-1, +1)/L for the two hats
// (hypersingular_layer_2d.py:55-60,130-141).
//
// Quadrature (the reference's, point for point): a Q x Q Gauss rule on the
// two unit segments, x(r) = (1-r) x1 + r x2, weight w_x w_y L_x L_y, for
// separate panels and for panels sharing a vertex; for a panel with itself
// the two Duffy triangles D1 (r_x = xsi, r_y = xsi eta) and D2 (r_x = xsi eta,
// r_y = xsi), each with Jacobian xsi.  Hats phi_0 = 1 - r, phi_1 = r
// (BEM_manager.py:404-423); P0 has phi = 1.
//
// Everything is FP64: the 2D operators are O(N^2 Q^2) with small N and the
// Hankel functions have no cheap FP32 form; the precision flag of the
// descriptor does not change them.
//
// Layout: one CTA row per test panel (grid.y, strided), 128 trial panels per
// CTA (grid.x, one thread each).  Dense blocks scatter with atomics (P1 columns
// are shared by two panels); matrix-free products reduce over the warp, whose
// 32 threads share the test panel, before one atomic per row.
#include <cuda_runtime.h>

#include "bem_internal.cuh"

namespace {

constexpr int A2_THREADS = 128;
constexpr int A2_MAX_GRID_Y = 65535;
constexpr double INV2PI = 0.15915494309189533577;  // 1 / (2 pi)
constexpr double INV4PI = 0.07957747154594766788;  // 1 / (4 pi)

struct Asm2dArgs {
    int n_test, n_trial, nt;
    const int32_t* test_panels;
    const int32_t* test_dof;
    const int32_t* trial_panels;
    const int32_t* trial_dof;
    const double4* seg;  // [nt] (x1, y1, x2, y2)
    const double2* nrm;  // [nt] unit normal (e.y, -e.x) / |e|
    const double* len;   // [nt] segment length
    const double* gp;    // [Q] Gauss points on [0,1]
    const double* gw;    // [Q] Gauss weights
    int Q;
    double k, k2;
    int mode;  // 0 dense, 1 matrix-free
    double* out;
    int64_t ld;
    double scale;
    double* out_t;
    double scale_t;
    const double* x;
    double* y;
    int conj_x;
    int32_t* flags;
};

template <int NB>
__device__ __forceinline__ double hat(double r, int b) {
    return NB == 1 ? 1.0 : (b == 0 ? 1.0 - r : r);
}

// One pair of points (rx on the test panel, ry on the trial panel) with
// quadrature weight w, accumulated into the NBX x NBY block.
template <int OP, bool HELM, int NBX, int NBY>
__device__ __forceinline__ void point2d(const double4& sx, const double4& sy, const double2& nx, const double2& ny,
                                        double rx, double ry, double w, double k, double k2, double nn,
                                        const double* cx, const double* cy, double (&re)[NBX][NBY],
                                        double (&im)[NBX][NBY]) {
    const double px = sx.x + rx * (sx.z - sx.x), py = sx.y + rx * (sx.w - sx.y);
    const double qx = sy.x + ry * (sy.z - sy.x), qy = sy.y + ry * (sy.w - sy.y);
    const double dx = px - qx, dy = py - qy;
    const double r2 = dx * dx + dy * dy;
    double gr, gi = 0.0;  // kernel value (complex for Helmholtz)
    if (OP == BEM_OP_V || OP == BEM_OP_W) {
        if (HELM) {
            const double z = k * sqrt(r2);
            gr = -0.25 * y0(z);
            gi = 0.25 * j0(z);
        } else {
            gr = -INV4PI * log(r2);
        }
    } else {
        // K: (x - y).n_y ; K': (y - x).n_x
        const double dn = OP == BEM_OP_K ? (dx * ny.x + dy * ny.y) : -(dx * nx.x + dy * nx.y);
        if (HELM) {
            const double r = sqrt(r2);
            const double z = k * r;
            const double f = k * dn / r;
            gr = -0.25 * y1(z) * f;
            gi = 0.25 * j1(z) * f;
        } else {
            gr = INV2PI * dn / r2;
        }
    }
    gr *= w;
    gi *= w;
#pragma unroll
    for (int a = 0; a < NBX; ++a) {
        const double fa = hat<NBX>(rx, a);
#pragma unroll
        for (int b = 0; b < NBY; ++b) {
            double c = fa * hat<NBY>(ry, b);
            if (OP == BEM_OP_W) c = cx[a] * cy[b] - k2 * c * nn;
            re[a][b] += gr * c;
            if (HELM) im[a][b] += gi * c;
        }
    }
}

template <int OP, bool HELM, int NBX, int NBY>
__global__ void __launch_bounds__(A2_THREADS) asm2d_kernel(Asm2dArgs a) {
    const int lj = blockIdx.x * A2_THREADS + threadIdx.x;
    const int lane = threadIdx.x & 31;
    for (int li = blockIdx.y; li < a.n_test; li += gridDim.y) {
        const int gi = a.test_panels[li];
        int gj = lj < a.n_trial ? a.trial_panels[lj] : -1;
        bool ok_i = gi >= 0 && gi < a.nt;
        bool ok = ok_i && lj < a.n_trial && gj >= 0 && gj < a.nt;
        if (!ok_i || (lj < a.n_trial && !(gj >= 0 && gj < a.nt))) atomicExch(&a.flags[1], 1 + (ok_i ? lj : li));
        double re[NBX][NBY], im[NBX][NBY];
#pragma unroll
        for (int p = 0; p < NBX; ++p)
#pragma unroll
            for (int q = 0; q < NBY; ++q) re[p][q] = im[p][q] = 0.0;
        if (ok) {
            const double4 sx = a.seg[gi], sy = a.seg[gj];
            const double2 nx = a.nrm[gi], ny = a.nrm[gj];
            const double Lx = a.len[gi], Ly = a.len[gj];
            const double nn = nx.x * ny.x + nx.y * ny.y;
            double cx[NBX], cy[NBY];
#pragma unroll
            for (int p = 0; p < NBX; ++p) cx[p] = NBX == 1 ? 0.0 : (p == 0 ? -1.0 : 1.0) / Lx;
#pragma unroll
            for (int q = 0; q < NBY; ++q) cy[q] = NBY == 1 ? 0.0 : (q == 0 ? -1.0 : 1.0) / Ly;
            const double LL = Lx * Ly;
            if (gi != gj) {
                for (int ix = 0; ix < a.Q; ++ix) {
                    const double rx = a.gp[ix], wx = a.gw[ix] * LL;
                    for (int iy = 0; iy < a.Q; ++iy)
                        point2d<OP, HELM, NBX, NBY>(sx, sy, nx, ny, rx, a.gp[iy], wx * a.gw[iy], a.k, a.k2, nn, cx,
                                                    cy, re, im);
                }
            } else {
                for (int ix = 0; ix < a.Q; ++ix) {
                    const double xsi = a.gp[ix], wx = a.gw[ix] * LL * xsi;
                    for (int iy = 0; iy < a.Q; ++iy) {
                        const double eta = a.gp[iy], w = wx * a.gw[iy];
                        point2d<OP, HELM, NBX, NBY>(sx, sy, nx, ny, xsi, xsi * eta, w, a.k, a.k2, nn, cx, cy, re,
                                                    im);
                        point2d<OP, HELM, NBX, NBY>(sx, sy, nx, ny, xsi * eta, xsi, w, a.k, a.k2, nn, cx, cy, re,
                                                    im);
                    }
                }
            }
        }
        if (a.mode == 0) {
            if (ok) {
#pragma unroll
                for (int p = 0; p < NBX; ++p) {
                    const int row = a.test_dof[li * NBX + p];
                    if (row < 0) continue;
#pragma unroll
                    for (int q = 0; q < NBY; ++q) {
                        const int col = a.trial_dof[lj * NBY + q];
                        if (col < 0) continue;
                        if (HELM) {
                            double* o = a.out + 2 * ((int64_t)row * a.ld + col);
                            atomicAdd(o, a.scale * re[p][q]);
                            atomicAdd(o + 1, a.scale * im[p][q]);
                            if (a.out_t) {
                                double* t = a.out_t + 2 * ((int64_t)col * a.ld + row);
                                atomicAdd(t, a.scale_t * re[p][q]);
                                atomicAdd(t + 1, a.scale_t * im[p][q]);
                            }
                        } else {
                            atomicAdd(a.out + (int64_t)row * a.ld + col, a.scale * re[p][q]);
                            if (a.out_t) atomicAdd(a.out_t + (int64_t)col * a.ld + row, a.scale_t * re[p][q]);
                        }
                    }
                }
            }
        } else {
            // y[row_p] += scale * sum_q A[p][q] x[col_q] (x conjugated when conj_x)
#pragma unroll
            for (int p = 0; p < NBX; ++p) {
                double sr = 0.0, si = 0.0;
                if (ok) {
#pragma unroll
                    for (int q = 0; q < NBY; ++q) {
                        const int col = a.trial_dof[lj * NBY + q];
                        if (col < 0) continue;
                        if (HELM) {
                            const double xr = a.x[2 * col];
                            const double xi = a.conj_x ? -a.x[2 * col + 1] : a.x[2 * col + 1];
                            sr += re[p][q] * xr - im[p][q] * xi;
                            si += re[p][q] * xi + im[p][q] * xr;
                        } else {
                            sr += re[p][q] * a.x[col];
                        }
                    }
                }
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    sr += __shfl_xor_sync(0xffffffffu, sr, o);
                    if (HELM) si += __shfl_xor_sync(0xffffffffu, si, o);
                }
                const int row = ok_i ? a.test_dof[li * NBX + p] : -1;
                if (lane == 0 && row >= 0) {
                    if (HELM) {
                        atomicAdd(a.y + 2 * row, a.scale * sr);
                        atomicAdd(a.y + 2 * row + 1, a.scale * si);
                    } else {
                        atomicAdd(a.y + row, a.scale * sr);
                    }
                }
            }
        }
    }
}

struct Mass2dArgs {
    int n_panels, nbx, nby, nt;
    const int32_t* panels;
    const int32_t* test_dof;
    const int32_t* trial_dof;
    const double* len;
    const double* gp;
    const double* gw;
    int Q;
    int cplx, mode;
    double* out;
    int64_t ld;
    double scale;
    double* out_t;
    double scale_t;
    const double* x;
    double* y;
    int conj_x;
    int32_t* flags;
};

// Mass block on one panel list: L sum_q w_q phi_a(r_q) phi_b(r_q)
// (identity_layer_2d.py:45-110, rhs_constructor_2d.py:185-230), one thread
// per (panel, test basis, trial basis).
__global__ void mass2d_kernel(Mass2dArgs a) {
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    const int per = a.nbx * a.nby;
    if (id >= a.n_panels * per) return;
    const int li = id / per, r = id - li * per, p = r / a.nby, q = r - p * a.nby;
    const int row = a.test_dof[li * a.nbx + p], col = a.trial_dof[li * a.nby + q];
    if (row < 0 || col < 0) return;
    const int g = a.panels[li];
    if (g < 0 || g >= a.nt) {
        atomicExch(&a.flags[1], 1 + li);
        return;
    }
    const double L = a.len[g];
    double acc = 0.0;
    for (int iq = 0; iq < a.Q; ++iq) {
        const double t = a.gp[iq];
        const double fa = a.nbx == 1 ? 1.0 : (p == 0 ? 1.0 - t : t);
        const double fb = a.nby == 1 ? 1.0 : (q == 0 ? 1.0 - t : t);
        acc += fa * fb * (a.gw[iq] * L);
    }
    if (a.mode == 0) {
        if (a.cplx) {
            atomicAdd(a.out + 2 * ((int64_t)row * a.ld + col), a.scale * acc);
            if (a.out_t) atomicAdd(a.out_t + 2 * ((int64_t)col * a.ld + row), a.scale_t * acc);
        } else {
            atomicAdd(a.out + (int64_t)row * a.ld + col, a.scale * acc);
            if (a.out_t) atomicAdd(a.out_t + (int64_t)col * a.ld + row, a.scale_t * acc);
        }
    } else if (a.cplx) {
        const double xr = a.x[2 * col], xi = a.conj_x ? -a.x[2 * col + 1] : a.x[2 * col + 1];
        atomicAdd(a.y + 2 * row, a.scale * acc * xr);
        atomicAdd(a.y + 2 * row + 1, a.scale * acc * xi);
    } else {
        atomicAdd(a.y + row, a.scale * acc * a.x[col]);
    }
}

template <int OP, bool HELM>
int launch_nb(bem_ctx* ctx, int nbx, int nby, const Asm2dArgs& a, cudaStream_t s) {
    const dim3 grid((a.n_trial + A2_THREADS - 1) / A2_THREADS, a.n_test < A2_MAX_GRID_Y ? a.n_test : A2_MAX_GRID_Y);
    if (nbx == 1 && nby == 1)
        asm2d_kernel<OP, HELM, 1, 1><<<grid, A2_THREADS, 0, s>>>(a);
    else if (nbx == 1 && nby == 2)
        asm2d_kernel<OP, HELM, 1, 2><<<grid, A2_THREADS, 0, s>>>(a);
    else if (nbx == 2 && nby == 1)
        asm2d_kernel<OP, HELM, 2, 1><<<grid, A2_THREADS, 0, s>>>(a);
    else if (nbx == 2 && nby == 2)
        asm2d_kernel<OP, HELM, 2, 2><<<grid, A2_THREADS, 0, s>>>(a);
    else
        return bem_fail(ctx, BEM_ERR_INVALID, "2D spaces have nb = 1 (P0) or 2 (P1)");
    ctx->launches++;
    return bem_check_cuda(ctx, cudaGetLastError(), "asm2d_kernel launch");
}

template <int OP>
int launch_op(bem_ctx* ctx, bool helm, int nbx, int nby, const Asm2dArgs& a, cudaStream_t s) {
    return helm ? launch_nb<OP, true>(ctx, nbx, nby, a, s) : launch_nb<OP, false>(ctx, nbx, nby, a, s);
}

}  // namespace

int bem_launch_assemble2d(bem_ctx* ctx, const bem_op_desc* op, const bem_space* test, const bem_space* trial,
                          int mode, void* out, int64_t ld, double scale, void* out_t, double scale_t, const void* x,
                          void* y, int conj_x, cudaStream_t s) {
    if (test->n_panels == 0 || trial->n_panels == 0) return BEM_OK;
    Asm2dArgs a;
    a.n_test = test->n_panels;
    a.n_trial = trial->n_panels;
    a.nt = ctx->nt;
    a.test_panels = test->panels;
    a.test_dof = test->dof;
    a.trial_panels = trial->panels;
    a.trial_dof = trial->dof;
    a.seg = ctx->seg2;
    a.nrm = ctx->nrm2;
    a.len = ctx->area;
    a.gp = ctx->gp;
    a.gw = ctx->gw;
    a.Q = ctx->Q;
    a.k = op->k;
    a.k2 = op->k2;
    a.mode = mode;
    a.out = (double*)out;
    a.ld = ld;
    a.scale = scale;
    a.out_t = (double*)out_t;
    a.scale_t = scale_t;
    a.x = (const double*)x;
    a.y = (double*)y;
    a.conj_x = conj_x;
    a.flags = ctx->flags;
    const bool helm = op->kernel == BEM_KERNEL_HELMHOLTZ;
    switch (op->op) {
        case BEM_OP_V: return launch_op<BEM_OP_V>(ctx, helm, test->nb, trial->nb, a, s);
        case BEM_OP_K: return launch_op<BEM_OP_K>(ctx, helm, test->nb, trial->nb, a, s);
        case BEM_OP_KP: return launch_op<BEM_OP_KP>(ctx, helm, test->nb, trial->nb, a, s);
        case BEM_OP_W: return launch_op<BEM_OP_W>(ctx, helm, test->nb, trial->nb, a, s);
        default: return bem_fail(ctx, BEM_ERR_INVALID, "unknown operator");
    }
}

int bem_launch_mass2d(bem_ctx* ctx, const bem_space* test, const bem_space* trial, int is_complex, int mode,
                      void* out, int64_t ld, double scale, void* out_t, double scale_t, const void* x, void* y,
                      int conj_x, cudaStream_t s) {
    Mass2dArgs m;
    m.n_panels = test->n_panels;
    m.nbx = test->nb;
    m.nby = trial->nb;
    m.nt = ctx->nt;
    m.panels = test->panels;
    m.test_dof = test->dof;
    m.trial_dof = trial->dof;
    m.len = ctx->area;
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
    m.flags = ctx->flags;
    const int total = m.n_panels * m.nbx * m.nby;
    if (total == 0) return BEM_OK;
    mass2d_kernel<<<(total + 127) / 128, 128, 0, s>>>(m);
    ctx->launches++;
    return bem_check_cuda(ctx, cudaGetLastError(), "mass2d_kernel launch");
}
