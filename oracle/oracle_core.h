/*
 * CPU restatement of the reference's 3D Galerkin BEM quadrature -- TEST
 * INFRASTRUCTURE (the oracle).  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference legs of bench.py load it, and only as the checker
 * or as the timed CPU baseline; the product path never calls it.
 *
 * Parity is pinned by tests/test_oracle_golden.py against fixtures produced by
 * running the reference's own Python kernels (tests/golden/gen_golden.py).
 *
 * This header is included twice by bem_oracle.c, once with REAL=double
 * (suffix _f64, the FP64 oracle) and once with REAL=float (suffix _f32, the
 * reference's own 3D precision, used as the restated CPU baseline).
 *
 * Loop structure follows the reference on purpose (one outer iteration per
 * test panel, serial over trial panels x basis pairs x GaussQR^4 points, the
 * integrand recomputed per basis pair):
 *   single layer  src/BEM_functions/single_layer/single_layer_3d.py:55-433
 *   double layer  src/BEM_functions/double_layer/double_layer_3d.py:56-501
 *   adjoint K'    src/BEM_functions/adj_double_layer/adj_double_layer_3d.py:57-506
 *   hypersingular src/BEM_functions/hypersingular_layer/hypersingular_layer_3d.py:55-565
 *   identity      src/BEM_functions/identity_layer/identity_layer_3d.py:45-196
 *   G, grad_G_y   src/managers/BEM_manager.py:452-525
 *   coincide maps src/managers/BEM_manager.py:141-165
 *   relation      src/managers/mesh_manager.py:538-573
 */

#define CAT2(a, b) a##b
#define CAT(a, b) CAT2(a, b)
#define FN(name) CAT(name, SFX)

typedef struct { REAL re, im; } FN(cplx);

static inline FN(cplx) FN(c_make)(REAL a, REAL b) { FN(cplx) c; c.re = a; c.im = b; return c; }

typedef struct {
    REAL x1[3], x2[3], x3[3];  /* parametrisation vertices (possibly permuted) */
    REAL area;
    REAL normal[3];            /* geometric panel normal (original orientation) */
    REAL curl[3][3];           /* n x grad(phi_b) for original vertex b        */
    int inv_perm[3];           /* original vertex b sits at parameter slot inv_perm[b] */
} FN(panel_t);

static void FN(load_panel)(FN(panel_t)* P, const double* verts, const int* tris, int p, const int* perm) {
    const int* t = tris + 3 * p;
    double v[3][3];
    for (int a = 0; a < 3; ++a)
        for (int c = 0; c < 3; ++c) v[a][c] = verts[3 * t[a] + c];
    /* area and normal: mesh_manager.py:116-125 */
    double e1[3], e2[3], cr[3];
    for (int c = 0; c < 3; ++c) { e1[c] = v[1][c] - v[0][c]; e2[c] = v[2][c] - v[1][c]; }
    cr[0] = e1[1] * e2[2] - e1[2] * e2[1];
    cr[1] = e1[2] * e2[0] - e1[0] * e2[2];
    cr[2] = e1[0] * e2[1] - e1[1] * e2[0];
    double nrm = sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
    P->area = (REAL)(0.5 * nrm);
    for (int c = 0; c < 3; ++c) P->normal[c] = (REAL)(cr[c] / nrm);
    int pm[3] = {0, 1, 2};
    if (perm) { pm[0] = perm[0]; pm[1] = perm[1]; pm[2] = perm[2]; }
    for (int c = 0; c < 3; ++c) {
        P->x1[c] = (REAL)v[pm[0]][c];
        P->x2[c] = (REAL)v[pm[1]][c];
        P->x3[c] = (REAL)v[pm[2]][c];
    }
    for (int s = 0; s < 3; ++s) P->inv_perm[pm[s]] = s;
    /* surface gradient of the P1 hat of vertex b, then curl = n x grad:
       hypersingular_layer_3d.py:55-64,163-169 (original vertex order). */
    for (int b = 0; b < 3; ++b) {
        REAL u[3] = {0, 0, 0};
        u[b] = 1;
        REAL g[3] = {0, 0, 0};
        REAL d32[3], d13[3], d21[3];
        for (int c = 0; c < 3; ++c) {
            d32[c] = (REAL)(v[2][c] - v[1][c]);
            d13[c] = (REAL)(v[0][c] - v[2][c]);
            d21[c] = (REAL)(v[1][c] - v[0][c]);
        }
        const REAL* n = P->normal;
        REAL c32[3] = {n[1] * d32[2] - n[2] * d32[1], n[2] * d32[0] - n[0] * d32[2], n[0] * d32[1] - n[1] * d32[0]};
        REAL c13[3] = {n[1] * d13[2] - n[2] * d13[1], n[2] * d13[0] - n[0] * d13[2], n[0] * d13[1] - n[1] * d13[0]};
        REAL c21[3] = {n[1] * d21[2] - n[2] * d21[1], n[2] * d21[0] - n[0] * d21[2], n[0] * d21[1] - n[1] * d21[0]};
        for (int c = 0; c < 3; ++c) g[c] = (u[0] * c32[c] + u[1] * c13[c] + u[2] * c21[c]) / ((REAL)2 * P->area);
        P->curl[b][0] = n[1] * g[2] - n[2] * g[1];
        P->curl[b][1] = n[2] * g[0] - n[0] * g[2];
        P->curl[b][2] = n[0] * g[1] - n[1] * g[0];
    }
}

/* shape_function (BEM_manager.py:404-425); i = -1 means the P0 constant. */
static inline REAL FN(shape)(REAL r1, REAL r2, int i) {
    if (i == 0) return (REAL)1 - r1;
    if (i == 1) return r1 - r2;
    if (i == 2) return r2;
    return (REAL)1;
}

static inline void FN(interp)(const FN(panel_t)* P, REAL r1, REAL r2, REAL* out) {
    for (int c = 0; c < 3; ++c) out[c] = ((REAL)1 - r1) * P->x1[c] + (r1 - r2) * P->x2[c] + r2 * P->x3[c];
}

/* G (BEM_manager.py:473-483): k <= 0 selects Laplace. */
static inline FN(cplx) FN(green)(const REAL* x, const REAL* y, REAL k, int helm) {
    REAL d0 = x[0] - y[0], d1 = x[1] - y[1], d2 = x[2] - y[2];
    REAL r = (REAL)sqrt(d0 * d0 + d1 * d1 + d2 * d2);
    REAL s = (REAL)(0.25 / M_PI) / r;
    if (!helm) return FN(c_make)(s, 0);
    REAL kr = k * r;
    return FN(c_make)(s * (REAL)cos(kr), s * (REAL)sin(kr));
}

/* grad_G_y (BEM_manager.py:509-523): (x-y).n_y/(4 pi r^3) * (1 - ikr) e^{ikr}. */
static inline FN(cplx) FN(grad_green_y)(const REAL* x, const REAL* y, const REAL* ny, REAL k, int helm) {
    REAL d0 = x[0] - y[0], d1 = x[1] - y[1], d2 = x[2] - y[2];
    REAL r = (REAL)sqrt(d0 * d0 + d1 * d1 + d2 * d2);
    REAL dn = (d0 * ny[0] + d1 * ny[1] + d2 * ny[2]) / r;
    REAL s = (REAL)(0.25 / M_PI) * dn / (r * r);
    if (!helm) return FN(c_make)(s, 0);
    REAL kr = k * r;
    REAL c = (REAL)cos(kr), sn = (REAL)sin(kr);
    return FN(c_make)(s * (c + kr * sn), s * (sn - kr * c));
}

typedef struct {
    int op, helm;
    REAL k, k2;          /* k2 = (k sqrt_n)^2 for the W mass term */
    REAL curldot, ndot;  /* W only */
} FN(opctx_t);

/* One kernel evaluation at (x, y) with basis values phix/phiy, for the
   regular argument order (first=1) or the swapped coincide order (first=0). */
static inline FN(cplx) FN(eval)(const FN(opctx_t)* o, const FN(panel_t)* X, const FN(panel_t)* Y,
                                const REAL* x, const REAL* y, REAL phix, REAL phiy, int first) {
    FN(cplx) g;
    switch (o->op) {
        case OP_V:
            g = first ? FN(green)(x, y, o->k, o->helm) : FN(green)(y, x, o->k, o->helm);
            g.re *= phix * phiy; g.im *= phix * phiy;
            return g;
        case OP_K:
            g = first ? FN(grad_green_y)(x, y, Y->normal, o->k, o->helm) : FN(grad_green_y)(y, x, Y->normal, o->k, o->helm);
            g.re *= phix * phiy; g.im *= phix * phiy;
            return g;
        case OP_KP:
            g = first ? FN(grad_green_y)(y, x, X->normal, o->k, o->helm) : FN(grad_green_y)(x, y, X->normal, o->k, o->helm);
            g.re *= phix * phiy; g.im *= phix * phiy;
            return g;
        default: { /* W */
            g = first ? FN(green)(x, y, o->k, o->helm) : FN(green)(y, x, o->k, o->helm);
            REAL f = o->curldot - o->k2 * phix * phiy * o->ndot;
            g.re *= f; g.im *= f;
            return g;
        }
    }
}

/* integrate_on_two_panels for one 4D Gauss point (single_layer_3d.py:55-369
   and its double/adjoint/hypersingular twins).  bx/by are ORIGINAL vertex
   indices (-1 = P0); quirk=1 reproduces the reference's coincide treatment
   (basis values not swapped with the kernel arguments). */
static FN(cplx) FN(point)(const FN(opctx_t)* o, const FN(panel_t)* X, const FN(panel_t)* Y, int rel,
                          int bx, int by, REAL xsi, REAL eta1, REAL eta2, REAL eta3, REAL weight, int quirk) {
    FN(cplx) acc = FN(c_make)(0, 0);
    REAL x[3], y[3];
    int sx = bx < 0 ? -1 : X->inv_perm[bx];
    int sy = by < 0 ? -1 : Y->inv_perm[by];
#define ADDPT(r1x, r2x, r1y, r2y, jac)                                                   \
    do {                                                                                 \
        FN(interp)(X, (r1x), (r2x), x);                                                  \
        FN(interp)(Y, (r1y), (r2y), y);                                                  \
        REAL phx = FN(shape)((r1x), (r2x), sx), phy = FN(shape)((r1y), (r2y), sy);       \
        FN(cplx) v = FN(eval)(o, X, Y, x, y, phx, phy, 1);                               \
        acc.re += v.re * weight * (jac); acc.im += v.im * weight * (jac);                \
    } while (0)

    if (rel == REL_SEPARATE) {
        REAL r1x = xsi, r2x = eta1 * r1x, r1y = eta2, r2y = eta3 * r1y;
        ADDPT(r1x, r2x, r1y, r2y, r1x * r1y);
    } else if (rel == REL_COINCIDE) {
        REAL jac = xsi * xsi * xsi * eta1 * eta1 * eta2;
        REAL w[4] = {xsi, xsi * eta1, xsi * eta1 * eta2, xsi * eta1 * eta2 * eta3};
        static const REAL M[3][4][4] = {
            {{1, 0, 0, 0}, {1, -1, 1, 0}, {0, 0, 0, 1}, {0, 0, 1, 0}},
            {{1, 0, 0, 0}, {0, 1, -1, 1}, {0, 0, 1, 0}, {0, 0, 0, 1}},
            {{1, 0, 0, -1}, {0, 1, 0, -1}, {0, 0, 0, -1}, {0, 0, 1, -1}},
        };
        for (int m = 0; m < 3; ++m) {
            REAL z[4];
            for (int r = 0; r < 4; ++r) z[r] = M[m][r][0] * w[0] + M[m][r][1] * w[1] + M[m][r][2] * w[2] + M[m][r][3] * w[3];
            REAL r1x = z[0], r2x = z[1], r1y = z[0] - z[2], r2y = z[1] - z[3];
            FN(interp)(X, r1x, r2x, x);
            FN(interp)(Y, r1y, r2y, y);
            REAL phx = FN(shape)(r1x, r2x, sx), phy = FN(shape)(r1y, r2y, sy);
            FN(cplx) v1 = FN(eval)(o, X, Y, x, y, phx, phy, 1);
            FN(cplx) v2;
            if (quirk) {
                v2 = FN(eval)(o, X, Y, x, y, phx, phy, 0);
            } else {
                /* mirrored region: the test point is y's parameter, the trial point x's */
                REAL phx2 = FN(shape)(r1y, r2y, sx), phy2 = FN(shape)(r1x, r2x, sy);
                v2 = FN(eval)(o, X, Y, x, y, phx2, phy2, 0);
            }
            acc.re += (v1.re * weight * jac) + (v2.re * weight * jac);
            acc.im += (v1.im * weight * jac) + (v2.im * weight * jac);
        }
    } else if (rel == REL_VERTEX) {
        REAL jac = xsi * xsi * xsi * eta2;
        ADDPT(xsi, xsi * eta1, xsi * eta2, xsi * eta2 * eta3, jac);
        ADDPT(xsi * eta2, xsi * eta2 * eta3, xsi, xsi * eta1, jac);
    } else { /* REL_EDGE */
        REAL w0, w1, w2, w3;
        w0 = xsi; w1 = -xsi * eta1 * eta2; w2 = xsi * eta1 * ((REAL)1 - eta2); w3 = xsi * eta1 * eta3;
        ADDPT(w0, w3, w0 + w1, w2, xsi * xsi * xsi * eta1 * eta1);
        REAL jac = xsi * xsi * xsi * eta1 * eta1 * eta2;
        w0 = xsi; w1 = -xsi * eta1 * eta2 * eta3; w2 = xsi * eta1 * eta2 * ((REAL)1 - eta3); w3 = xsi * eta1;
        ADDPT(w0, w3, w0 + w1, w2, jac);
        w0 = xsi * ((REAL)1 - eta1 * eta2); w1 = xsi * eta1 * eta2; w2 = xsi * eta1 * eta2 * eta3; w3 = xsi * eta1 * ((REAL)1 - eta2);
        ADDPT(w0, w3, w0 + w1, w2, jac);
        w0 = xsi * ((REAL)1 - eta1 * eta2 * eta3); w1 = xsi * eta1 * eta2 * eta3; w2 = xsi * eta1; w3 = xsi * eta1 * eta2 * ((REAL)1 - eta3);
        ADDPT(w0, w3, w0 + w1, w2, jac);
        w0 = xsi * ((REAL)1 - eta1 * eta2 * eta3); w1 = xsi * eta1 * eta2 * eta3; w2 = xsi * eta1 * eta2; w3 = xsi * eta1 * ((REAL)1 - eta2 * eta3);
        ADDPT(w0, w3, w0 + w1, w2, jac);
    }
#undef ADDPT
    return acc;
}

/* Full GaussQR^4 sum for one panel pair and one basis pair (the reference's
   `for gauss_number in range(GaussQR4)` loop, same point order). */
static FN(cplx) FN(pair_integral)(const FN(opctx_t)* o0, const FN(panel_t)* X, const FN(panel_t)* Y, int rel,
                                  int bx, int by, int Q, const REAL* gp, const REAL* gw, int quirk) {
    FN(opctx_t) o = *o0;
    if (o.op == OP_W) {
        /* a P0 side has no hat function: surface_grad sees phi1=phi2=phi3=0 (basis index -1) */
        o.curldot = (bx < 0 || by < 0) ? (REAL)0
                    : X->curl[bx][0] * Y->curl[by][0] + X->curl[bx][1] * Y->curl[by][1] + X->curl[bx][2] * Y->curl[by][2];
        o.ndot = X->normal[0] * Y->normal[0] + X->normal[1] * Y->normal[1] + X->normal[2] * Y->normal[2];
    }
    FN(cplx) acc = FN(c_make)(0, 0);
    for (int ix = 0; ix < Q; ++ix)
        for (int iy = 0; iy < Q; ++iy)
            for (int iz = 0; iz < Q; ++iz)
                for (int iw = 0; iw < Q; ++iw) {
                    REAL wx = gw[ix] * gw[iy] * (X->area * (REAL)2);
                    REAL wy = gw[iz] * gw[iw] * (Y->area * (REAL)2);
                    FN(cplx) v = FN(point)(&o, X, Y, rel, bx, by, gp[ix], gp[iy], gp[iz], gp[iw], wx * wy, quirk);
                    acc.re += v.re; acc.im += v.im;
                }
    return acc;
}

/*
 * Assemble one operator block.
 *   mode 0: out[row*ld+col] += scale*val                  (dense block, real or complex interleaved)
 *           and, if out_t != NULL, out_t[col*ld+row] += scale_t*val  (the -K^T block of BEM_manager.py:619-622)
 *   mode 1: y[row] += scale * val * x[col]  (conj(x) when conj_x; matrix-free apply_*_boundary)
 * test/trial: panel lists (global ids) and dof tables [n*nb], dof < 0 = skipped,
 * nb = 1 (P0, basis -1) or 3 (P1, original vertex order).
 */
static int FN(assemble_block)(const double* verts, const int* tris, int nt,
                              int op, int helm, double k, double k2, int Q, int quirk,
                              int n_test, const int* test_panels, int nbx, const int* test_dof,
                              int n_trial, const int* trial_panels, int nby, const int* trial_dof,
                              int is_complex, int mode, double* out, long ld, double scale,
                              double* out_t, double scale_t, const double* xvec, double* yvec, int conj_x) {
    double gpd[16], gwd[16];
    if (oracle_gauss(Q, gpd, gwd) != 0) return -1;
    REAL gp[16], gw[16];
    for (int i = 0; i < Q; ++i) { gp[i] = (REAL)gpd[i]; gw[i] = (REAL)gwd[i]; }
    FN(opctx_t) o;
    o.op = op; o.helm = helm; o.k = (REAL)k; o.k2 = (REAL)k2; o.curldot = 0; o.ndot = 0;
    (void)nt;
#pragma omp parallel for schedule(dynamic, 1)
    for (int li = 0; li < n_test; ++li) {
        int gi = test_panels[li];
        for (int lj = 0; lj < n_trial; ++lj) {
            int gj = trial_panels[lj];
            int perm_x[3], perm_y[3];
            int rel = oracle_relation(tris, gi, gj);
            int use_perm = (!quirk) && (rel == REL_VERTEX || rel == REL_EDGE);
            if (use_perm) oracle_near_perm(tris, gi, gj, rel, perm_x, perm_y);
            FN(panel_t) X, Y;
            FN(load_panel)(&X, verts, tris, gi, use_perm ? perm_x : NULL);
            FN(load_panel)(&Y, verts, tris, gj, use_perm ? perm_y : NULL);
            for (int ii = 0; ii < nbx; ++ii) {
                for (int jj = 0; jj < nby; ++jj) {
                    int row = test_dof[li * nbx + ii];
                    int col = trial_dof[lj * nby + jj];
                    if (row < 0 || col < 0) continue;
                    int bx = nbx == 1 ? -1 : ii, by = nby == 1 ? -1 : jj;
                    FN(cplx) v = FN(pair_integral)(&o, &X, &Y, rel, bx, by, Q, gp, gw, quirk);
                    double vr = (double)v.re, vi = (double)v.im;
                    if (mode == 0) {
                        if (is_complex) {
#pragma omp atomic
                            out[2 * (row * ld + col)] += scale * vr;
#pragma omp atomic
                            out[2 * (row * ld + col) + 1] += scale * vi;
                            if (out_t) {
#pragma omp atomic
                                out_t[2 * (col * ld + row)] += scale_t * vr;
#pragma omp atomic
                                out_t[2 * (col * ld + row) + 1] += scale_t * vi;
                            }
                        } else {
#pragma omp atomic
                            out[row * ld + col] += scale * vr;
                            if (out_t) {
#pragma omp atomic
                                out_t[col * ld + row] += scale_t * vr;
                            }
                        }
                    } else {
                        if (is_complex) {
                            double xr = xvec[2 * col], xi = conj_x ? -xvec[2 * col + 1] : xvec[2 * col + 1];
#pragma omp atomic
                            yvec[2 * row] += scale * (vr * xr - vi * xi);
#pragma omp atomic
                            yvec[2 * row + 1] += scale * (vr * xi + vi * xr);
                        } else {
#pragma omp atomic
                            yvec[row] += scale * vr * xvec[col];
                        }
                    }
                }
            }
        }
    }
    return 0;
}

/* Identity (mass) block on one panel list: integrate_on_single_panel /
   integrate_on_single_triangle (identity_layer_3d.py:45-146,
   rhs_constructor_3d.py:203-254).  Same dof conventions as assemble_block;
   mode 0 writes out (and out_t transposed), mode 1 applies to x. */
static int FN(mass_block)(const double* verts, const int* tris, int Q,
                          int n_panels, const int* panels, int nbx, const int* test_dof, int nby, const int* trial_dof,
                          int is_complex, int mode, double* out, long ld, double scale, double* out_t, double scale_t,
                          const double* xvec, double* yvec, int conj_x) {
    double gpd[16], gwd[16];
    if (oracle_gauss(Q, gpd, gwd) != 0) return -1;
    for (int li = 0; li < n_panels; ++li) {
        FN(panel_t) X;
        FN(load_panel)(&X, verts, tris, panels[li], NULL);
        for (int ii = 0; ii < nbx; ++ii)
            for (int jj = 0; jj < nby; ++jj) {
                int row = test_dof[li * nbx + ii], col = trial_dof[li * nby + jj];
                if (row < 0 || col < 0) continue;
                int bx = nbx == 1 ? -1 : ii, by = nby == 1 ? -1 : jj;
                REAL acc = 0;
                for (int ix = 0; ix < Q; ++ix)
                    for (int iy = 0; iy < Q; ++iy) {
                        REAL r1 = (REAL)gpd[ix], r2 = (REAL)gpd[iy] * r1;
                        REAL w = (REAL)gwd[ix] * (REAL)gwd[iy] * (X.area * (REAL)2);
                        acc += (FN(shape)(r1, r2, bx) * FN(shape)(r1, r2, by)) * w * r1;
                    }
                double v = (double)acc;
                if (mode == 0) {
                    if (is_complex) {
                        out[2 * (row * ld + col)] += scale * v;
                        if (out_t) out_t[2 * (col * ld + row)] += scale_t * v;
                    } else {
                        out[row * ld + col] += scale * v;
                        if (out_t) out_t[col * ld + row] += scale_t * v;
                    }
                } else {
                    if (is_complex) {
                        double xr = xvec[2 * col], xi = conj_x ? -xvec[2 * col + 1] : xvec[2 * col + 1];
                        yvec[2 * row] += scale * v * xr;
                        yvec[2 * row + 1] += scale * v * xi;
                    } else {
                        yvec[row] += scale * v * xvec[col];
                    }
                }
            }
    }
    return 0;
}

#undef FN
#undef CAT
#undef CAT2
