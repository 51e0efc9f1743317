/*
 * Oracle (TEST INFRASTRUCTURE): CPU restatement of the reference's 3D BEM
 * assembly, in FP64 (the parity oracle) and FP32 (the reference's own 3D
 * precision, timed as the restated CPU baseline).  See oracle_core.h for the
 * reference file:line map.  Built by oracle/Makefile into oracle/liboracle.so;
 * loaded only by tests/, __graft_entry__.smoke() and bench.py's CPU legs.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* Gauss-Legendre nodes/weights on [0,1]: get_gaussion_integration_points_and_weights
   (src/BEM_functions/utils/functions.py:5-85) maps the [-1,1] rule by
   p = (x+1)/2, w = w/2.  The rule is computed here by Newton iteration on the
   Legendre recurrence (Golub-Welsch/Newton textbook method), which agrees with
   the reference's 16-digit tables to the last digit. */
int oracle_gauss(int n, double* pts, double* wts) {
    if (n < 1 || n > 16) return -1;
    for (int i = 0; i < n; ++i) {
        double x = cos(M_PI * (i + 0.75) / (n + 0.5));
        double dp = 0.0;
        for (int it = 0; it < 100; ++it) {
            double p0 = 1.0, p1 = x;
            for (int k = 2; k <= n; ++k) {
                double p2 = ((2.0 * k - 1.0) * x * p1 - (k - 1.0) * p0) / k;
                p0 = p1; p1 = p2;
            }
            if (n == 1) { p1 = x; p0 = 1.0; }
            dp = n * (x * p1 - p0) / (x * x - 1.0);
            double dx = p1 / dp;
            x -= dx;
            if (fabs(dx) < 1e-16) break;
        }
        /* recompute derivative at the converged node */
        double p0 = 1.0, p1 = x;
        for (int k = 2; k <= n; ++k) {
            double p2 = ((2.0 * k - 1.0) * x * p1 - (k - 1.0) * p0) / k;
            p0 = p1; p1 = p2;
        }
        dp = n * (x * p1 - p0) / (x * x - 1.0);
        double w = 2.0 / ((1.0 - x * x) * dp * dp);
        /* ascending order, as in the reference tables */
        pts[n - 1 - i] = (x + 1.0) / 2.0;
        wts[n - 1 - i] = w / 2.0;
    }
    if (n == 1) { pts[0] = 0.5; wts[0] = 1.0; }
    return 0;
}

/* get_panels_relation (src/managers/mesh_manager.py:538-573), 3D branch. */
int oracle_relation(const int* tris, int i, int j) {
    if (i == j) return 1;
    int rel = 0, common_vertex = 0;
    for (int ii = 0; ii < 3; ++ii) {
        int a1 = tris[3 * i + ii], a2 = tris[3 * i + (ii + 1) % 3];
        for (int jj = 0; jj < 3; ++jj) {
            int b1 = tris[3 * j + jj], b2 = tris[3 * j + (jj + 1) % 3];
            if (a1 == b1 && a2 == b2) rel = 3;
            if (a1 == b2 && a2 == b1) rel = 3;
            if (a1 == b1) common_vertex = 1;
        }
    }
    if (common_vertex && rel != 3) rel = 2;
    return rel;
}

/* Corrected-mode local orders for a near pair: the shared vertex becomes
   parameter slot 0 of both panels (vertex pair), or the shared edge becomes
   slots (0,1) of both panels with matching endpoints (edge pair), which is
   where the reference's Sauter-Schwab maps put the singularity. */
void oracle_near_perm(const int* tris, int i, int j, int rel, int* px, int* py) {
    const int* a = tris + 3 * i;
    const int* b = tris + 3 * j;
    px[0] = 0; px[1] = 1; px[2] = 2; py[0] = 0; py[1] = 1; py[2] = 2;
    if (rel == 2) {
        for (int s = 0; s < 3; ++s)
            for (int t = 0; t < 3; ++t)
                if (a[s] == b[t]) {
                    px[0] = s; px[1] = (s + 1) % 3; px[2] = (s + 2) % 3;
                    py[0] = t; py[1] = (t + 1) % 3; py[2] = (t + 2) % 3;
                    return;
                }
    } else if (rel == 3) {
        /* find the edge (s, s+1) of panel i whose endpoints both occur in panel j */
        for (int s = 0; s < 3; ++s) {
            int v0 = a[s], v1 = a[(s + 1) % 3];
            int t0 = -1, t1 = -1;
            for (int t = 0; t < 3; ++t) {
                if (b[t] == v0) t0 = t;
                if (b[t] == v1) t1 = t;
            }
            if (t0 >= 0 && t1 >= 0) {
                px[0] = s; px[1] = (s + 1) % 3; px[2] = (s + 2) % 3;
                py[0] = t0; py[1] = t1; py[2] = 3 - t0 - t1;
                return;
            }
        }
    }
}

enum { OP_V = 0, OP_K = 1, OP_KP = 2, OP_W = 3 };
enum { REL_SEPARATE = 0, REL_COINCIDE = 1, REL_VERTEX = 2, REL_EDGE = 3 };

#define REAL double
#define SFX _f64
#include "oracle_core.h"
#undef REAL
#undef SFX

#define REAL float
#define SFX _f32
#include "oracle_core.h"
#undef REAL
#undef SFX

int oracle_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}

/* helm: 0 Laplace, 1 Helmholtz.  k: kernel wavenumber (k*sqrt_n for the
   transmission kernel); k2: coefficient of the W mass term (k*sqrt_n)^2. */
int oracle_assemble(int fp32, const double* verts, const int* tris, int nt,
                    int op, int helm, double k, double k2, int Q, int quirk,
                    int n_test, const int* test_panels, int nbx, const int* test_dof,
                    int n_trial, const int* trial_panels, int nby, const int* trial_dof,
                    int is_complex, int mode, double* out, long ld, double scale,
                    double* out_t, double scale_t, const double* xvec, double* yvec, int conj_x) {
    if (fp32)
        return assemble_block_f32(verts, tris, nt, op, helm, k, k2, Q, quirk, n_test, test_panels, nbx, test_dof,
                                  n_trial, trial_panels, nby, trial_dof, is_complex, mode, out, ld, scale, out_t,
                                  scale_t, xvec, yvec, conj_x);
    return assemble_block_f64(verts, tris, nt, op, helm, k, k2, Q, quirk, n_test, test_panels, nbx, test_dof,
                              n_trial, trial_panels, nby, trial_dof, is_complex, mode, out, ld, scale, out_t,
                              scale_t, xvec, yvec, conj_x);
}

int oracle_mass(int fp32, const double* verts, const int* tris, int Q, int n_panels, const int* panels,
                int nbx, const int* test_dof, int nby, const int* trial_dof, int is_complex, int mode,
                double* out, long ld, double scale, double* out_t, double scale_t,
                const double* xvec, double* yvec, int conj_x) {
    if (fp32)
        return mass_block_f32(verts, tris, Q, n_panels, panels, nbx, test_dof, nby, trial_dof, is_complex, mode, out,
                              ld, scale, out_t, scale_t, xvec, yvec, conj_x);
    return mass_block_f64(verts, tris, Q, n_panels, panels, nbx, test_dof, nby, trial_dof, is_complex, mode, out, ld,
                          scale, out_t, scale_t, xvec, yvec, conj_x);
}
