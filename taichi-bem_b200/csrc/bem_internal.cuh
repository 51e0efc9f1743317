// Internal declarations shared by the bem_b200 translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <functional>
#include <string>

#include "../../include/bem_b200.h"

#define BEM_PI 3.14159265358979323846
#define BEM_INV4PI 0.079577471545947667884  // 1 / (4 pi)

// Maximum Gauss order (the reference ships tables for 1..8 and 12).
#define BEM_MAX_Q 12

struct bem_ctx {
    std::string err;
    int64_t launches = 0;
    int device = 0;
    int num_sms = 148;
    int tune[BEM_TUNE_KEYS] = {0};  // launch-shape choices (bem_ctx_set_tuning); 0 = built-in default

    // ---- mesh (device) ----
    int dim = 3;                 // 3: triangles (bem_mesh_set), 2: segments (bem_mesh_set_2d)
    int nv = 0, nt = 0, Q = 0, Q2 = 0;
    double* verts = nullptr;     // [nv*dim]
    int32_t* tris = nullptr;     // [nt*dim]
    double* area = nullptr;      // [nt] (2D: segment length)
    double* normal = nullptr;    // [nt*dim]
    double4* seg2 = nullptr;     // 2D: [nt] endpoints (x1, y1, x2, y2)
    double2* nrm2 = nullptr;     // 2D: [nt] unit normals
    double* centroid = nullptr;  // [nt*3]
    double* curl = nullptr;      // [nt*9]  curl of P1 hat b: [p*9 + b*3 + c]
    double4* pts64 = nullptr;    // [nt*Q2] separate-rule point offset from centroid (xyz) + weight (w)
    float4* pts32 = nullptr;     // [nt*Q2] same in FP32, weight of the reference triangle (no 2A)
    double wcorr32 = 1.0;        // (exact / FP32 reference weight sum)^2
    double rho_max = 0.0;        // largest centroid-to-vertex distance of a panel
    double* phi64 = nullptr;     // [Q2*3] P1 hat values at the separate-rule points
    float* phi32 = nullptr;      // [Q2*3]
    double* gp = nullptr;        // [Q]   Gauss points on [0,1]
    double* gw = nullptr;        // [Q]   Gauss weights on [0,1]
    int64_t n_near = 0;
    int4* near = nullptr;        // [n_near] (i, j, rel, perm bits)

    // ---- workspace (device) ----
    int32_t* test_local = nullptr;   // [nt] global panel -> local test index, -1 = absent
    int32_t* trial_local = nullptr;  // [nt]
    int32_t* flags = nullptr;        // [16] device-side status words
    void* ws = nullptr;              // linear-algebra workspace
    size_t ws_bytes = 0;
    void* big_ws = nullptr;          // FP16 split operands of the least-squares normal matrix
    size_t big_ws_bytes = 0;
    // high-priority side stream and events of the LU lookahead (made on first use)
    cudaStream_t aux = nullptr;
    cudaEvent_t ev_next = nullptr, ev_diag = nullptr;
};

// Host helpers (bem_api.cu)
int bem_fail(bem_ctx* ctx, int code, const std::string& msg);
int bem_check_cuda(bem_ctx* ctx, cudaError_t e, const char* what);
int bem_ws_reserve(bem_ctx* ctx, size_t bytes);
// Reports (BEM_ERR_TIMEOUT) and clears a tensor-core wait of an earlier
// bem_lu_factor_tiled that ran out (flags[4], read by the caller after a
// synchronisation as `value`).
int bem_take_factor_error(bem_ctx* ctx, int32_t value, cudaStream_t s);
// Flexible restarted GMRES(restart) in FP64 on op(x) = b, right-preconditioned
// by precond (applied in place to a vector; it may differ between
// applications, as a low-precision solve does): Arnoldi with classical
// Gram-Schmidt twice, Givens rotations on the host.  Each restart starts from
// the true residual b - op(x); a cycle that no longer halves it ends the
// iteration once it is <= accept.  x holds the initial guess (bem_linalg.cu).
int bem_fgmres(bem_ctx* ctx, bool C, int64_t n, const std::function<int(const double*, double*)>& apply_op,
               const std::function<int(double*)>& precond, const double* b, double* x, double tol, int maxit,
               int restart, double accept, int* iters, double* relres, cudaStream_t s);
// out[p][q] -= sum_k L[p][k] conj(L[q][k]) (FP64 out, lower 64 x 64 tiles;
// real when !C) on the tcgen05 tensor cores from FP16 hi/lo splits of the
// panel L (m x kb, ld), FP64 sums (bem_lstsq.cu).
int bem_herk_tc_update(bem_ctx* ctx, bool C, const double* L, int64_t ld, int m, int kb, double* out, int64_t ldo,
                       cudaStream_t s);
// The near-pair list of the uploaded triangle mesh (ctx->tris) into
// ctx->near / ctx->n_near, built on the device (bem_mesh.cu); synchronous.
int bem_build_near_list(bem_ctx* ctx, int nv, int nt);
// A device buffer of at least `bytes` owned by the context (grown, never
// shrunk; freed with it), for scratch that lives within one call.
int bem_big_ws(bem_ctx* ctx, size_t bytes, void** out);
// Explicit inverses of the 64 x 64 diagonal tiles of a tile-LU factor into
// dinv (bem_tilelu.cu); dtype BEM_F64/C128/F32/C64.
int bem_tile_inverses(bem_ctx* ctx, int dtype, const void* A, int64_t n, int64_t lda, void* dinv, cudaStream_t s);
// Asynchronous preconditioner step of the refinement (bem_tilelu.cu).
int bem_tiled_precond_async(bem_ctx* ctx, int dtype, const void* LU, int64_t n, int64_t lda, const int32_t* piv,
                            const void* dinv, const double* r, double** out, const int* skip, cudaStream_t s);

// Launch wrappers (bem_assembly.cu)
int bem_launch_geometry(bem_ctx* ctx, cudaStream_t s);
int bem_fill_local_map(bem_ctx* ctx, const bem_space* sp, int32_t* map, cudaStream_t s);
int bem_launch_adjoint(bem_ctx* ctx, const bem_op_desc* op, const bem_space* test, const bem_space* trial,
                       const double* lam, const double* u, double* grad, cudaStream_t s);
int bem_lookahead_stream(bem_ctx* ctx);
int bem_launch_assemble(bem_ctx* ctx, const bem_op_desc* op, const bem_space* test, const bem_space* trial,
                        int mode, void* out, int64_t ld, double scale, void* out_t, double scale_t, const void* x,
                        void* y, int conj_x, cudaStream_t s);
// bem_launch_assemble restricted to the near-pair (coincident / edge / vertex)
// kernel when near_only (the far pairs then come from a fused sweep).
int bem_launch_assemble_parts(bem_ctx* ctx, const bem_op_desc* op, const bem_space* test, const bem_space* trial,
                              int mode, void* out, int64_t ld, double scale, void* out_t, double scale_t,
                              const void* x, void* y, int conj_x, cudaStream_t s, bool near_only);
// One operator at nk Helmholtz wavenumbers (bem_kbatch.cu): far pairs in
// k-batched launches, near pairs per wavenumber.
int bem_launch_assemble_batch(bem_ctx* ctx, const bem_op_desc* op, const bem_space* test, const bem_space* trial,
                              int nk, const double* k, const double* k2, void* const* out, int64_t ld,
                              const double* scale, void* const* out_t, const double* scale_t, cudaStream_t s);
// Class of the bound on the FP32 split phase |k (r - R)| <= k (rho_i + rho_j):
// 2 when <= 0.3 (short polynomials), 1 when <= 0.78 < pi/4 (no reduction), 0 otherwise
int bem_phase_class(double bound);
int bem_launch_dirichlet(bem_ctx* ctx, const bem_op_desc* op, const bem_space* test, const bem_space* trial,
                         void* out, int64_t ld, double scale, const bem_space* rows, const bem_space* data,
                         const void* g, void* y, double scale_k, int conj_g, cudaStream_t s);
// 2D operators (bem_assembly2d.cu)
int bem_launch_assemble2d(bem_ctx* ctx, const bem_op_desc* op, const bem_space* test, const bem_space* trial,
                          int mode, void* out, int64_t ld, double scale, void* out_t, double scale_t, const void* x,
                          void* y, int conj_x, cudaStream_t s);
int bem_launch_mass2d(bem_ctx* ctx, const bem_space* test, const bem_space* trial, int is_complex, int mode,
                      void* out, int64_t ld, double scale, void* out_t, double scale_t, const void* x, void* y,
                      int conj_x, cudaStream_t s);
int bem_launch_mass(bem_ctx* ctx, const bem_space* test, const bem_space* trial, int is_complex, int mode, void* out,
                    int64_t ld, double scale, void* out_t, double scale_t, const void* x, void* y, int conj_x,
                    cudaStream_t s);

// Relation / near-pair encoding shared by host and device.
enum { REL_SEPARATE = 0, REL_COINCIDE = 1, REL_VERTEX = 2, REL_EDGE = 3 };

__host__ __device__ inline int bem_relation(const int32_t* a, const int32_t* b, bool same) {
    // get_panels_relation, src/managers/mesh_manager.py:538-573 (3D branch)
    if (same) return REL_COINCIDE;
    int rel = REL_SEPARATE;
    bool cv = false;
    for (int ii = 0; ii < 3; ++ii) {
        int a1 = a[ii], a2 = a[(ii + 1) % 3];
        for (int jj = 0; jj < 3; ++jj) {
            int b1 = b[jj], b2 = b[(jj + 1) % 3];
            if ((a1 == b1 && a2 == b2) || (a1 == b2 && a2 == b1)) rel = REL_EDGE;
            if (a1 == b1) cv = true;
        }
    }
    if (cv && rel != REL_EDGE) rel = REL_VERTEX;
    return rel;
}
