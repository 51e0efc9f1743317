/*
 * bem_b200 -- C ABI of the B200 Galerkin BEM engine (libbem_b200.so).
 *
 * The reference (GeCao/taichi-BEM) is Python + Taichi; its hot path is the
 * dense assembly of the boundary integral operators and the dense solve.
 * Each entry point below replaces one reference interface (cited per
 * function).  Conventions:
 *   - all array arguments are DEVICE pointers owned by the caller, except
 *     where a comment says "host";
 *   - calls are stream-ordered on the given stream and return BEM_OK (0) or
 *     a negative BEM_ERR_* code; the message of the last failure is
 *     bem_last_error(ctx);
 *   - the assembly, apply, mass, gemv, tiled-factorisation, adjoint and
 *     post-processing calls queue their work without synchronising.  The
 *     mesh uploads, the partial-pivoting factorisation and solves, the tiled
 *     solves, the refinement and GMRES synchronise the stream (to read a
 *     device status word or a residual norm).  A call that has to grow the context's
 *     workspace allocates device memory, which synchronises the device;
 *   - complex values are interleaved (re, im) doubles, as torch.complex128
 *     and the reference's ti.Vector(2) [re, im];
 *   - matrices are row-major with a leading dimension `ld` (elements);
 *   - a context is used by one host thread at a time.
 */
#ifndef BEM_B200_H
#define BEM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------- */
#define BEM_OK 0
#define BEM_ERR_INVALID (-1)     /* bad argument (sizes, enums, null pointers) */
#define BEM_ERR_CUDA (-2)        /* a CUDA runtime call failed */
#define BEM_ERR_NOMESH (-3)      /* no mesh set on the context */
#define BEM_ERR_NOCONVERGE (-4)  /* iterative refinement did not reach tol */
#define BEM_ERR_SINGULAR (-5)    /* zero pivot in the LU factorisation */
#define BEM_ERR_TIMEOUT (-6)     /* a device-side wait hit its iteration cap */
#define BEM_ERR_MESH (-7)        /* degenerate or non-finite mesh */

/* ---- enums (values follow src/BEM_functions/utils/types.py) -------------- */
#define BEM_OP_V 0   /* single layer      (single_layer_3d.py)          */
#define BEM_OP_K 1   /* double layer      (double_layer_3d.py)          */
#define BEM_OP_KP 2  /* adjoint double    (adj_double_layer_3d.py)      */
#define BEM_OP_W 3   /* hypersingular     (hypersingular_layer_3d.py)   */

#define BEM_KERNEL_LAPLACE 0
#define BEM_KERNEL_HELMHOLTZ 1

#define BEM_PREC_FP64 0   /* every quadrature point in FP64 (the plain path)           */
#define BEM_PREC_MIXED 1  /* separate pairs in FP32, coincident/edge/vertex pairs in FP64 */

#define BEM_F64 0   /* real double     */
#define BEM_C128 1  /* complex double  */
#define BEM_F32 2   /* real float      */
#define BEM_C64 3   /* complex float   */

typedef struct bem_ctx bem_ctx;

/* One operator evaluation (the arguments of the reference's
   `forward(scope_type, k, sqrt_n)`, single_layer_3d.py:371-372). */
typedef struct {
    int op;          /* BEM_OP_*                                                 */
    int kernel;      /* BEM_KERNEL_*                                             */
    double k;        /* kernel wavenumber: k, or k*sqrt_n for the transmission kernel */
    double k2;       /* coefficient of the W mass term, (k*sqrt_n)^2 (0 for Laplace) */
    int quirk;       /* 1: the reference's Sauter-Schwab orientation/basis handling;
                        0: shared vertex/edge moved to the map's singular point   */
    int precision;   /* BEM_PREC_*                                               */
    int deriv_k;     /* 1: the derivative of the Helmholtz kernel in its
                        wavenumber k at fixed k2 (dG/dk = i r G for V and W,
                        whose k2 mass term keeps its coefficient; d/dk of
                        grad G for K and K'), for bem_assemble and bem_apply
                        only (no reference counterpart: the k-derivative of
                        the operators of single_layer_3d.py:55-369 and
                        BEM_manager.py:476-517); 0 otherwise            */
} bem_op_desc;

/* One side (test or trial) of an operator block: the reference's local panel
   loop (`for local_I in range(num_of_panels_X)` + map_local_X_index_to_panel_index)
   with the charge index of each basis function
   (proj_from_local_panel_index_to_local_charge_index, BEM_manager.py:244-277). */
typedef struct {
    int n_panels;            /* panels on this side                                 */
    const int32_t* panels;   /* device [n_panels]: global panel index               */
    int nb;                  /* 1 = P0 (constant), P1 (hat at each vertex): 3 on a
                                triangle mesh, 2 on a segment mesh                  */
    const int32_t* dof;      /* device [n_panels*nb]: row/column index, <0 = skipped */
} bem_space;

/* ---- context ------------------------------------------------------------- */
/* No reference counterpart (the reference keeps its state in Taichi fields). */
int bem_ctx_create(bem_ctx** out_ctx);
int bem_ctx_destroy(bem_ctx* ctx);
const char* bem_last_error(const bem_ctx* ctx);
/* Number of kernels this library launched through ctx since creation (no
 * reference counterpart). */
int64_t bem_launch_count(const bem_ctx* ctx);
/* Launch-shape choices of this context (no reference counterpart), set by the
 * autotuner (bem_b200/tuning.py) after timing the candidates on this GPU;
 * value 0 restores the built-in default.  Keys:
 *   BEM_TUNE_CALDERON_GROUP  form of the fused Calderon sweep: 1 scalar, one
 *                            wavenumber per launch; 2 scalar, both in one
 *                            launch (the default for two wavenumbers); 3 packed
 *                            FP32x2 over test points, one wavenumber per
 *                            launch (the default of a single-wavenumber mixed
 *                            Helmholtz sweep); 4 both wavenumbers packed into
 *                            the FP32x2 lanes, one launch (mixed Helmholtz);
 *                            5 the same with its FP64 moments in shared memory
 *   BEM_TUNE_GRAM_KSEG       64-wide K stages per TMEM accumulation segment of
 *                            the tensor-core normal matrix (>= 1)
 *   BEM_TUNE_CHOL_NB         panel width of bem_chol_factor (a multiple of 64)
 *   BEM_TUNE_GRAM_BAND       tile columns per band of the normal-matrix tile
 *                            order (tiles running together share the L2's
 *                            operand panels); 1 gives row order
 *   BEM_TUNE_KBATCH_GROUP    wavenumbers per far-field launch of
 *                            bem_assemble_batch: 2 or 4 (default 4 in mixed
 *                            precision, 2 in FP64; P1 x P1 blocks always 2)
 *   BEM_TUNE_GRAM_PAIR       form of the tensor-core normal matrix and
 *                            Cholesky updates: 1 one CTA per 128 x 128 tile
 *                            (eight epilogue warps), 2 CTA pairs (tcgen05
 *                            cta_group::2) on 256 x 128 tiles, column order,
 *                            3 one CTA per tile with sixteen epilogue warps
 *   BEM_TUNE_LU_UPDATE       form of the FP32 tile LU's large trailing
 *                            updates on the tensor cores: 1 register-staged
 *                            operands, 2 TMA-fed persistent kernel over
 *                            pre-split TF32 operands */
#define BEM_TUNE_CALDERON_GROUP 0
#define BEM_TUNE_GRAM_KSEG 1
#define BEM_TUNE_CHOL_NB 2
#define BEM_TUNE_GRAM_BAND 3
#define BEM_TUNE_KBATCH_GROUP 4
#define BEM_TUNE_GRAM_PAIR 5
#define BEM_TUNE_LU_UPDATE 6
#define BEM_TUNE_KEYS 8
int bem_ctx_set_tuning(bem_ctx* ctx, int key, int value);

/* ---- mesh ------------------------------------------------------------------
 * Replaces MeshManager.initialization geometry (mesh_manager.py:84-139) and the
 * per-pair get_panels_relation (mesh_manager.py:538-573): uploads the mesh,
 * computes areas/normals/curls and the separate-pair quadrature points for
 * gauss_qr on the device, and builds the coincident/edge/vertex pair list.
 * verts (host) [nv*3] double, tris (host) [nt*3] int32.  Synchronous. */
int bem_mesh_set(bem_ctx* ctx, const double* verts, const int32_t* tris, int nv, int nt, int gauss_qr);
/* 2D variant (the reference's dim = 2 path): line-segment panels.  Replaces
 * MeshManager.initialization for dim = 2 (mesh_manager.py:74-75,108-113, e.g.
 * the segments of load_analytical_disk, :520-536) and the 2D branch of
 * get_panels_relation (mesh_manager.py:544-551).  verts (host) [nv*2] double,
 * segs (host) [nt*2] int32 (panel p runs from vertex segs[2p] to segs[2p+1]).
 * Lengths (the 2D "areas") and normals (e.y, -e.x)/|e| are computed here.
 * Afterwards bem_assemble, bem_apply, bem_assemble_dirichlet, bem_mass and
 * bem_mesh_geometry (normals [nt*2]) act on the 2D operators
 * (single_layer_2d.py, double_layer_2d.py, adj_double_layer_2d.py,
 * hypersingular_layer_2d.py, identity_layer_2d.py, rhs_constructor_2d.py),
 * always in FP64; P1 spaces have nb = 2; bem_adjoint_vertices is 3D only.
 * Synchronous. */
int bem_mesh_set_2d(bem_ctx* ctx, const double* verts, const int32_t* segs, int nv, int nt, int gauss_qr);
/* Number of ordered panel pairs of the current mesh that share a vertex
 * (coincident + edge + vertex pairs; on a 2D mesh, coincident + vertex): the
 * pairs get_panels_relation (mesh_manager.py:538-573) does not call
 * SEPARATE. */
int64_t bem_near_pair_count(const bem_ctx* ctx);
/* The near-pair list itself (no reference counterpart; the pairs
 * get_panels_relation, mesh_manager.py:538-573, does not classify as
 * separate): bem_near_pair_count(ctx) entries of four int32 (test panel,
 * trial panel, relation 1 coincident / 2 common vertex / 3 common edge,
 * packed parameter orders), ordered by test then trial panel, copied into
 * out (host or device memory).  Synchronous. */
int bem_near_pair_list(const bem_ctx* ctx, int32_t* out);
/* Copies the per-panel areas [nt] and unit normals [nt*3] (device pointers):
 * MeshManager's panel_areas / panel_normals (mesh_manager.py:108-139). */
int bem_mesh_geometry(const bem_ctx* ctx, double* areas, double* normals, void* stream);

/* ---- assembly ---------------------------------------------------------------
 * Dense block: out[row*ld+col] += scale*A(row,col) for every (test basis,
 * trial basis) pair with both dof >= 0; when out_t != NULL also
 * out_t[col*ld+row] += scale_t*A(row,col).  Replaces the operator forward
 * passes SingleLayer3d.forward (single_layer_3d.py:371-433),
 * DoubleLayer3d.forward (double_layer_3d.py:376-438),
 * HypersingularLayer3d.forward (hypersingular_layer_3d.py:437-500) and the
 * block scatter BEMManager.matA_add_M (BEM_manager.py:608-628, out_t = the
 * -K^T block).  out_dtype: BEM_F64 (Laplace) or BEM_C128 (Helmholtz). */
int bem_assemble(bem_ctx* ctx, const bem_op_desc* op, const bem_space* test, const bem_space* trial,
                 int out_dtype, void* out, int64_t ld, double scale, void* out_t, double scale_t,
                 void* stream);

/* Fused Calderon-block assembly of the transmission operator.  For each
 * wavenumber w < nk (nk = 1 or 2; kernel wavenumber k[w], W mass coefficient
 * k2[w]) adds to out[w] (BEM_F64 for Laplace or BEM_C128, row-major, ld) the
 * block operator c = coef[w] times M(k) = [K -V; -W -K'] with the reference's
 * placement (matA_add_M, BEM_manager.py:608-628):
 *   out_NN += -c V,  out_ND += c K,  out_DN += -c K^T,  out_DD += -c W,
 * rows and columns given by the dof tables of `neu` (P0, nb = 1) and `dir`
 * (P1, nb = 3), two spaces over the same panel list.  Replaces
 * matrix_layer_forward (BEM_manager.py:829-844: SingleLayer3d.forward,
 * DoubleLayer3d.forward, HypersingularLayer3d.forward, one Taichi kernel per
 * operator and scope) followed by assemble_matA(ADD_P_MINUS / ADD_P_PLUS)
 * without the identity term (bem_mass adds that).  Separate pairs run in ONE
 * sweep over unordered panel pairs whose point evaluations serve V, K, K^T
 * and W; near pairs take the FP64 Sauter-Schwab kernels.  op gives kernel,
 * precision and quirk (op->op is ignored).  3D only; queued without
 * synchronising. */
int bem_assemble_calderon(bem_ctx* ctx, const bem_op_desc* op, int nk, const double* k, const double* k2,
                          const bem_space* neu, const bem_space* dir, void* const* out, const double* coef,
                          int64_t ld, void* stream);

/* Batched dense assembly over wavenumbers: for w < nk,
 *   out[w][row*ld+col] += scale[w] * A(k[w])(row,col)   and, when out_t and
 *   out_t[w] are not NULL, out_t[w][col*ld+row] += scale_t[w] * A(k[w])(row,col),
 * A(k) the Helmholtz operator op->op with kernel wavenumber k[w] and W mass
 * coefficient k2[w] (op->k and op->k2 are ignored; with op->deriv_k the
 * kernel's k-derivative at fixed k2, as in bem_assemble).  k, k2, scale, scale_t,
 * out and out_t are host arrays of nk entries; out/out_t hold device
 * pointers to BEM_C128 blocks.  Every separate panel pair's geometry is
 * evaluated once for 2 or 4 wavenumbers (BEM_TUNE_KBATCH_GROUP); near pairs
 * take the FP64 Sauter-Schwab kernel per wavenumber.  Replaces the per-k
 * operator forward passes of the reference's wavenumber sweep
 * (demo/demo_3d_plot_Sio.py:63-82 -> get_mat_A1_inv_norm /
 * get_augment_mat_A1_inv_norm, BEM_manager.py:922-988 ->
 * matrix_layer_forward, BEM_manager.py:829-844, at the exterior and the
 * interior wavenumber).  3D Helmholtz only; 1 <= nk <= BEM_MAX_KBATCH; queued
 * without synchronising. */
#define BEM_MAX_KBATCH 64
int bem_assemble_batch(bem_ctx* ctx, const bem_op_desc* op, const bem_space* test, const bem_space* trial,
                       int nk, const double* k, const double* k2, void* const* out, int64_t ld,
                       const double* scale, void* const* out_t, const double* scale_t, void* stream);

/* One step of a growing orthonormal basis by classical Gram-Schmidt with
 * one re-orthogonalisation (no reference counterpart: the reference takes
 * full SVDs in compute_inv_norm, BEM_manager.py:874-920; this is the basis
 * growth of this library's block-Krylov norm estimator).  Q is n x ldq
 * (row-major, BEM_F64 or BEM_C128) whose first j columns are orthonormal; v
 * (n entries, element stride ldv) is not modified.  Twice h = Q^H v,
 * v' -= Q h, r += h; r_jj = ||v'||; q = v' / r_jj projected twice more and
 * normalised; then Q[:, j] = q, Rt[j][0..j-1] = r, Rt[j][j] = r_jj (Rt
 * row-major, ldr).  One cooperative launch, deterministic sums, queued
 * without synchronising unless check != 0, which synchronises and reports a
 * grid-barrier timeout of this or an earlier unchecked call. */
int bem_cgs2_append(bem_ctx* ctx, int dtype, void* Q, int64_t n, int64_t ldq, int j, const void* v, int64_t ldv,
                    void* Rt, int64_t ldr, int check, void* stream);

/* Matrix-free apply: y[row] += scale * sum_col A(row,col) * x[col]
 * (x conjugated when conj_x != 0, the reference's cmul(integrand, cconj(g))).
 * Replaces apply_V_dot_N_boundary (single_layer_3d.py:435-498),
 * apply_K_dot_D_boundary (double_layer_3d.py:440-501),
 * apply_K_dot_N_boundary (adj_double_layer_3d.py:444-506) and
 * apply_W_dot_D_boundary (hypersingular_layer_3d.py:502-565).
 * dtype: BEM_F64 or BEM_C128 for both x and y. */
int bem_apply(bem_ctx* ctx, const bem_op_desc* op, const bem_space* test, const bem_space* trial,
              int dtype, const void* x, void* y, double scale, int conj_x, void* stream);

/* Fused Dirichlet-system pass: out[row*ld+col] += scale*V(row,col) over
 * test x trial (both P0) AND y[rows(i)] += scale_k * sum_j K(i,j) g over the
 * same panel pairs, K's trial basis and data indices given by `data` (same
 * panel list as `trial`, nb = 1 or 3, indices into g; g conjugated when
 * conj_g).  One sweep over the quadrature points serves both integrands; it
 * replaces SingleLayer3d.forward (single_layer_3d.py:371-433) followed by
 * DoubleLayer3d.apply_K_dot_D_boundary (double_layer_3d.py:440-501) in
 * BEMManager.run for the Dirichlet problem.  op->op must be BEM_OP_V. */
int bem_assemble_dirichlet(bem_ctx* ctx, const bem_op_desc* op, const bem_space* test, const bem_space* trial,
                           void* out, int64_t ld, double scale, const bem_space* rows, const bem_space* data,
                           const void* g, void* y, double scale_k, int conj_g, void* stream);

/* Identity (mass) block on one panel list (the test side's `panels`; the
 * trial side must have the same n_panels and only contributes its dof table):
 * dense (out/out_t) or apply (x != NULL: y += scale*M*x).  Replaces
 * IdentityLayer3d.matA_add_global_Identity_matrix (identity_layer_3d.py:148-196)
 * and RHSConstructor3d.multiply_identity_to_vector (rhs_constructor_3d.py:256-359). */
int bem_mass(bem_ctx* ctx, const bem_space* test, const bem_space* trial, int dtype,
             void* out, int64_t ld, double scale, void* out_t, double scale_t,
             const void* x, void* y, int conj_x, void* stream);

/* Shape derivative of a Laplace bilinear form (no reference counterpart: the
 * reference has no derivatives; this is the adjoint pass of the shape-gradient
 * workload).  grad (device [nv*3], FP64) is accumulated:
 *   grad[3 v + c] += d/dX_{v,c}  sum_{r, c'} lam[r] A(r, c') u[c']
 * with A the block of op->op (BEM_OP_V with P0 test and P0 trial spaces, or
 * BEM_OP_K with a P0 test and a P1 trial space), op->kernel BEM_KERNEL_LAPLACE,
 * lam indexed by the test space's dof numbers and u by the trial space's.
 * Every quadrature point is recomputed in FP64 (op->quirk selects the near-
 * field maps as in bem_assemble); nothing is stored by the forward pass. */
int bem_adjoint_vertices(bem_ctx* ctx, const bem_op_desc* op, const bem_space* test, const bem_space* trial,
                         const double* lam, const double* u, double* grad, void* stream);

/* ---- dense linear algebra (replaces torch.linalg.solve, BEM_manager.py:1056) --
 * LU with partial pivoting in place (row-major, n x n, lda).  dtype
 * BEM_F64/BEM_C128 (plain FP64 path) or BEM_F32/BEM_C64 (low-precision factor
 * of the mixed path; trailing updates on the tensor cores).  piv: device
 * int32[n] (LAPACK-style: row i was swapped with piv[i]).  info: device int32,
 * set to 0 or to 1+index of the first zero pivot. */
int bem_lu_factor(bem_ctx* ctx, int dtype, void* A, int64_t n, int64_t lda, int32_t* piv, int32_t* info,
                  void* stream);
/* Solve with the factors: b (n x nrhs, row-major, ldb) overwritten by x (the
 * solve half of torch.linalg.solve, BEM_manager.py:1056). */
int bem_lu_solve(bem_ctx* ctx, int dtype, const void* LU, int64_t n, int64_t lda, const int32_t* piv,
                 void* b, int64_t nrhs, int64_t ldb, void* stream);
/* y = alpha*A*x + beta*y for one vector (dtype of A: F64/C128/F32/C64; x, y in
 * the matching FP64 type F64/C128).  Replaces the product of assemble_rhs
 * (BEM_manager.py:647-662) and Jacobian_solver (:803-821); also the
 * refinement residual. */
int bem_gemv(bem_ctx* ctx, int a_dtype, const void* A, int64_t m, int64_t n, int64_t lda,
             const void* x, void* y, double alpha, double beta, void* stream);

/* Tile-pivoted LU (the low-precision factor of the mixed path; replaces the
 * same torch.linalg.solve call, BEM_manager.py:1056): partial pivoting restricted to each 64x64
 * diagonal tile, explicit inverses of the diagonal tiles written to `dinv`
 * (device, bem_lu_dinv_elems(n) elements of the dtype's complex-pair width:
 * 2 x float / 2 x double per element).  No grid-wide synchronisation. */
int64_t bem_lu_dinv_elems(int64_t n);
/* The factorisation (replaces the factor half of torch.linalg.solve,
 * BEM_manager.py:1056).  Queued without synchronisation, except that the
 * first factorisation of a size may grow the context's workspace for the
 * split operands of its large trailing updates (BEM_TUNE_LU_UPDATE = 2, a
 * device synchronisation).  A tensor-core wait
 * of the trailing updates
 * that ran out of its iteration cap is reported (BEM_ERR_TIMEOUT) by the next
 * bem_lu_solve_tiled, bem_refine_solve or bem_lu_factor_status on the same
 * context. */
int bem_lu_factor_tiled(bem_ctx* ctx, int dtype, void* A, int64_t n, int64_t lda, int32_t* piv, void* dinv,
                        int32_t* info, void* stream);
/* Status of the last bem_lu_factor_tiled on ctx (no reference counterpart):
 * synchronises the stream and returns BEM_ERR_TIMEOUT if a tensor-core wait of
 * that factorisation ran out of its iteration cap (the factors are then not
 * valid), else BEM_OK.  Reading the status clears it. */
int bem_lu_factor_status(bem_ctx* ctx, void* stream);
/* The solve half of torch.linalg.solve (BEM_manager.py:1056):
 * x = U^{-1} L^{-1} P b for one FP64 right-hand side b (overwritten), with the
 * factors of bem_lu_factor_tiled; a persistent kernel driven by per-tile ready
 * flags (bounded waits; BEM_ERR_TIMEOUT if one runs out). */
int bem_lu_solve_tiled(bem_ctx* ctx, int dtype, const void* LU, int64_t n, int64_t lda, const int32_t* piv,
                       const void* dinv, void* b, void* stream);

/* Allocation-free variant of bem_lu_solve_tiled (no reference counterpart
 * beyond the solve of BEM_manager.py:1056).  For callers that must not allocate device memory once they are
 * running -- for example an application whose device memory is owned by
 * another allocator, or a latency-critical loop where cudaMalloc's implicit
 * device synchronisation is not acceptable -- and that therefore cannot create
 * a bem_ctx workspace.  It takes no context and performs no allocation: its
 * scratch is a file-scope device array sized for n <= BEM_STATIC_SOLVE_MAX_N
 * (about 0.65 MB, held by every GPU that loads the library until the process
 * exits); larger n is rejected with BEM_ERR_INVALID.  The first call on a
 * device looks up the array's device address (cudaGetSymbolAddress) with that
 * device current and caches it per device ordinal, i.e. for the runtime's
 * primary context of that device; a caller that switches the current device
 * between driver-API contexts of one device is not supported.  All calls
 * share the one array, so calls that overlap on the GPU (other streams, other
 * host threads) race; serialise them.  Every call synchronises the stream (it
 * reads its wait status back to the host).  Same arguments as
 * bem_lu_solve_tiled without the context.  Unlike bem_lu_solve_tiled it
 * cannot see the factorisation's own status, which lives in the context: a
 * factor whose tensor-core wait timed out is not reported here, so check
 * bem_lu_factor_status on the factor's context before the first solve with a
 * new factor.  Returns BEM_OK, BEM_ERR_INVALID, BEM_ERR_CUDA or
 * BEM_ERR_TIMEOUT (a wait of this solve ran out). */
#define BEM_STATIC_SOLVE_MAX_N 32768
int bem_lu_solve_tiled_static(int dtype, const void* LU, int64_t n, int64_t lda, const int32_t* piv,
                              const void* dinv, void* b, void* stream);

/* Mixed-precision solve, in place of torch.linalg.solve (BEM_manager.py:1056):
 * x = A_hi^{-1} b to relative residual tol by FP64
 * iterative refinement on the residual b - A_hi x, each correction solved with
 * the low-precision factors (LU_lo, piv[, dinv]) of A_hi: tile-pivoted factors
 * when dinv != NULL, else partial-pivoting factors.  A_hi: F64/C128, LU_lo:
 * F32/C64.  iters/relres: host pointers (may be NULL).  Returns
 * BEM_ERR_NOCONVERGE if maxit is reached or the residual stops decreasing.
 * With tile-pivoted factors the iterations are queued in batches and the
 * convergence test runs on the device, so the call synchronises the stream
 * once per batch of three iterations (and reports a timeout of the preceding
 * bem_lu_factor_tiled); with partial-pivoting factors once per iteration. */
int bem_refine_solve(bem_ctx* ctx, int dtype_hi, const void* A_hi, const void* LU_lo, const int32_t* piv,
                     const void* dinv, int64_t n, int64_t lda, const void* b, void* x, double tol, int maxit,
                     int* iters, double* relres, void* stream);

/* GMRES-based refinement: restarted GMRES(restart) in FP64 on A_hi x = b,
 * right-preconditioned by the low-precision factors of bem_refine_solve
 * (tile-pivoted when dinv != NULL, else partial pivoting), Arnoldi with
 * classical Gram-Schmidt applied twice.  For systems where plain refinement
 * contracts too slowly (cond(A) times the FP32 unit roundoff near 1).  x
 * (device, FP64) holds the initial guess and is overwritten.  Each restart
 * begins from the true FP64 residual; once a restart cycle no longer halves
 * it, a relative residual <= accept ends the iteration with BEM_OK.  Returns
 * BEM_ERR_NOCONVERGE after maxit Arnoldi steps otherwise.  Synchronises the
 * stream once per Arnoldi step.  The reference solves with
 * torch.linalg.solve / lstsq (BEM_manager.py:1049-1056); this is the
 * fallback the driver takes when refinement stagnates. */
int bem_gmres_ir(bem_ctx* ctx, int dtype_hi, const void* A_hi, const void* LU_lo, const int32_t* piv,
                 const void* dinv, int64_t n, int64_t lda, const void* b, void* x, double tol, int maxit, int restart,
                 double accept, int* iters, double* relres, void* stream);

/* ---- least squares of the transmission system ------------------------------------
 * The reference solves the stacked system [A; P+_i] x = rhs (2n rows) with
 * torch.linalg.lstsq (BEM_manager.py:1039-1050).  Here: the column-equilibrated
 * normal equations N z = g, N = D (A^H A + P^H P) D, x = D z, with D the
 * power-of-two column scaling of [A; P].
 *
 * Normal matrix (the Gram half of that lstsq call): colscale (device [n]
 * doubles) receives D; out (n x n, ldo; BEM_C64 / BEM_C128 for complex,
 * BEM_F32 / BEM_F64 for real input) receives the full Hermitian N.
 * A, P: BEM_C128 (16-byte aligned) or BEM_F64, n x n, ld.  method
 * BEM_PREC_MIXED forms N on the tcgen05 tensor cores from FP16 hi/lo splits
 * of the scaled columns (about 22 significant bits per product, TMEM sums of
 * one 64-wide K stage folded into FP64; the split operands use a context
 * workspace of 8 n^2 bytes); BEM_PREC_FP64 forms it in FP64 on the FP64
 * tensor cores (DMMA).  Queued without synchronising; a tensor-core wait
 * that runs out is reported by the next bem_lstsq_refine. */
int bem_gram(bem_ctx* ctx, int dtype, const void* A, const void* P, int64_t n, int64_t ld, double* colscale,
             int method, int out_dtype, void* out, int64_t ldo, void* stream);
/* Cholesky factor of a Hermitian positive definite A = L L^H (the factor half
 * of the lstsq call, BEM_manager.py:1049, applied to the normal matrix of
 * bem_gram), in place, left in the tile-LU form of bem_lu_factor_tiled
 * (unit lower L D^{-1} below the diagonal, U = D L^H on and above it,
 * identity tile pivots in piv, explicit inverses of the 64 x 64 diagonal
 * tiles in dinv, bem_lu_dinv_elems(n) elements), so bem_lu_solve_tiled,
 * bem_refine_solve and bem_lstsq_refine take it.  A: BEM_C128 or BEM_F64 (the
 * lower triangle is read).  Panels of 1024 columns (BEM_TUNE_CHOL_NB) in FP64
 * on the FP64 tensor cores (DMMA); the trailing Hermitian updates on the FP64 tensor
 * cores (method BEM_PREC_FP64) or on tcgen05 from FP16 hi/lo splits of the
 * panel with FP64 sums subtracted from the FP64 Schur complement
 * (BEM_PREC_MIXED).  info: device int32, 0 or 1 + the first column whose
 * pivot was not positive.  Queued without synchronising. */
int bem_chol_factor(bem_ctx* ctx, int dtype, void* A, int64_t n, int64_t lda, int method, int32_t* piv, void* dinv,
                    int32_t* info, void* stream);
/* C += alpha op(A) op(B) in FP64 on the FP64 tensor cores (DMMA), dtype
 * BEM_F64 or BEM_C128, row-major: op(A) = A (m x k, lda) or, with conj_a, A^H
 * (A stored k x m); op(B) = B (k x n, ldb) or, with conj_b, B^H (B stored
 * n x k).  tri: bit 0 declares op(A) lower triangular, bit 1 op(B) upper
 * triangular: each 64-wide tile's K range then ends with the diagonal tile,
 * so entries beyond the diagonal must be zero within the diagonal tiles and
 * are not read beyond them.  Products with few output tiles split K (FP64 atomic
 * sums, so the last bits depend on the order).  The matrix products of the reference's
 * operator-norm analysis (compute_inv_norm, BEM_manager.py:874-920: the
 * scaled operator L^{-1} A L^{-H}) and of the Krylov estimators that replace
 * its SVD.  Queued without synchronising. */
int bem_gemm(bem_ctx* ctx, int dtype, int conj_a, int conj_b, int tri, int64_t m, int64_t n, int64_t k,
             double alpha, const void* A, int64_t lda, const void* B, int64_t ldb, void* C, int64_t ldc,
             void* stream);
/* X = L^{-1} with A = L L^H (the torch.linalg.inv(torch.linalg.cholesky(MV))
 * of compute_inv_norm, BEM_manager.py:885-899): the FP64 Cholesky of A in
 * place (L in the lower triangle; the upper triangle is left as it was),
 * then the lower-triangular inverse into X (n x n, ldx; zero above the
 * diagonal), both on the FP64 tensor cores.  A, X: BEM_F64 or BEM_C128.
 * info: device int32, 0 or 1 + the first column whose pivot was not
 * positive (X is then not valid).  Queued without synchronising. */
int bem_chol_inverse(bem_ctx* ctx, int dtype, void* A, int64_t n, int64_t lda, void* X, int64_t ldx, int32_t* info,
                     void* stream);
/* The solve half of the same lstsq call (BEM_manager.py:1049): x (device, n,
 * FP64 real or complex, holding the initial guess) is refined by flexible
 * GMRES(restart) in FP64 on the scaled normal equations, with FP64 products
 * against A and P and preconditioned by the tile-pivoted factors (LU, piv,
 * dinv of bem_lu_factor_tiled, dtype lu_dtype, leading dimension ldlu) of the
 * normal matrix from bem_gram.  b: device [2n] (the stacked right-hand side).
 * Stops at relative normal-equation residual tol, or, once a restart cycle no
 * longer halves it, at <= accept.  iters, relres: host pointers (may be NULL).
 * Synchronises the stream once per Arnoldi step. */
int bem_lstsq_refine(bem_ctx* ctx, int dtype, const void* A, const void* P, int64_t n, int64_t ld,
                     const double* colscale, int lu_dtype, const void* LU, int64_t ldlu, const int32_t* piv,
                     const void* dinv, const void* b, void* x, double tol, int maxit, int restart, double accept,
                     int* iters, double* relres, void* stream);
/* The same iteration for a normal-equation right-hand side (no reference
 * counterpart; the adjoint solve of the k-derivative of that lstsq):
 * (A^H A + P^H P) x = g, g: device [n]. */
int bem_normal_refine(bem_ctx* ctx, int dtype, const void* A, const void* P, int64_t n, int64_t ld,
                      const double* colscale, int lu_dtype, const void* LU, int64_t ldlu, const int32_t* piv,
                      const void* dinv, const void* g, void* x, double tol, int maxit, int restart, double accept,
                      int* iters, double* relres, void* stream);

/* ---- post-processing (headless) ------------------------------------------------
 * The two kernels the reference runs at the end of BEMManager.run for its
 * GGUI window (BEM_manager.py:1028-1029), writing plain device buffers; there
 * is no window.  Both queue one launch without synchronising.
 *
 * BEMManager.compute_color (BEM_manager.py:527-587).  solved, exact [nv*n]
 * doubles per vertex (n = 1 real, 2 complex interleaved); vert_types [nv]
 * int32 (VertAttachType); show = BEMManager._show (-1 default, 0 Neumann,
 * 1 Dirichlet).  solved is shifted IN PLACE at the Dirichlet-to-be-solved
 * vertices (every vertex when show = 1) by mean(exact) - mean(solved) over
 * those vertices, as the reference does.  Writes the colours [nv*3] float
 * (r, g, b) of the solved, exact and difference values. */
int bem_compute_color(bem_ctx* ctx, int n, double* solved, const double* exact, const int32_t* vert_types, int show,
                      float* solved_color, float* exact_color, float* diff_color, void* stream);
/* BEMManager.set_mesh_instances (BEM_manager.py:589-606): the mesh's vertices
 * as [nv*3] float (z = 0 on a 2D mesh) into solved_vertices, moved by -2.2
 * along x into exact_vertices and by +2.2 into diff_vertices. */
int bem_set_mesh_instances(bem_ctx* ctx, float* solved_vertices, float* exact_vertices, float* diff_vertices,
                           void* stream);

/* ---- device probes ------------------------------------------------------------
 * No reference counterpart.  Measures the throughput of the pipes the assembly
 * kernels are bound by (they are neither HBM- nor tensor-core-bound):
 * out[0] = FP32 FMA TFLOP/s, out[1] = FP64 FMA TFLOP/s, out[2] = MUFU (rsqrt)
 * Gop/s.  Synchronous; allocates a small buffer. */
int bem_measure_peaks(bem_ctx* ctx, double* out, void* stream);
/* No reference counterpart.  *version = the binary architecture (major*10 +
 * minor, cudaFuncGetAttributes' binaryVersion) of this library's device code
 * as loaded on the current device: 100 for the sm_100a build.  Needs a GPU. */
int bem_binary_version(int* version);

#ifdef __cplusplus
}
#endif

#endif /* BEM_B200_H */
