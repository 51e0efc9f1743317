// C ABI entry points: context, mesh upload + near-pair list, assembly dispatch.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "bem_internal.cuh"

int bem_fail(bem_ctx* ctx, int code, const std::string& msg) {
    if (ctx) ctx->err = msg;
    return code;
}

int bem_check_cuda(bem_ctx* ctx, cudaError_t e, const char* what) {
    if (e == cudaSuccess) return BEM_OK;
    cudaGetLastError();  // clear a non-sticky launch error so later calls start clean
    return bem_fail(ctx, BEM_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

int bem_take_factor_error(bem_ctx* ctx, int32_t value, cudaStream_t s) {
    if (value == 0) return BEM_OK;
    cudaMemsetAsync(ctx->flags + 4, 0, sizeof(int32_t), s);
    return bem_fail(ctx, BEM_ERR_TIMEOUT, "tiled lu: a tensor-core wait of the factorisation hit its iteration cap");
}

int bem_ws_reserve(bem_ctx* ctx, size_t bytes) {
    if (bytes <= ctx->ws_bytes) return BEM_OK;
    if (ctx->ws) cudaFree(ctx->ws);
    ctx->ws = nullptr;
    ctx->ws_bytes = 0;
    if (int rc = bem_check_cuda(ctx, cudaMalloc(&ctx->ws, bytes), "cudaMalloc(workspace)")) return rc;
    ctx->ws_bytes = bytes;
    return BEM_OK;
}

namespace {

// Gauss-Legendre rule on [0,1] (the reference's tables in
// src/BEM_functions/utils/functions.py:5-85 are this rule to 16 digits),
// computed by Newton iteration on the three-term Legendre recurrence.
void gauss01(int n, double* p, double* w) {
    if (n == 1) {
        p[0] = 0.5;
        w[0] = 1.0;
        return;
    }
    for (int i = 0; i < n; ++i) {
        double x = std::cos(BEM_PI * (i + 0.75) / (n + 0.5));
        for (int it = 0; it < 100; ++it) {
            double p0 = 1.0, p1 = x;
            for (int k = 2; k <= n; ++k) {
                double p2 = ((2.0 * k - 1.0) * x * p1 - (k - 1.0) * p0) / k;
                p0 = p1;
                p1 = p2;
            }
            double dp = n * (x * p1 - p0) / (x * x - 1.0);
            double dx = p1 / dp;
            x -= dx;
            if (std::fabs(dx) < 1e-16) break;
        }
        double p0 = 1.0, p1 = x;
        for (int k = 2; k <= n; ++k) {
            double p2 = ((2.0 * k - 1.0) * x * p1 - (k - 1.0) * p0) / k;
            p0 = p1;
            p1 = p2;
        }
        double dp = n * (x * p1 - p0) / (x * x - 1.0);
        p[n - 1 - i] = (x + 1.0) / 2.0;
        w[n - 1 - i] = 1.0 / ((1.0 - x * x) * dp * dp);
    }
}

void free_mesh(bem_ctx* ctx) {
    void* ptrs[] = {ctx->verts, ctx->tris, ctx->area, ctx->normal, ctx->centroid, ctx->curl, ctx->pts64,
                    ctx->pts32, ctx->phi64, ctx->phi32, ctx->gp, ctx->gw, ctx->near, ctx->test_local,
                    ctx->trial_local, ctx->seg2, ctx->nrm2};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    ctx->verts = nullptr; ctx->tris = nullptr; ctx->area = nullptr; ctx->normal = nullptr;
    ctx->centroid = nullptr; ctx->curl = nullptr; ctx->pts64 = nullptr; ctx->pts32 = nullptr;
    ctx->phi64 = nullptr; ctx->phi32 = nullptr; ctx->gp = nullptr; ctx->gw = nullptr; ctx->near = nullptr;
    ctx->test_local = nullptr; ctx->trial_local = nullptr; ctx->seg2 = nullptr; ctx->nrm2 = nullptr;
    ctx->nv = ctx->nt = ctx->Q = ctx->Q2 = 0;
    ctx->dim = 3;
    ctx->n_near = 0;
}

template <typename T>
int dmalloc(bem_ctx* ctx, T** p, size_t n) {
    return bem_check_cuda(ctx, cudaMalloc((void**)p, sizeof(T) * std::max<size_t>(n, 1)), "cudaMalloc(mesh)");
}

int check_space(bem_ctx* ctx, const bem_space* sp, const char* name) {
    if (!sp) return bem_fail(ctx, BEM_ERR_INVALID, std::string(name) + " space is NULL");
    if (sp->n_panels < 0 || (sp->n_panels > 0 && (!sp->panels || !sp->dof)))
        return bem_fail(ctx, BEM_ERR_INVALID, std::string(name) + " space has no panel/dof arrays");
    if (ctx->dim == 3 && sp->nb != 1 && sp->nb != 3)
        return bem_fail(ctx, BEM_ERR_INVALID, std::string(name) + " nb must be 1 or 3");
    if (ctx->dim == 2 && sp->nb != 1 && sp->nb != 2)
        return bem_fail(ctx, BEM_ERR_INVALID, std::string(name) + " nb must be 1 or 2 on a 2D mesh");
    if (sp->n_panels > ctx->nt) return bem_fail(ctx, BEM_ERR_INVALID, std::string(name) + " has more panels than the mesh");
    return BEM_OK;
}

// allow_dk: the caller takes the k-derivative operators (deriv_k, 3D Helmholtz)
int check_op(bem_ctx* ctx, const bem_op_desc* op, bool allow_dk = false) {
    if (!op) return bem_fail(ctx, BEM_ERR_INVALID, "op is NULL");
    if (op->deriv_k) {
        if (!allow_dk) return bem_fail(ctx, BEM_ERR_INVALID, "deriv_k is taken by bem_assemble and bem_apply only");
        if (op->kernel != BEM_KERNEL_HELMHOLTZ || ctx->dim != 3)
            return bem_fail(ctx, BEM_ERR_INVALID, "deriv_k needs the 3D Helmholtz kernel");
    }
    if (op->op < BEM_OP_V || op->op > BEM_OP_W) return bem_fail(ctx, BEM_ERR_INVALID, "unknown operator");
    if (op->kernel != BEM_KERNEL_LAPLACE && op->kernel != BEM_KERNEL_HELMHOLTZ)
        return bem_fail(ctx, BEM_ERR_INVALID, "unknown kernel");
    if (op->precision != BEM_PREC_FP64 && op->precision != BEM_PREC_MIXED)
        return bem_fail(ctx, BEM_ERR_INVALID, "unknown precision");
    if (!std::isfinite(op->k) || !std::isfinite(op->k2)) return bem_fail(ctx, BEM_ERR_INVALID, "non-finite wavenumber");
    return BEM_OK;
}

}  // namespace

int bem_lookahead_stream(bem_ctx* ctx) {
    if (ctx->aux) return BEM_OK;
    int least = 0, greatest = 0;
    if (int rc = bem_check_cuda(ctx, cudaDeviceGetStreamPriorityRange(&least, &greatest), "stream priorities"))
        return rc;
    if (int rc = bem_check_cuda(ctx, cudaStreamCreateWithPriority(&ctx->aux, cudaStreamNonBlocking, greatest),
                                "side stream"))
        return rc;
    if (int rc = bem_check_cuda(ctx, cudaEventCreateWithFlags(&ctx->ev_next, cudaEventDisableTiming), "event"))
        return rc;
    return bem_check_cuda(ctx, cudaEventCreateWithFlags(&ctx->ev_diag, cudaEventDisableTiming), "event");
}

extern "C" {

int bem_ctx_set_tuning(bem_ctx* ctx, int key, int value) {
    if (!ctx) return BEM_ERR_INVALID;
    if (key < 0 || key >= BEM_TUNE_KEYS) return bem_fail(ctx, BEM_ERR_INVALID, "set_tuning: unknown key");
    if (key == BEM_TUNE_CALDERON_GROUP && (value < 0 || value > 5))
        return bem_fail(ctx, BEM_ERR_INVALID, "set_tuning: calderon form must be in 1..5");
    if (key == BEM_TUNE_GRAM_PAIR && (value < 0 || value > 3))
        return bem_fail(ctx, BEM_ERR_INVALID, "set_tuning: normal-matrix form must be 1, 2 or 3");
    if (key == BEM_TUNE_LU_UPDATE && (value < 0 || value > 2))
        return bem_fail(ctx, BEM_ERR_INVALID, "set_tuning: LU update form must be 1 or 2");
    if (key == BEM_TUNE_KBATCH_GROUP && value != 0 && value != 2 && value != 4)
        return bem_fail(ctx, BEM_ERR_INVALID, "set_tuning: wavenumbers per batched launch must be 2 or 4");
    if (key == BEM_TUNE_GRAM_KSEG && value < 0) return bem_fail(ctx, BEM_ERR_INVALID, "set_tuning: negative segment");
    if (key == BEM_TUNE_GRAM_BAND && (value < 0 || value > 4096))
        return bem_fail(ctx, BEM_ERR_INVALID, "set_tuning: band width must be in 0..4096");
    if (key == BEM_TUNE_CHOL_NB && (value < 0 || value % 64 != 0 || value > 4096))
        return bem_fail(ctx, BEM_ERR_INVALID, "set_tuning: panel width must be a multiple of 64 up to 4096");
    ctx->tune[key] = value;
    return BEM_OK;
}

int bem_ctx_create(bem_ctx** out_ctx) {
    if (!out_ctx) return BEM_ERR_INVALID;
    *out_ctx = nullptr;
    bem_ctx* ctx = new (std::nothrow) bem_ctx();
    if (!ctx) return BEM_ERR_INVALID;
    if (cudaGetDevice(&ctx->device) != cudaSuccess) {
        delete ctx;
        return BEM_ERR_CUDA;
    }
    cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, ctx->device);
    if (cudaMalloc((void**)&ctx->flags, 16 * sizeof(int32_t)) != cudaSuccess) {
        delete ctx;
        return BEM_ERR_CUDA;
    }
    cudaMemset(ctx->flags, 0, 16 * sizeof(int32_t));
    *out_ctx = ctx;
    return BEM_OK;
}

int bem_ctx_destroy(bem_ctx* ctx) {
    if (!ctx) return BEM_OK;
    free_mesh(ctx);
    if (ctx->ev_next) cudaEventDestroy(ctx->ev_next);
    if (ctx->ev_diag) cudaEventDestroy(ctx->ev_diag);
    if (ctx->aux) cudaStreamDestroy(ctx->aux);
    if (ctx->ws) cudaFree(ctx->ws);
    if (ctx->big_ws) cudaFree(ctx->big_ws);
    if (ctx->flags) cudaFree(ctx->flags);
    delete ctx;
    return BEM_OK;
}

const char* bem_last_error(const bem_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int64_t bem_launch_count(const bem_ctx* ctx) { return ctx ? ctx->launches : 0; }

int64_t bem_near_pair_count(const bem_ctx* ctx) { return ctx ? ctx->n_near : 0; }

int bem_near_pair_list(const bem_ctx* cctx, int32_t* out) {
    bem_ctx* ctx = const_cast<bem_ctx*>(cctx);
    if (!ctx) return BEM_ERR_INVALID;
    if (!out) return bem_fail(ctx, BEM_ERR_INVALID, "near_pair_list: out is NULL");
    if (ctx->n_near == 0 || ctx->dim != 3) return BEM_OK;
    return bem_check_cuda(ctx, cudaMemcpy(out, ctx->near, sizeof(int4) * (size_t)ctx->n_near, cudaMemcpyDefault),
                          "near_pair_list copy");
}

int bem_mesh_set(bem_ctx* ctx, const double* verts, const int32_t* tris, int nv, int nt, int gauss_qr) {
    if (!ctx) return BEM_ERR_INVALID;
    if (!verts || !tris || nv <= 0 || nt <= 0) return bem_fail(ctx, BEM_ERR_INVALID, "empty mesh");
    if (gauss_qr < 1 || gauss_qr > BEM_MAX_Q) return bem_fail(ctx, BEM_ERR_INVALID, "GaussQR must be in 1..12");
    for (int64_t i = 0; i < 3LL * nv; ++i)
        if (!std::isfinite(verts[i])) return bem_fail(ctx, BEM_ERR_MESH, "non-finite vertex coordinate");
    for (int64_t i = 0; i < 3LL * nt; ++i)
        if (tris[i] < 0 || tris[i] >= nv) return bem_fail(ctx, BEM_ERR_MESH, "panel vertex index out of range");

    free_mesh(ctx);
    const int Q = gauss_qr, Q2 = Q * Q;
    std::vector<double> gp(Q), gw(Q);
    gauss01(Q, gp.data(), gw.data());
    // FP32 separate rule: reference weights (gw_x gw_y r1, rounded once to
    // float, as geometry_kernel does) rescaled to the exact weight sum
    double wsum = 0.0, wsum32 = 0.0;
    for (int ix = 0; ix < Q; ++ix)
        for (int iy = 0; iy < Q; ++iy) {
            const double wref = (gw[ix] * gw[iy]) * gp[ix];
            wsum += wref;
            wsum32 += (double)(float)wref;
        }
    std::vector<double> phi64((size_t)Q2 * 3);
    std::vector<float> phi32((size_t)Q2 * 3);
    for (int ix = 0; ix < Q; ++ix)
        for (int iy = 0; iy < Q; ++iy) {
            double r1 = gp[ix], r2 = gp[iy] * r1;
            double v[3] = {1.0 - r1, r1 - r2, r2};
            for (int b = 0; b < 3; ++b) {
                phi64[(ix * Q + iy) * 3 + b] = v[b];
                phi32[(ix * Q + iy) * 3 + b] = (float)v[b];
            }
        }
    int rc = 0;
    if ((rc = dmalloc(ctx, &ctx->verts, 3 * (size_t)nv)) || (rc = dmalloc(ctx, &ctx->tris, 3 * (size_t)nt)) ||
        (rc = dmalloc(ctx, &ctx->area, nt)) || (rc = dmalloc(ctx, &ctx->normal, 3 * (size_t)nt)) ||
        (rc = dmalloc(ctx, &ctx->centroid, 3 * (size_t)nt)) || (rc = dmalloc(ctx, &ctx->curl, 9 * (size_t)nt)) ||
        (rc = dmalloc(ctx, &ctx->pts64, (size_t)nt * Q2)) || (rc = dmalloc(ctx, &ctx->pts32, (size_t)nt * Q2)) ||
        (rc = dmalloc(ctx, &ctx->phi64, (size_t)Q2 * 3)) || (rc = dmalloc(ctx, &ctx->phi32, (size_t)Q2 * 3)) ||
        (rc = dmalloc(ctx, &ctx->gp, Q)) || (rc = dmalloc(ctx, &ctx->gw, Q)) ||
        (rc = dmalloc(ctx, &ctx->test_local, nt)) || (rc = dmalloc(ctx, &ctx->trial_local, nt))) {
        free_mesh(ctx);
        return rc;
    }
    ctx->nv = nv;
    ctx->nt = nt;
    ctx->Q = Q;
    ctx->Q2 = Q2;
    ctx->wcorr32 = (wsum / wsum32) * (wsum / wsum32);
    double rho = 0.0;
    for (int t = 0; t < nt; ++t) {
        double c[3] = {0.0, 0.0, 0.0};
        for (int a = 0; a < 3; ++a)
            for (int d = 0; d < 3; ++d) c[d] += verts[3 * tris[3 * t + a] + d] / 3.0;
        for (int a = 0; a < 3; ++a) {
            double q = 0.0;
            for (int d = 0; d < 3; ++d) {
                const double e = verts[3 * tris[3 * t + a] + d] - c[d];
                q += e * e;
            }
            rho = std::max(rho, std::sqrt(q));
        }
    }
    ctx->rho_max = rho;
    cudaMemcpy(ctx->verts, verts, sizeof(double) * 3 * nv, cudaMemcpyHostToDevice);
    cudaMemcpy(ctx->tris, tris, sizeof(int32_t) * 3 * nt, cudaMemcpyHostToDevice);
    cudaMemcpy(ctx->gp, gp.data(), sizeof(double) * Q, cudaMemcpyHostToDevice);
    cudaMemcpy(ctx->gw, gw.data(), sizeof(double) * Q, cudaMemcpyHostToDevice);
    cudaMemcpy(ctx->phi64, phi64.data(), sizeof(double) * Q2 * 3, cudaMemcpyHostToDevice);
    cudaMemcpy(ctx->phi32, phi32.data(), sizeof(float) * Q2 * 3, cudaMemcpyHostToDevice);
    // near-pair list: every ordered pair sharing at least one vertex index (on the device)
    if ((rc = bem_build_near_list(ctx, nv, nt))) {
        free_mesh(ctx);
        return rc;
    }
    cudaMemset(ctx->flags, 0, 16 * sizeof(int32_t));
    if ((rc = bem_launch_geometry(ctx, 0))) return rc;
    if ((rc = bem_check_cuda(ctx, cudaDeviceSynchronize(), "mesh geometry"))) return rc;
    int32_t flags[16];
    cudaMemcpy(flags, ctx->flags, sizeof(flags), cudaMemcpyDeviceToHost);
    if (flags[0] != 0) {
        int bad = flags[0] - 1;
        free_mesh(ctx);
        return bem_fail(ctx, BEM_ERR_MESH, "degenerate panel " + std::to_string(bad) + " (zero or non-finite area)");
    }
    return BEM_OK;
}

int bem_mesh_set_2d(bem_ctx* ctx, const double* verts, const int32_t* segs, int nv, int nt, int gauss_qr) {
    if (!ctx) return BEM_ERR_INVALID;
    if (!verts || !segs || nv <= 0 || nt <= 0) return bem_fail(ctx, BEM_ERR_INVALID, "empty mesh");
    if (gauss_qr < 1 || gauss_qr > BEM_MAX_Q) return bem_fail(ctx, BEM_ERR_INVALID, "GaussQR must be in 1..12");
    for (int64_t i = 0; i < 2LL * nv; ++i)
        if (!std::isfinite(verts[i])) return bem_fail(ctx, BEM_ERR_MESH, "non-finite vertex coordinate");
    for (int64_t i = 0; i < 2LL * nt; ++i)
        if (segs[i] < 0 || segs[i] >= nv) return bem_fail(ctx, BEM_ERR_MESH, "panel vertex index out of range");
    // length and normal (e.y, -e.x)/|e| of each segment, mesh_manager.py:108-113
    std::vector<double> len(nt), nrm(2 * (size_t)nt);
    std::vector<double4> seg(nt);
    for (int p = 0; p < nt; ++p) {
        const double* a = verts + 2 * segs[2 * p];
        const double* b = verts + 2 * segs[2 * p + 1];
        const double ex = b[0] - a[0], ey = b[1] - a[1];
        const double L = std::sqrt(ex * ex + ey * ey);
        if (!(L > 0.0) || !std::isfinite(L))
            return bem_fail(ctx, BEM_ERR_MESH, "degenerate panel " + std::to_string(p) + " (zero length)");
        len[p] = L;
        nrm[2 * p] = ey / L;
        nrm[2 * p + 1] = -ex / L;
        seg[p] = make_double4(a[0], a[1], b[0], b[1]);
    }
    // ordered pairs that the reference integrates with its coincide or
    // common-vertex branch (get_panels_relation, mesh_manager.py:539-551)
    std::vector<std::vector<int>> vp(nv);
    for (int p = 0; p < nt; ++p)
        for (int c = 0; c < 2; ++c) vp[segs[2 * p + c]].push_back(p);
    int64_t n_near = 0;
    std::vector<int> cand;
    for (int i = 0; i < nt; ++i) {
        cand.clear();
        for (int c = 0; c < 2; ++c)
            for (int j : vp[segs[2 * i + c]]) cand.push_back(j);
        std::sort(cand.begin(), cand.end());
        n_near += std::unique(cand.begin(), cand.end()) - cand.begin();
    }

    free_mesh(ctx);
    const int Q = gauss_qr;
    std::vector<double> gp(Q), gw(Q);
    gauss01(Q, gp.data(), gw.data());
    int rc = 0;
    if ((rc = dmalloc(ctx, &ctx->verts, 2 * (size_t)nv)) || (rc = dmalloc(ctx, &ctx->tris, 2 * (size_t)nt)) ||
        (rc = dmalloc(ctx, &ctx->area, nt)) || (rc = dmalloc(ctx, &ctx->normal, 2 * (size_t)nt)) ||
        (rc = dmalloc(ctx, &ctx->seg2, nt)) || (rc = dmalloc(ctx, &ctx->nrm2, nt)) ||
        (rc = dmalloc(ctx, &ctx->gp, Q)) || (rc = dmalloc(ctx, &ctx->gw, Q))) {
        free_mesh(ctx);
        return rc;
    }
    const cudaMemcpyKind h2d = cudaMemcpyHostToDevice;
    if ((rc = bem_check_cuda(ctx, cudaMemcpy(ctx->verts, verts, sizeof(double) * 2 * nv, h2d), "upload")) ||
        (rc = bem_check_cuda(ctx, cudaMemcpy(ctx->tris, segs, sizeof(int32_t) * 2 * nt, h2d), "upload")) ||
        (rc = bem_check_cuda(ctx, cudaMemcpy(ctx->area, len.data(), sizeof(double) * nt, h2d), "upload")) ||
        (rc = bem_check_cuda(ctx, cudaMemcpy(ctx->normal, nrm.data(), sizeof(double) * 2 * nt, h2d), "upload")) ||
        (rc = bem_check_cuda(ctx, cudaMemcpy(ctx->seg2, seg.data(), sizeof(double4) * nt, h2d), "upload")) ||
        (rc = bem_check_cuda(ctx, cudaMemcpy(ctx->nrm2, nrm.data(), sizeof(double2) * nt, h2d), "upload")) ||
        (rc = bem_check_cuda(ctx, cudaMemcpy(ctx->gp, gp.data(), sizeof(double) * Q, h2d), "upload")) ||
        (rc = bem_check_cuda(ctx, cudaMemcpy(ctx->gw, gw.data(), sizeof(double) * Q, h2d), "upload"))) {
        free_mesh(ctx);
        return rc;
    }
    cudaMemset(ctx->flags, 0, 16 * sizeof(int32_t));
    ctx->dim = 2;
    ctx->nv = nv;
    ctx->nt = nt;
    ctx->Q = Q;
    ctx->Q2 = Q * Q;
    ctx->n_near = n_near;
    return BEM_OK;
}

int bem_mesh_geometry(const bem_ctx* cctx, double* areas, double* normals, void* stream) {
    bem_ctx* ctx = const_cast<bem_ctx*>(cctx);
    if (!ctx) return BEM_ERR_INVALID;
    if (ctx->nt == 0) return bem_fail(ctx, BEM_ERR_NOMESH, "no mesh set");
    cudaStream_t s = (cudaStream_t)stream;
    if (areas)
        if (int rc = bem_check_cuda(ctx, cudaMemcpyAsync(areas, ctx->area, sizeof(double) * ctx->nt,
                                                          cudaMemcpyDeviceToDevice, s), "copy areas"))
            return rc;
    if (normals)
        if (int rc = bem_check_cuda(ctx, cudaMemcpyAsync(normals, ctx->normal, sizeof(double) * ctx->dim * ctx->nt,
                                                          cudaMemcpyDeviceToDevice, s), "copy normals"))
            return rc;
    return BEM_OK;
}

int bem_assemble(bem_ctx* ctx, const bem_op_desc* op, const bem_space* test, const bem_space* trial, int out_dtype,
                 void* out, int64_t ld, double scale, void* out_t, double scale_t, void* stream) {
    if (!ctx) return BEM_ERR_INVALID;
    if (ctx->nt == 0) return bem_fail(ctx, BEM_ERR_NOMESH, "no mesh set");
    if (int rc = check_op(ctx, op, true)) return rc;
    if (int rc = check_space(ctx, test, "test")) return rc;
    if (int rc = check_space(ctx, trial, "trial")) return rc;
    int want = op->kernel == BEM_KERNEL_HELMHOLTZ ? BEM_C128 : BEM_F64;
    if (out_dtype != want)
        return bem_fail(ctx, BEM_ERR_INVALID, "out dtype must be BEM_F64 for Laplace and BEM_C128 for Helmholtz");
    if (!out || ld <= 0) return bem_fail(ctx, BEM_ERR_INVALID, "out is NULL or ld <= 0");
    if (ctx->dim == 2)
        return bem_launch_assemble2d(ctx, op, test, trial, 0, out, ld, scale, out_t, scale_t, nullptr, nullptr, 0,
                                     (cudaStream_t)stream);
    return bem_launch_assemble(ctx, op, test, trial, 0, out, ld, scale, out_t, scale_t, nullptr, nullptr, 0,
                               (cudaStream_t)stream);
}

int bem_assemble_batch(bem_ctx* ctx, const bem_op_desc* op, const bem_space* test, const bem_space* trial,
                       int nk, const double* k, const double* k2, void* const* out, int64_t ld,
                       const double* scale, void* const* out_t, const double* scale_t, void* stream) {
    if (!ctx) return BEM_ERR_INVALID;
    if (ctx->nt == 0) return bem_fail(ctx, BEM_ERR_NOMESH, "no mesh set");
    if (int rc = check_op(ctx, op, true)) return rc;
    if (ctx->dim != 3 || op->kernel != BEM_KERNEL_HELMHOLTZ)
        return bem_fail(ctx, BEM_ERR_INVALID, "bem_assemble_batch takes the 3D Helmholtz kernel");
    if (int rc = check_space(ctx, test, "test")) return rc;
    if (int rc = check_space(ctx, trial, "trial")) return rc;
    if (nk < 1 || nk > BEM_MAX_KBATCH) return bem_fail(ctx, BEM_ERR_INVALID, "nk must be in [1, BEM_MAX_KBATCH]");
    if (!k || !k2 || !out || !scale || ld <= 0)
        return bem_fail(ctx, BEM_ERR_INVALID, "k, k2, out or scale is NULL, or ld <= 0");
    for (int w = 0; w < nk; ++w) {
        if (!std::isfinite(k[w]) || !std::isfinite(k2[w]) || !std::isfinite(scale[w]))
            return bem_fail(ctx, BEM_ERR_INVALID, "non-finite wavenumber or scale");
        if (!out[w]) return bem_fail(ctx, BEM_ERR_INVALID, "out[w] is NULL");
        if (out_t && out_t[w] && (!scale_t || !std::isfinite(scale_t[w])))
            return bem_fail(ctx, BEM_ERR_INVALID, "out_t[w] given without a finite scale_t[w]");
    }
    return bem_launch_assemble_batch(ctx, op, test, trial, nk, k, k2, out, ld, scale, out_t, scale_t,
                                     (cudaStream_t)stream);
}

int bem_apply(bem_ctx* ctx, const bem_op_desc* op, const bem_space* test, const bem_space* trial, int dtype,
              const void* x, void* y, double scale, int conj_x, void* stream) {
    if (!ctx) return BEM_ERR_INVALID;
    if (ctx->nt == 0) return bem_fail(ctx, BEM_ERR_NOMESH, "no mesh set");
    if (int rc = check_op(ctx, op, true)) return rc;
    if (int rc = check_space(ctx, test, "test")) return rc;
    if (int rc = check_space(ctx, trial, "trial")) return rc;
    int want = op->kernel == BEM_KERNEL_HELMHOLTZ ? BEM_C128 : BEM_F64;
    if (dtype != want)
        return bem_fail(ctx, BEM_ERR_INVALID, "x/y dtype must be BEM_F64 for Laplace and BEM_C128 for Helmholtz");
    if (!x || !y) return bem_fail(ctx, BEM_ERR_INVALID, "x or y is NULL");
    if (ctx->dim == 2)
        return bem_launch_assemble2d(ctx, op, test, trial, 1, nullptr, 0, scale, nullptr, 0.0, x, y, conj_x,
                                     (cudaStream_t)stream);
    return bem_launch_assemble(ctx, op, test, trial, 1, nullptr, 0, scale, nullptr, 0.0, x, y, conj_x,
                               (cudaStream_t)stream);
}

int bem_assemble_dirichlet(bem_ctx* ctx, const bem_op_desc* op, const bem_space* test, const bem_space* trial,
                           void* out, int64_t ld, double scale, const bem_space* rows, const bem_space* data,
                           const void* g, void* y, double scale_k, int conj_g, void* stream) {
    if (!ctx) return BEM_ERR_INVALID;
    if (ctx->nt == 0) return bem_fail(ctx, BEM_ERR_NOMESH, "no mesh set");
    if (int rc = check_op(ctx, op)) return rc;
    if (op->op != BEM_OP_V) return bem_fail(ctx, BEM_ERR_INVALID, "assemble_dirichlet: op must be BEM_OP_V");
    if (int rc = check_space(ctx, test, "test")) return rc;
    if (int rc = check_space(ctx, trial, "trial")) return rc;
    if (int rc = check_space(ctx, rows, "rows")) return rc;
    if (int rc = check_space(ctx, data, "data")) return rc;
    if (test->nb != 1 || trial->nb != 1 || rows->nb != 1)
        return bem_fail(ctx, BEM_ERR_INVALID, "assemble_dirichlet: V test/trial and rhs rows must be P0");
    if (rows->n_panels != test->n_panels || data->n_panels != trial->n_panels)
        return bem_fail(ctx, BEM_ERR_INVALID, "assemble_dirichlet: rows/data must run over the test/trial panels");
    if (!out || ld <= 0 || !g || !y) return bem_fail(ctx, BEM_ERR_INVALID, "assemble_dirichlet: NULL buffer");
    if (ctx->dim == 2) {
        // 2D: the V block and K g as two launches on the caller's stream
        if (int rc = bem_launch_assemble2d(ctx, op, test, trial, 0, out, ld, scale, nullptr, 0.0, nullptr, nullptr,
                                           0, (cudaStream_t)stream))
            return rc;
        bem_op_desc kop = *op;
        kop.op = BEM_OP_K;
        return bem_launch_assemble2d(ctx, &kop, rows, data, 1, nullptr, 0, scale_k, nullptr, 0.0, g, y, conj_g,
                                     (cudaStream_t)stream);
    }
    return bem_launch_dirichlet(ctx, op, test, trial, out, ld, scale, rows, data, g, y, scale_k, conj_g,
                                (cudaStream_t)stream);
}

int bem_mass(bem_ctx* ctx, const bem_space* test, const bem_space* trial, int dtype, void* out, int64_t ld,
             double scale, void* out_t, double scale_t, const void* x, void* y, int conj_x, void* stream) {
    if (!ctx) return BEM_ERR_INVALID;
    if (ctx->nt == 0) return bem_fail(ctx, BEM_ERR_NOMESH, "no mesh set");
    if (int rc = check_space(ctx, test, "test")) return rc;
    if (int rc = check_space(ctx, trial, "trial")) return rc;
    if (test->n_panels != trial->n_panels)
        return bem_fail(ctx, BEM_ERR_INVALID, "mass: test and trial must run over the same panel list");
    if (dtype != BEM_F64 && dtype != BEM_C128) return bem_fail(ctx, BEM_ERR_INVALID, "mass: dtype must be F64/C128");
    int mode = x ? 1 : 0;
    if (mode == 0 && (!out || ld <= 0)) return bem_fail(ctx, BEM_ERR_INVALID, "mass: out is NULL");
    if (mode == 1 && !y) return bem_fail(ctx, BEM_ERR_INVALID, "mass: y is NULL");
    if (ctx->dim == 2)
        return bem_launch_mass2d(ctx, test, trial, dtype == BEM_C128, mode, out, ld, scale, out_t, scale_t, x, y,
                                 conj_x, (cudaStream_t)stream);
    return bem_launch_mass(ctx, test, trial, dtype == BEM_C128, mode, out, ld, scale, out_t, scale_t, x, y, conj_x,
                           (cudaStream_t)stream);
}

int bem_adjoint_vertices(bem_ctx* ctx, const bem_op_desc* op, const bem_space* test, const bem_space* trial,
                         const double* lam, const double* u, double* grad, void* stream) {
    if (!ctx) return BEM_ERR_INVALID;
    if (ctx->nt == 0) return bem_fail(ctx, BEM_ERR_NOMESH, "no mesh set");
    if (!op || !lam || !u || !grad) return bem_fail(ctx, BEM_ERR_INVALID, "adjoint: null argument");
    if (ctx->dim != 3) return bem_fail(ctx, BEM_ERR_INVALID, "adjoint: triangle meshes only");
    if (op->kernel != BEM_KERNEL_LAPLACE || (op->op != BEM_OP_V && op->op != BEM_OP_K) || op->deriv_k)
        return bem_fail(ctx, BEM_ERR_INVALID, "adjoint: Laplace V or K only");
    if (int rc = check_space(ctx, test, "test")) return rc;
    if (int rc = check_space(ctx, trial, "trial")) return rc;
    if (test->nb != 1 || trial->nb != (op->op == BEM_OP_V ? 1 : 3))
        return bem_fail(ctx, BEM_ERR_INVALID, "adjoint: V needs P0 x P0 spaces, K a P0 test and a P1 trial space");
    return bem_launch_adjoint(ctx, op, test, trial, lam, u, grad, (cudaStream_t)stream);
}

}  // extern "C"
