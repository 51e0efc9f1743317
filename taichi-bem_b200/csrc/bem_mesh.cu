// Near-pair list of a triangle mesh, built on the device: every ordered panel
// pair (i, j) that shares at least one vertex index, with its relation
// (coincident, common edge, common vertex: get_panels_relation,
// src/managers/mesh_manager.py:538-573) and the parameter orders of the
// corrected Sauter-Schwab maps.  Entries are ordered by i, then j, both
// ascending.
//
//   vertex_degree_kernel   incidences per vertex (atomics)
//   scan_kernel            exclusive prefix sums (one CTA walking the array)
//   vertex_fill_kernel     vertex -> panel adjacency lists (CSR)
//   near_pairs_kernel      per panel i, the union of its three vertices'
//                          lists taken in ascending order (repeated minimum
//                          above the last one taken): first the count, then,
//                          at the scanned offsets, the entries
//
// Work is O(sum over panels of (distinct neighbours x incident list
// lengths)), about 13 x 18 list reads per panel on a regular triangulation.
#include <climits>

#include "bem_internal.cuh"

namespace {

constexpr int NL_THREADS = 256;

// Parameter orders of a near pair for the corrected maps (packed 2 bits per
// slot): the shared vertex at slot 0 of both panels, or the shared edge at
// slots (0, 1) of both panels with matching endpoints.
__device__ int near_perm(const int32_t* a, const int32_t* b, int rel) {
    int px[3] = {0, 1, 2}, py[3] = {0, 1, 2};
    if (rel == REL_VERTEX) {
        bool done = false;
        for (int s = 0; s < 3 && !done; ++s)
            for (int t = 0; t < 3 && !done; ++t)
                if (a[s] == b[t]) {
                    px[0] = s; px[1] = (s + 1) % 3; px[2] = (s + 2) % 3;
                    py[0] = t; py[1] = (t + 1) % 3; py[2] = (t + 2) % 3;
                    done = true;
                }
    } else if (rel == REL_EDGE) {
        for (int s = 0; s < 3; ++s) {
            const int v0 = a[s], v1 = a[(s + 1) % 3];
            int t0 = -1, t1 = -1;
            for (int t = 0; t < 3; ++t) {
                if (b[t] == v0) t0 = t;
                if (b[t] == v1) t1 = t;
            }
            if (t0 >= 0 && t1 >= 0) {
                px[0] = s; px[1] = (s + 1) % 3; px[2] = (s + 2) % 3;
                py[0] = t0; py[1] = t1; py[2] = 3 - t0 - t1;
                break;
            }
        }
    }
    const int bx = px[0] | (px[1] << 2) | (px[2] << 4);
    const int by = py[0] | (py[1] << 2) | (py[2] << 4);
    return bx | (by << 6);
}

__global__ void vertex_degree_kernel(const int32_t* __restrict__ tris, int64_t n_inc, int32_t* __restrict__ deg) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e < n_inc) atomicAdd(&deg[tris[e]], 1);
}

// off[0..n] = exclusive prefix sums of cnt[0..n) (off[n] = the total), one
// CTA of 1024 threads, 1024 values per pass
__global__ void __launch_bounds__(1024) scan_kernel(const int32_t* __restrict__ cnt, int64_t n,
                                                    int64_t* __restrict__ off) {
    __shared__ int64_t s_warp[32];
    __shared__ int64_t s_carry;
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    if (tid == 0) s_carry = 0;
    __syncthreads();
    for (int64_t base = 0; base < n; base += 1024) {
        const int64_t i = base + tid;
        const int64_t v = i < n ? cnt[i] : 0;
        int64_t x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int64_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) s_warp[w] = x;
        __syncthreads();
        if (w == 0) {
            int64_t t = s_warp[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int64_t y = __shfl_up_sync(0xffffffffu, t, o);
                if (lane >= o) t += y;
            }
            s_warp[lane] = t;
        }
        __syncthreads();
        const int64_t excl = s_carry + (w ? s_warp[w - 1] : 0) + x - v;
        if (i < n) off[i] = excl;
        __syncthreads();
        if (tid == 1023) s_carry = excl + v;
        __syncthreads();
    }
    if (tid == 0) off[n] = s_carry;
}

__global__ void vertex_fill_kernel(const int32_t* __restrict__ tris, int64_t n_inc, const int64_t* __restrict__ voff,
                                   int32_t* __restrict__ cursor, int32_t* __restrict__ adj) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n_inc) return;
    const int v = tris[e];
    const int slot = atomicAdd(&cursor[v], 1);
    adj[voff[v] + slot] = (int32_t)(e / 3);
}

template <bool WRITE>
__global__ void near_pairs_kernel(const int32_t* __restrict__ tris, int nt, const int64_t* __restrict__ voff,
                                  const int32_t* __restrict__ adj, int32_t* __restrict__ cnt,
                                  const int64_t* __restrict__ poff, int4* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nt) return;
    const int32_t ti[3] = {tris[3 * i], tris[3 * i + 1], tris[3 * i + 2]};
    int64_t b[3], e[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        b[c] = voff[ti[c]];
        e[c] = voff[ti[c] + 1];
    }
    int cur = -1, count = 0;
    const int64_t o = WRITE ? poff[i] : 0;
    for (;;) {
        int nxt = INT_MAX;
#pragma unroll
        for (int c = 0; c < 3; ++c)
            for (int64_t q = b[c]; q < e[c]; ++q) {
                const int j = adj[q];
                if (j > cur && j < nxt) nxt = j;
            }
        if (nxt == INT_MAX) break;
        cur = nxt;
        const int32_t tj[3] = {tris[3 * nxt], tris[3 * nxt + 1], tris[3 * nxt + 2]};
        const int rel = bem_relation(ti, tj, i == nxt);
        if (rel == REL_SEPARATE) continue;
        if (WRITE) out[o + count] = make_int4(i, nxt, rel, near_perm(ti, tj, rel));
        ++count;
    }
    if (!WRITE) cnt[i] = count;
}

}  // namespace

int bem_build_near_list(bem_ctx* ctx, int nv, int nt) {
    const int64_t n_inc = 3LL * nt;
    // scratch: deg/cursor (nv), voff (nv + 1), adj (3 nt), cnt (nt), poff (nt + 1)
    const size_t bytes = sizeof(int32_t) * (2 * (size_t)nv + 3 * (size_t)nt + (size_t)nt) +
                         sizeof(int64_t) * ((size_t)nv + 1 + (size_t)nt + 1);
    char* ws = nullptr;
    if (int rc = bem_check_cuda(ctx, cudaMalloc((void**)&ws, bytes), "near list scratch")) return rc;
    int64_t* voff = reinterpret_cast<int64_t*>(ws);
    int64_t* poff = voff + nv + 1;
    int32_t* deg = reinterpret_cast<int32_t*>(poff + nt + 1);
    int32_t* cursor = deg + nv;
    int32_t* adj = cursor + nv;
    int32_t* cnt = adj + n_inc;
    int rc = bem_check_cuda(ctx, cudaMemset(deg, 0, sizeof(int32_t) * 2 * (size_t)nv), "near list zero");
    const unsigned gi = (unsigned)((n_inc + NL_THREADS - 1) / NL_THREADS);
    const unsigned gp = (unsigned)((nt + NL_THREADS - 1) / NL_THREADS);
    if (!rc) {
        vertex_degree_kernel<<<gi, NL_THREADS>>>(ctx->tris, n_inc, deg);
        scan_kernel<<<1, 1024>>>(deg, nv, voff);
        vertex_fill_kernel<<<gi, NL_THREADS>>>(ctx->tris, n_inc, voff, cursor, adj);
        near_pairs_kernel<false><<<gp, NL_THREADS>>>(ctx->tris, nt, voff, adj, cnt, nullptr, nullptr);
        scan_kernel<<<1, 1024>>>(cnt, nt, poff);
        ctx->launches += 5;
        rc = bem_check_cuda(ctx, cudaGetLastError(), "near list count");
    }
    int64_t total = 0;
    if (!rc) rc = bem_check_cuda(ctx, cudaMemcpy(&total, poff + nt, sizeof(int64_t), cudaMemcpyDeviceToHost),
                                 "near list total");
    if (!rc && total > 0) {
        rc = bem_check_cuda(ctx, cudaMalloc((void**)&ctx->near, sizeof(int4) * (size_t)total), "near list");
        if (!rc) {
            near_pairs_kernel<true><<<gp, NL_THREADS>>>(ctx->tris, nt, voff, adj, nullptr, poff, ctx->near);
            ctx->launches++;
            rc = bem_check_cuda(ctx, cudaGetLastError(), "near list write");
        }
    }
    if (!rc) ctx->n_near = total;
    cudaFree(ws);
    return rc;
}
