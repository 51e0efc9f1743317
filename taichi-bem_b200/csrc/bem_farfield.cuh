// Device helpers shared by the far-field assembly kernels (bem_assembly.cu,
// bem_calderon.cu): the FP32 pair frame, r and 1/r with one Newton step, the
// sine/cosine of the Helmholtz phase, packed FP32x2 arithmetic and the block
// entry update.
#pragma once

#include "bem_internal.cuh"

namespace {

template <typename T>
struct V4T;
template <>
struct V4T<float> {
    using type = float4;
};
template <>
struct V4T<double> {
    using type = double4;
};

// r = |d| and 1/r from r2 = |d|^2.  In FP32 the MUFU reciprocal square root
// carries a deterministic error of up to ~1e-7 that varies slowly with r2, so
// every quadrature point of a pair (and every nearby pair) would share it: a
// relative error of r acts on e^{ikr} like a perturbation of k.  One Newton
// step whose residual 1 - r2 y0^2 is formed with a single rounding (FMA) leaves
// only the independent rounding errors of the products.
__device__ __forceinline__ void dev_r_rinv(float r2, float& r, float& rinv) {
    const float y0 = rsqrtf(r2);
    const float p = r2 * y0;
    const float e = fmaf(-p, y0, 1.0f);
    rinv = fmaf(0.5f * y0, e, y0);
    r = fmaf(0.5f * p, e, p);
}
__device__ __forceinline__ void dev_r_rinv(double r2, double& r, double& rinv) {
    rinv = rsqrt(r2);
    r = r2 * rinv;
}

// Pair frame of an FP32 separate pair.  With D = c_i - c_j (FP64 centroid
// difference) and e = x_a - y_b (centroid-relative point offsets, |e| at most
// the two panel diameters):
//   r^2 = R^2 + s,   s = e.(2D + e),   r - R = s / (r + R),   d.n = D.n + e.n,
// so each FP32 rounding is relative to a quantity of size |e| or to a per-pair
// constant, and none is shared by the quadrature points of a pair (rounding
// D - y_b once per trial point, say, would be shared by all test points and
// would not average out over the GaussQR^4 sum).  The Helmholtz factor is
//   e^{ikr} = e^{ikR} e^{ik(r-R)}:
// e^{ikR} is evaluated once per pair in FP64 and FP32 carries only the phase
// k (r - R) = O(k h), whose error no longer grows with k R.  In FP64
// (SPLIT = false) the kernels use d = x - y directly and the frame is inert.
//
// FP32 points carry the reference-triangle weights, identical on every panel;
// the pair factor pf = (2 A_i)(2 A_j) wcorr is applied in FP64, where wcorr =
// (W / W_f)^2 rescales the sum W_f of the FP32 weights to the exact sum W.  A
// rounding that differed per panel would scale whole rows of the far field
// against the FP64 near field and identity terms.
template <typename T, bool HELM>
struct Frame {
    static constexpr bool SPLIT = sizeof(T) == 4;
    T ux = T(0), uy = T(0), uz = T(0);  // 2D
    T R2 = T(0), Rf = T(0);
    double cR = 1.0, sR = 0.0, pf = 1.0;
    __device__ __forceinline__ void init(double dx, double dy, double dz, double k, double Ai, double Aj,
                                         double wcorr) {
        if (SPLIT) {
            pf = 4.0 * Ai * Aj * wcorr;
            ux = T(2.0 * dx);
            uy = T(2.0 * dy);
            uz = T(2.0 * dz);
            const double R2d = dx * dx + dy * dy + dz * dz;
            R2 = T(R2d);
            if (HELM) {
                const double R = sqrt(R2d);
                Rf = T(R);
                sincos(k * R, &sR, &cR);
            }
        }
    }
    // (re, im) <- (re, im) pf e^{ikR}
    __device__ __forceinline__ void rotate(double& re, double& im) const {
        if (SPLIT) {
            re *= pf;
            im *= pf;
        }
        if (SPLIT && HELM) {
            const double a = re * cR - im * sR, b = re * sR + im * cR;
            re = a;
            im = b;
        }
    }
};

// FP32 sine/cosine of the Helmholtz phase k r (k r >= 0 and moderate): Cody-
// Waite reduction by pi/2 with a two-term split of pi/2 (exact FMA products
// for |n| < 2^12), Taylor polynomials of sin (through y^9) and cos (through
// y^10) on |y| <= pi/4 (truncation below 3e-9), and the quadrant rotation.
// sin/cos polynomials on |y| <= pi/4
__device__ __forceinline__ void dev_sincos_poly(float y, float* s, float* c) {
    const float y2 = y * y;
    // sin y = y (1 - y^2/3! + y^4/5! - y^6/7! + y^8/9!)
    float ps = fmaf(y2, 2.75573192239858907e-06f, -1.98412698412698413e-04f);
    ps = fmaf(y2, ps, 8.33333333333333333e-03f);
    ps = fmaf(y2, ps, -1.66666666666666667e-01f);
    *s = fmaf(y * y2, ps, y);
    // cos y = 1 - y^2/2! + y^4/4! - y^6/6! + y^8/8! - y^10/10!
    float pc = fmaf(y2, -2.75573192239858907e-07f, 2.48015873015873016e-05f);
    pc = fmaf(y2, pc, -1.38888888888888889e-03f);
    pc = fmaf(y2, pc, 4.16666666666666667e-02f);
    pc = fmaf(y2, pc, -0.5f);
    *c = fmaf(y2, pc, 1.0f);
}
__device__ __forceinline__ void dev_sincos(float x, float* s, float* c) {
    const float kTwoOverPi = 0.636619772367581343f;
    const float kPio2Hi = 1.57079637050628662109375f;  // pi/2 rounded to float
    const float kPio2Lo = -4.37113900018624283e-08f;   // pi/2 - kPio2Hi
    const float fn = rintf(x * kTwoOverPi);
    const int q = (int)fn;
    float y = fmaf(-fn, kPio2Hi, x);
    y = fmaf(-fn, kPio2Lo, y);
    float sy, cy;
    dev_sincos_poly(y, &sy, &cy);
    float ss = (q & 1) ? cy : sy;
    float cc = (q & 1) ? sy : cy;
    *s = (q & 2) ? -ss : ss;
    *c = ((q + 1) & 2) ? -cc : cc;
}
// Split phase k (r - R): |k (r - R)| <= k |x_a - y_b - (c_i - c_j)| <= k (rho_i + rho_j)
// with rho the largest centroid-to-vertex distance; when the host has bounded
// that by pi/4 (`small`, uniform over the launch) the reduction is skipped.
__device__ __forceinline__ void dev_sincos_phase(float x, bool small, float* s, float* c) {
    if (small)
        dev_sincos_poly(x, s, c);
    else
        dev_sincos(x, s, c);
}
__device__ __forceinline__ void dev_sincos(double x, double* s, double* c) { sincos(x, s, c); }

struct cxd {
    double re, im;
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

constexpr int FAR_THREADS = 128;
constexpr int FAR_TI = 8;

template <bool CPLX>
__device__ __forceinline__ void add_entry(double* base, int64_t idx, double re, double im, bool atomic) {
    if (CPLX) {
        if (atomic) {
            atomicAdd(base + 2 * idx, re);
            atomicAdd(base + 2 * idx + 1, im);
        } else {
            base[2 * idx] += re;
            base[2 * idx + 1] += im;
        }
    } else {
        if (atomic)
            atomicAdd(base + idx, re);
        else
            base[idx] += re;
    }
}

__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 fadd2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 fmul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 ffma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

// dev_r_rinv on two lanes: one Newton step on the MUFU reciprocal square
// root, written with e' = p y0 - 1 = -e so that no operand needs a negation
__device__ __forceinline__ void dev_r_rinv2(float2 r2, float2& r, float2& rinv) {
    const float2 y0 = make_float2(rsqrtf(r2.x), rsqrtf(r2.y));
    const float2 p = fmul2(r2, y0);
    const float2 e = ffma2(p, y0, f2(-1.0f));
    rinv = ffma2(fmul2(f2(-0.5f), y0), e, y0);
    r = ffma2(fmul2(f2(-0.5f), p), e, p);
}

// dev_sincos_poly on two lanes (|y| <= pi/4); SHORT drops the y^9 term of
// sin and the y^10 term of cos (for |y| <= 0.3)
template <bool SHORT>
__device__ __forceinline__ void dev_sincos_poly2(float2 y, float2& s, float2& c) {
    const float2 y2 = fmul2(y, y);
    float2 ps;
    if (SHORT) {
        ps = ffma2(y2, f2(-1.98412698412698413e-04f), f2(8.33333333333333333e-03f));
    } else {
        ps = ffma2(y2, f2(2.75573192239858907e-06f), f2(-1.98412698412698413e-04f));
        ps = ffma2(y2, ps, f2(8.33333333333333333e-03f));
    }
    ps = ffma2(y2, ps, f2(-1.66666666666666667e-01f));
    s = ffma2(fmul2(y, y2), ps, y);
    float2 pc;
    if (SHORT) {
        pc = ffma2(y2, f2(2.48015873015873016e-05f), f2(-1.38888888888888889e-03f));
    } else {
        pc = ffma2(y2, f2(-2.75573192239858907e-07f), f2(2.48015873015873016e-05f));
        pc = ffma2(y2, pc, f2(-1.38888888888888889e-03f));
    }
    pc = ffma2(y2, pc, f2(4.16666666666666667e-02f));
    pc = ffma2(y2, pc, f2(-0.5f));
    c = ffma2(y2, pc, f2(1.0f));
}

}  // namespace
