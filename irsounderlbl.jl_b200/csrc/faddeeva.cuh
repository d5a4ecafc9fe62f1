// faddeeva.cuh -- Voigt H-function evaluators on the device.
//
// The reference evaluates H(x, y) = Re w(x + i y) three ways (VoigtMethod,
// src/CrossSections/voigt.jl:32-36):
//   FullFaddeeva  Re erfcx(y - i x) through SpecialFunctions/OpenSpecFun (:158-160)
//   Weideman      its own 24-node trapezoid rule with a two-sum correction (:89-117)
//   PseudoVoigt   Thompson eta-mixing (:134-147), evaluated inline by the kernels
// and switches to the Lorentz far wing y/(sqrt(pi)(x^2 + y^2)) for |x| > x_far (:170-172).
//
// FullFaddeeva is restated from published methods (no third-party source):
//   FP64: Laplace continued fraction (24 levels) for |x| + y >= 8, else the
//         Weideman (1994, SIAM J. Numer. Anal. 31:1497) rational series, N = 40.
//   FP32: continued fraction with 2 levels for |x| + y >= 15, 4 levels for
//         8 <= |x| + y < 15, else the Weideman series with N = 16, each written as
//         one rational function with a single MUFU reciprocal.
// The series coefficients are the DFT of exp(-t^2)(L^2 + t^2) at
// t = L tan(theta/2), computed once on the host (irs_host.cpp) and held in
// constant memory.
#pragma once
#include <cuda_runtime.h>

namespace irs {

constexpr double kInvSqrtPi = 0.56418958354775628695;  // 1/sqrt(pi)
constexpr double kSqrtLn2 = 0.83255461115769775635;    // sqrt(log 2)
constexpr int kW64N = 40;
constexpr int kW32N = 16;

struct FaddeevaConsts {
    double w64_L;
    double w64_a[kW64N];  // highest power first
    float w32_L;
    float w32_a[kW32N];
    // reference Weideman-24 evaluator (voigt.jl:56-70)
    double wd_t[24], wd_w[24], wd_c[24], wd_scale;
    float wf_t[24], wf_w[24], wf_c[24], wf_scale;
};

// Filled by irs_host.cpp; uploaded with cudaMemcpyToSymbol at context creation.
void compute_faddeeva_consts(FaddeevaConsts* c);

}  // namespace irs

#ifdef __CUDACC__
static __constant__ irs::FaddeevaConsts c_fad;  // one copy per translation unit

namespace irs {

// ---------------------------------------------------------------- FP64
__device__ __forceinline__ double2 cdiv64(double2 a, double2 b) {
    const double d = b.x * b.x + b.y * b.y;
    return make_double2((a.x * b.x + a.y * b.y) / d, (a.y * b.x - a.x * b.y) / d);
}
__device__ __forceinline__ double2 cmul64(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

static __device__ __noinline__ double2 faddeeva64(double x, double y) {
    if (fabs(x) + y >= 8.0) {
        const double2 z = make_double2(x, y);
        double2 r = make_double2(0.0, 0.0);
#pragma unroll 1
        for (int k = 24; k >= 1; --k)
            r = cdiv64(make_double2(0.5 * k, 0.0), make_double2(z.x - r.x, z.y - r.y));
        return cdiv64(make_double2(0.0, kInvSqrtPi), make_double2(z.x - r.x, z.y - r.y));
    }
    const double L = c_fad.w64_L;
    const double2 den = make_double2(L + y, -x);  // L - i z
    const double2 num = make_double2(L - y, x);   // L + i z
    const double2 Z = cdiv64(num, den);
    double2 p = make_double2(c_fad.w64_a[0], 0.0);
#pragma unroll 8
    for (int n = 1; n < kW64N; ++n) {
        p = cmul64(p, Z);
        p.x += c_fad.w64_a[n];
    }
    const double2 d2 = cmul64(den, den);
    const double2 t1 = cdiv64(make_double2(2.0 * p.x, 2.0 * p.y), d2);
    const double2 t2 = cdiv64(make_double2(kInvSqrtPi, 0.0), den);
    return make_double2(t1.x + t2.x, t1.y + t2.y);
}

// erfcx(y) = w(i y) for real y >= 0 (the DPTMIN peak, voigt.jl:345); the same two
// methods as faddeeva64 restricted to the imaginary axis, in real arithmetic.  The
// continued fraction converges faster as y grows: 12 levels for y >= 8, 8 for y >= 15,
// 6 for y >= 26, 5 for y >= 40 and 4 for y >= 60 agree with 24 levels to within an
// ulp (checked in double precision over y in [8, 1e6]).
static __device__ double erfcx64(double y) {
    if (y >= 8.0) {
        const int K = y >= 60.0 ? 4 : y >= 40.0 ? 5 : y >= 26.0 ? 6 : y >= 15.0 ? 8 : 12;
        double rho = 0.0;
#pragma unroll 1
        for (int k = K; k >= 1; --k) rho = -(0.5 * k) / (y - rho);
        return kInvSqrtPi / (y - rho);
    }
    const double L = c_fad.w64_L;
    const double Z = (L - y) / (L + y);
    double p = c_fad.w64_a[0];
#pragma unroll 8
    for (int n = 1; n < kW64N; ++n) p = p * Z + c_fad.w64_a[n];
    const double den = L + y;
    return 2.0 * p / (den * den) + kInvSqrtPi / den;
}

// voigt.jl:89-101
static __device__ __noinline__ double weideman24_64(double x, double y) {
    double A = 0.0, B = 0.0;
#pragma unroll 4
    for (int n = 0; n < 24; ++n) {
        const double dx = x - c_fad.wd_t[n];
        const double d = dx * dx + y * y;
        A += c_fad.wd_c[n] / d;
        B += c_fad.wd_w[n] / d;
    }
    const double sc = y / c_fad.wd_scale;
    return fmax(0.0, exp(-(x * x)) * (1.0 - B * sc) + A * sc);
}

// H(x, y) for the FP64 kernels, method 1 = Weideman-24, 3 = FullFaddeeva
template <int METHOD>
__device__ __forceinline__ double hcore64(double x, double y) {
    if (METHOD == 1) return weideman24_64(x, y);
    return faddeeva64(x, y).x;
}

// ---------------------------------------------------------------- FP32
// 1/x by the MUFU approximation (about 1 ulp); x > 0 and finite where it is used
__device__ __forceinline__ float rcp_approx32(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// a / b; |b|^2 is a normal FP32 number wherever it is used (|b| between about 1 and 30)
__device__ __forceinline__ float2 cdiv32(float2 a, float2 b) {
    const float inv = rcp_approx32(b.x * b.x + b.y * b.y);
    return make_float2((a.x * b.x + a.y * b.y) * inv, (a.y * b.x - a.x * b.y) * inv);
}
__device__ __forceinline__ float2 cmul32(float2 a, float2 b) {
    return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}

// The continued fractions of the FP32 evaluator folded into rational functions, so
// that each branch takes a single reciprocal (the MUFU pipe runs at an eighth of the
// FMA rate, and chained reciprocals were the cost of the core pairs):
//   2 levels, i/sqrt(pi) / (z - 1/2 / (z - 1/z))
//       = (i/sqrt(pi)) (z^2 - 1) / (z (z^2 - 3/2))
//   4 levels, i/sqrt(pi) / (z - 1/2 / (z - 1 / (z - 3/2 / (z - 2/z))))
//       = (i/sqrt(pi)) (u^2 - 9/2 u + 2) / (z (u^2 - 5 u + 15/4)),  u = z^2
// Over their regions (|z| >= 10.6, resp. 5.6 <= |z| < 15) the polynomials' roots
// (|u| <= 4.1) are far away, so no cancellation; |den|^2 stays below 3e38 for
// |z| < 2.6e6.  The Weideman branch shares the reciprocal of |L - i z|^2 between its
// two divisions.

// w = (i/sqrt(pi)) N / D as (Re, Im), for N = (nr, ni), D = (dr, di)
__device__ __forceinline__ float2 wz_ratio32(float nr, float ni, float dr, float di) {
    const float s = (float)kInvSqrtPi * rcp_approx32(fmaf(dr, dr, di * di));
    return make_float2((nr * di - ni * dr) * s, fmaf(nr, dr, ni * di) * s);
}

// Faddeeva w(z) for |x| + y >= 15 (two levels); y2 = y^2
__device__ __forceinline__ float2 faddeeva_cf2(float x, float y, float y2) {
    const float ur = fmaf(x, x, -y2), ui = 2.f * x * y;              // u = z^2
    const float cr = ur - 1.5f;                                       // u - 3/2
    return wz_ratio32(ur - 1.f, ui, fmaf(x, cr, -y * ui), fmaf(x, ui, y * cr));
}

__device__ __forceinline__ float2 faddeeva32_inline(float x, float y) {
    const float s = fabsf(x) + y;
    if (s >= 15.0f) return faddeeva_cf2(x, y, y * y);
    if (s >= 8.0f) {  // four levels
        const float ur = fmaf(x, x, -y * y), ui = 2.f * x * y;
        const float ar = ur - 4.5f, br = ur - 5.f;
        const float nr = fmaf(ur, ar, fmaf(-ui, ui, 2.f)), ni = ui * (ar + ur);        // u (u - 9/2) + 2
        const float mr = fmaf(ur, br, fmaf(-ui, ui, 3.75f)), mi = ui * (br + ur);      // u (u - 5) + 15/4
        return wz_ratio32(nr, ni, fmaf(x, mr, -y * mi), fmaf(x, mi, y * mr));          // z m
    }
    const float L = c_fad.w32_L;
    const float er = L + y;  // den = L - i z = (er, -x), num = L + i z = (L - y, x)
    const float inv = rcp_approx32(fmaf(er, er, x * x));
    const float nr = L - y;
    // Z = num conj(den) / |den|^2
    const float2 Z = make_float2(fmaf(nr, er, -x * x) * inv, fmaf(x, er, nr * x) * inv);
    float2 p = make_float2(c_fad.w32_a[0], 0.0f);
#pragma unroll
    for (int n = 1; n < kW32N; ++n) {
        p = cmul32(p, Z);
        p.x += c_fad.w32_a[n];
    }
    // w = 2 p / den^2 + (1/sqrt(pi)) / den = (2 p + den / sqrt(pi)) conj(den)^2 / |den|^4
    const float qr = fmaf(2.f, p.x, er * (float)kInvSqrtPi), qi = fmaf(2.f, p.y, -x * (float)kInvSqrtPi);
    const float cr = fmaf(er, er, -x * x), ci = 2.f * x * er;  // conj(den)^2
    const float i2 = inv * inv;
    return make_float2(fmaf(qr, cr, -qi * ci) * i2, fmaf(qr, ci, qi * cr) * i2);
}
// the same as a call (per-point loops, where inlining it would cost registers)
static __device__ __noinline__ float2 faddeeva32(float x, float y) { return faddeeva32_inline(x, y); }


// faddeeva32 with its |x| + y >= 15 branch (the two-level continued fraction) inlined
// in real arithmetic; the CF4 and Weideman regions go through the shared routine
__device__ __forceinline__ float2 faddeeva32_fast(float x, float y) {
    if (fabsf(x) + y >= 15.0f) return faddeeva_cf2(x, y, y * y);
    return faddeeva32(x, y);
}

// voigt.jl:105-117 (Float32 Weideman-24, IEEE division as Julia's Float32 `/`)
static __device__ __noinline__ float weideman24_32(float x, float y) {
    float A = 0.0f, B = 0.0f;
#pragma unroll 4
    for (int n = 0; n < 24; ++n) {
        const float dx = x - c_fad.wf_t[n];
        const float d = dx * dx + y * y;
        A += __fdiv_rn(c_fad.wf_c[n], d);
        B += __fdiv_rn(c_fad.wf_w[n], d);
    }
    const float sc = __fdiv_rn(y, c_fad.wf_scale);
    return fmaxf(0.0f, expf(-(x * x)) * (1.0f - B * sc) + A * sc);
}

}  // namespace irs
#endif  // __CUDACC__
