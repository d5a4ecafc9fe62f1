// operators.cuh -- the reference's array-level operators as stand-alone device
// kernels, for callers that use them outside forward_model:
//   voigt_profile (voigt.jl:177-200) with its three evaluators, w(z) itself
//   (faddeeva_voigt / the VP_Y Im w, voigt.jl:152-160, line_mixing.jl:1182), and the
//   direct ILS convolution of a whole spectrum (apply_ils, ils.jl:131-153).
// The RTE (schwarzschild_rte) and the ILS taps (ils_kernel) reuse rte_kernel and
// ils_taps_kernel.
#pragma once
#include "faddeeva.cuh"

namespace irs {

// voigt_profile(nu, nu0, gL, gD, method), FP64
__global__ void __launch_bounds__(256) voigt_profile_kernel(const double* __restrict__ nu, long long n, double nu0,
                                                            double gL, double gD, int method,
                                                            double* __restrict__ out) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double d = nu[i] - nu0;
    if (method == 2) {  // pseudo_voigt_profile, Thompson et al. (1987) (voigt.jl:134-147)
        const double fG = 2.0 * gD, fL = 2.0 * gL;
        const double fV = pow(fG * fG * fG * fG * fG + 2.69269 * fG * fG * fG * fG * fL + 2.42843 * fG * fG * fG * fL * fL +
                                  4.47163 * fG * fG * fL * fL * fL + 0.07842 * fG * fL * fL * fL * fL +
                                  fL * fL * fL * fL * fL,
                              0.2);
        const double gV = 0.5 * fV, r = fL / fV;
        const double eta = 1.36603 * r - 0.47719 * r * r + 0.11116 * r * r * r;
        const double G = sqrt(0.69314718055994531 / 3.14159265358979324) / gV * exp(-0.69314718055994531 * d * d / (gV * gV));
        const double L = gV / (3.14159265358979324 * (d * d + gV * gV));
        out[i] = eta * L + (1.0 - eta) * G;
        return;
    }
    const double f = kSqrtLn2 / gD;
    const double x = d * f, y = gL * f;
    const double H = method == 1 ? weideman24_64(x, y) : faddeeva64(x, y).x;
    out[i] = f * H * kInvSqrtPi;
}

// w(x + i y) with the FP32 evaluator of the mixed line sums (faddeeva32: the rational
// continued fractions and the Weideman N = 16 series), for checking it on its own
__global__ void __launch_bounds__(256) faddeeva32_kernel(const double* __restrict__ x, const double* __restrict__ y,
                                                         long long n, double* __restrict__ re, double* __restrict__ im) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float2 w = faddeeva32_inline((float)x[i], (float)y[i]);
    re[i] = (double)w.x;
    im[i] = (double)w.y;
}

// w(x + i y) = erfcx(y - i x), FP64
__global__ void __launch_bounds__(256) faddeeva_kernel(const double* __restrict__ x, const double* __restrict__ y,
                                                       long long n, double* __restrict__ re, double* __restrict__ im) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double2 w = faddeeva64(x[i], y[i]);
    re[i] = w.x;
    im[i] = w.y;
}

// out[i] = dnu sum_k spectrum[i + k - half] kern[k] over the grid (zero outside), FP64.
// A block stages its 256 outputs' spectrum window (256 + 2 half points) in shared
// memory in chunks of kIlsChunk taps; the taps are read through the read-only path.
constexpr int kIlsThreads = 256;
constexpr int kIlsChunk = 4096;
__global__ void __launch_bounds__(kIlsThreads) apply_ils_kernel(const double* __restrict__ s, long long n_nu,
                                                                const double* __restrict__ kern, long long n_taps,
                                                                double dnu, double* __restrict__ out) {
    __shared__ double win[kIlsThreads + kIlsChunk];
    const long long half = (n_taps - 1) / 2;
    const long long i0 = (long long)blockIdx.x * kIlsThreads;
    const long long i = i0 + threadIdx.x;
    double acc = 0.0;
    for (long long k0 = 0; k0 < n_taps; k0 += kIlsChunk) {
        const int nk = (int)min((long long)kIlsChunk, n_taps - k0);
        // window: spectrum[i0 + k0 - half + t], t in [0, kIlsThreads + nk)
        __syncthreads();
        for (int t = threadIdx.x; t < kIlsThreads + nk; t += kIlsThreads) {
            const long long j = i0 + k0 - half + t;
            win[t] = (j >= 0 && j < n_nu) ? s[j] : 0.0;
        }
        __syncthreads();
        for (int k = 0; k < nk; ++k) acc = fma(win[threadIdx.x + k], __ldg(kern + k0 + k), acc);
    }
    if (i < n_nu) out[i] = acc * dnu;
}

}  // namespace irs
