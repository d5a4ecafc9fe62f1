// lm_pert.cuh -- the relaxation-matrix line-mixing perturbation as a pole sum.
//
// Every term of the perturbation has the form (amplitudes already times f/sqrt(pi))
//     ar Re w(x + iy) + ai Im w(x + iy),   x = (nu - c) f,
// evaluated in FP64 with the far-wing limit w = (y + ix)/(sqrt(pi)(x^2 + y^2)) for
// |x| > x_far (line_mixing.jl:1000-1016 for the VP_W eigenmodes, :1177-1184 for the
// first-order dispersive lines).  One list of such poles per (profile, layer), sorted
// by centre: the VP_W modes of the whitelisted bands, the same bands' no-coupling
// modes with negated amplitudes (compute_vpw_band_perturbation, :1065-1075) and the
// VP_Y lines of the other bands (ar = 0).  The perturbation is a difference of sums
// that nearly cancel, so it stays FP64.
#pragma once
#include "faddeeva.cuh"

namespace irs {

struct LmPoleDev {
    double c, f, y, ar, ai;
    int window;  // 0: |nu - c| <= cutoff (VP_W, :1003); 1: nu - cutoff <= c <= nu + cutoff (VP_Y, :1172-1173)
    int pad;
};

// out[pl][i] for i < stride (rows padded with zeros beyond n_nu).  grid (pl rows) x (points)
__global__ void __launch_bounds__(256) lm_pert_kernel(const LmPoleDev* __restrict__ poles,
                                                      const long long* __restrict__ pl_off,
                                                      const double* __restrict__ grid, long long n_nu,
                                                      long long stride, double cutoff, double x_far,
                                                      double* __restrict__ out) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int pl = blockIdx.y;
    if (i >= stride) return;
    double acc = 0.0;
    if (i < n_nu) {
        const double nu = grid[i];
        const double left = nu - cutoff, right = nu + cutoff;
        const long long hi = pl_off[pl + 1];
        long long a = pl_off[pl], b = hi;
        const double left_s = left - 1e-6 * cutoff;  // each pole applies its own window test below
        while (a < b) {
            const long long m = (a + b) >> 1;
            if (poles[m].c < left_s) a = m + 1; else b = m;
        }
        for (long long j = a; j < hi; ++j) {
            const LmPoleDev P = poles[j];
            if (P.c > right + 1e-6 * cutoff) break;
            const double d = nu - P.c;
            if (P.window == 0 ? fabs(d) > cutoff : (P.c < left || P.c > right)) continue;
            const double x = d * P.f;
            double rw, iw;
            if (fabs(x) > x_far) {
                const double den = kInvSqrtPi / (x * x + P.y * P.y);
                rw = P.y * den;
                iw = x * den;
            } else {
                const double2 w = faddeeva64(x, P.y);
                rw = w.x;
                iw = w.y;
            }
            acc += P.ar * rw + P.ai * iw;
        }
    }
    out[(size_t)pl * stride + i] = acc;
}

// tau[pl][i] += the relmat species' cross section max(sigma_V + d_sigma, 0) times its
// column amount (the clamp of compute_voigt_{lm,vpw}_cross_sections): sv holds the
// line-sum's clamped Voigt part (already times the column amount for the FP32 path),
// dsig the perturbation; coef[pl] = 0 where the species is absent.
template <typename TT>
__global__ void __launch_bounds__(256) relmat_finish_kernel(TT* __restrict__ tau, const double* __restrict__ sv,
                                                            const double* __restrict__ dsig,
                                                            const double* __restrict__ coef, long long n_nu,
                                                            long long pstride) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int pl = blockIdx.y;
    const double c = coef[pl];
    if (i >= n_nu || c == 0.0) return;
    const size_t k = (size_t)pl * pstride + i;
    if (sizeof(TT) == sizeof(float))
        tau[(size_t)pl * n_nu + i] += fmaxf((float)sv[k] + (float)c * (float)dsig[k], 0.f);
    else
        tau[(size_t)pl * n_nu + i] += fmax(sv[k] + dsig[k], 0.0) * c;
}

}  // namespace irs
