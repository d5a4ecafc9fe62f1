// rte_ils.cuh -- continuum + Schwarzschild RTE per grid point, then the ILS and
// brightness temperature at the channel nodes only.
//
//  rte_kernel (one thread per grid point and profile) restates
//    continua added to the layer optical depth   src/Sensor/sounder.jl:310-322,
//      h2o_continuum / co2_continuum              src/CrossSections/continuum.jl:169-250
//    level_transmittances (FP64 product)          src/Solver/transmittance.jl:26-43
//    schwarzschild_rte, :cim and :toon sources    src/Solver/schwarzschild.jl:130-209
//    add_reflected_downwelling! when eps < 1      schwarzschild.jl:228-274
//    planck_radiance                              src/Solver/planck.jl:22-24
//  for the plain FP64 path: FP64 throughout.
//  rte_mixed_kernel is the same for the FP32 optical depths of the mixed path: FP64
//  only in the cumulative optical depth and the transmittances, FP32 (Kahan-summed
//  radiance) elsewhere.
//
//  ils_bt_kernel (one warp per channel and profile) restates apply_ils
//  (src/Sensor/ils.jl:131-153) evaluated at the grid nodes that the linear channel
//  resampling reads (sounder.jl:372-377), then brightness_temperature
//  (planck.jl:53-57).  Channel nodes are grid nodes for every sounder, so this is the
//  full convolution sampled where it is used, not an approximation.
#pragma once
#include "irs_internal.h"

namespace irs {

struct GridDev {
    long long n, den;
    double a_n, s_n, start, step;
    __host__ __device__ double at(long long i) const {
        return den ? (a_n + double(i) * s_n) / double(den) : start + double(i) * step;
    }
};
inline GridDev to_dev(const GridSpec& g) {
    GridDev d;
    d.n = g.n; d.den = g.den; d.a_n = g.a_n; d.s_n = g.s_n; d.start = g.start; d.step = g.step;
    return d;
}

// HITRAN CIA tables on the device (continuum.jl:104-160): tables t = 0 CO2-CO2,
// 1 N2-N2, 2 O2-O2 hold blocks [b0[t], b0[t+1]) in file order, each described by
// (T, nu_min, nu_max, first knot, knot count) with ascending knots nu/sg.
struct CiaDev {
    const double* blk;
    const double* nu;
    const double* sg;
    int b0[4];
};
constexpr int kCiaMax = 16;  // applicable blocks of one table cached per grid point
// The blocks that contain one grid point, their temperatures and sigma(nu), in file
// order (the temperature bracket of each layer is then a scan of these).
struct CiaPoint {
    double T[3][kCiaMax], s[3][kCiaMax];
    int n[3];
};

struct ContDev {
    const double* h2o;  // nu[n], cs[n], cf[n], te[n]
    const double* co2;  // nu[n], seff[n], tdep[n]
    int n_h2o, n_co2;
    int mask;           // 1 h2o, 2 co2, 4 co2_cia, 8 n2, 16 o2 (only when apply_continuum)
    CiaDev cia;
};
constexpr int kCiaMask = 4 | 8 | 16;

// linear interpolation on the block's knots (Interpolations.jl linear_interpolation)
__device__ __forceinline__ double cia_block_value(const CiaDev& c, int b, double nu) {
    const double* d = c.blk + 5 * (size_t)b;
    const double* x = c.nu + (long long)d[3];
    const double* y = c.sg + (long long)d[3];
    const int n = (int)d[4];
    if (n == 1) return y[0];
    int lo = 0, hi = n;  // upper_bound
    while (lo < hi) { const int mid = (lo + hi) >> 1; if (x[mid] <= nu) lo = mid + 1; else hi = mid; }
    const int i = min(max(lo - 1, 0), n - 2);
    const double w = (nu - x[i]) / (x[i + 1] - x[i]);
    return y[i] * (1.0 - w) + y[i + 1] * w;
}
__device__ __forceinline__ void cia_prepare(const CiaDev& c, int mask, double nu, CiaPoint& cp) {
    for (int t = 0; t < 3; ++t) {
        cp.n[t] = 0;
        if (!(mask & (4 << t))) continue;
        for (int b = c.b0[t]; b < c.b0[t + 1]; ++b) {
            const double* d = c.blk + 5 * (size_t)b;
            if (nu < d[1] || nu > d[2]) continue;
            const int k = cp.n[t]++;
            if (k < kCiaMax) {
                cp.T[t][k] = d[0];
                cp.s[t][k] = cia_block_value(c, b, nu);
            }
        }
    }
}
// _cia_sigma (continuum.jl:333-362): the applicable blocks bracketing T (first in file
// order among equal temperatures), linear in T, the nearest one outside the range
__device__ __forceinline__ double cia_sigma_at(const CiaDev& c, const CiaPoint& cp, int t, double nu, double T) {
    const int na = cp.n[t];
    if (na == 0) return 0.0;
    bool hl = false, hh = false;
    double T_lo = 0, s_lo = 0, T_hi = 0, s_hi = 0;
    auto take = [&](double bt, double s) {
        if (bt <= T && (!hl || bt > T_lo)) { hl = true; T_lo = bt; s_lo = s; }
        if (bt >= T && (!hh || bt < T_hi)) { hh = true; T_hi = bt; s_hi = s; }
    };
    if (na <= kCiaMax) {
        for (int k = 0; k < na; ++k) take(cp.T[t][k], cp.s[t][k]);
    } else {  // more applicable blocks than cached: scan the table
        for (int b = c.b0[t]; b < c.b0[t + 1]; ++b) {
            const double* d = c.blk + 5 * (size_t)b;
            if (nu < d[1] || nu > d[2]) continue;
            take(d[0], cia_block_value(c, b, nu));
        }
    }
    if (!hl) return s_hi;
    if (!hh) return s_lo;
    if (T_lo == T_hi) return s_lo;
    const double w = (T - T_lo) / (T_hi - T_lo);
    return (1.0 - w) * s_lo + w * s_hi;
}
// co2_cia, n2_cia, o2_cia (continuum.jl:252-331) times dz: sigma x pair densities
__device__ __forceinline__ double cia_tau(const ContDev& c, const CiaPoint& cp, double nu, double vh, double vc,
                                          double p, double T, double dz) {
    const double nair = p * 100.0 / (1.380649e-23 * T) * 1e-6;
    const double vdry = 1.0 - vh;
    double k = 0.0;
    if (c.mask & 4) k += cia_sigma_at(c.cia, cp, 0, nu, T) * (vc * nair) * nair;
    if (c.mask & 8) {
        const double n2 = 0.78084 * vdry * nair;
        k += cia_sigma_at(c.cia, cp, 1, nu, T) * n2 * n2;
    }
    if (c.mask & 16) {
        const double o2 = 0.20946 * vdry * nair;
        k += cia_sigma_at(c.cia, cp, 2, nu, T) * o2 * o2;
    }
    return k * dz;
}

// compensated FP32 sum: the value is s - c
__device__ __forceinline__ void kahan_add32(float& s, float& c, float v) {
    const float y = v - c;
    const float t = s + y;
    c = (t - s) - y;
    s = t;
}

__global__ void grid_values_kernel(GridDev g, double* out) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < g.n) out[i] = g.at(i);
}

__device__ __forceinline__ double planck64(double nu, double T) {
    return 1.191042953e-5 * (nu * nu * nu) / expm1(1.4387769 * nu / T);
}
__device__ __forceinline__ double cim_corr(double s) {  // schwarzschild.jl:59-63
    if (s < 0.06) return s / 6.0;
    const double e = exp(-s);
    return 1.0 - 2.0 * (e / (e - 1.0) + 1.0 / s);
}
__device__ __forceinline__ double lit_corr(double s) {  // schwarzschild.jl:43-47
    if (s < 1e-4) return s * (0.5 - s * (1.0 / 3.0 - s * 0.125));
    const double e = exp(-s);
    return (1.0 - e) / s - e;
}
__device__ __forceinline__ double radfn(double nu, double T) {  // continuum.jl:169-174
    const double x = 1.4387769 * nu / T;
    if (x <= 0.01) return 0.5 * x * nu;
    if (x <= 10.0) return nu * (1.0 - exp(-x)) / (1.0 + exp(-x));
    return nu;
}
// Interpolations.jl linear interpolation, Flat() extrapolation
struct Lerp {
    int i;
    double w;
    int edge;  // -1 below, +1 above, 0 inside
};
__device__ __forceinline__ Lerp lerp_at(const double* k, int n, double x) {
    Lerp r{0, 0.0, 0};
    if (x <= k[0]) { r.edge = -1; return r; }
    if (x >= k[n - 1]) { r.edge = 1; r.i = n - 1; return r; }
    int lo = 0, hi = n;  // upper_bound
    while (lo < hi) { const int mid = (lo + hi) >> 1; if (k[mid] <= x) lo = mid + 1; else hi = mid; }
    r.i = min(max(lo - 1, 0), n - 2);
    r.w = (x - k[r.i]) / (k[r.i + 1] - k[r.i]);
    return r;
}
__device__ __forceinline__ double lerp_val(const double* v, const Lerp& l) {
    if (l.edge) return v[l.i];
    return v[l.i] * (1.0 - l.w) + v[l.i + 1] * l.w;
}

template <bool CIA, typename TT>
__device__ __forceinline__ double layer_tau(const TT* tau_l, long long i, double nu, const LayerRT& r,
                                            const ContDev& c, double Cs, double Cf, double te, double Se,
                                            double td, const CiaPoint& cp) {
    double t = (double)tau_l[i];
    if (CIA) t += cia_tau(c, cp, nu, r.vmr_h2o, r.vmr_co2, r.p_mid, r.T_mid, r.dz_cm);
    if (c.mask) {
        const double T = r.T_mid, p = r.p_mid;
        const double rho = (p / 1013.0) * (296.0 / T);
        const double rad = radfn(nu, T);
        if (c.mask & 1) {
            const double n = r.vmr_h2o * p * 100.0 / (1.380649e-23 * T) * 1e-6;
            const double ks = Cs * pow(296.0 / T, te) * r.vmr_h2o * rho * rad * n;
            const double kf = Cf * (1.0 - r.vmr_h2o) * rho * rad * n;
            t += (ks + kf) * r.dz_cm;
        }
        if (c.mask & 2) {
            const double n = r.vmr_co2 * p * 100.0 / (1.380649e-23 * T) * 1e-6;
            const double pref = 1e-20 * n * rho;
            const double tc = td == 0.0 ? 1.0 : pow(T / 246.0, td);
            t += Se * tc * pref * rad * r.dz_cm;
        }
    }
    return t;
}

// CIA: a CIA table is in use (a separate instantiation keeps the per-point CIA cache
// out of the common kernel)
template <typename TT, bool CIA = false>
__global__ void __launch_bounds__(256) rte_kernel(const TT* __restrict__ tau, const LayerRT* __restrict__ lrt,
                                                  const ProfileRT* __restrict__ prt, int L,
                                                  const double* __restrict__ grid, long long n_nu, int src,
                                                  ContDev cont, double* __restrict__ I) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int p = blockIdx.y;
    if (i >= n_nu) return;
    const double nu = grid[i];
    double Cs = 0, Cf = 0, te = 0, Se = 0, td = 0;
    if (cont.mask & 1) {
        const Lerp l = lerp_at(cont.h2o, cont.n_h2o, nu);
        Cs = lerp_val(cont.h2o + cont.n_h2o, l);
        Cf = lerp_val(cont.h2o + 2 * cont.n_h2o, l);
        te = lerp_val(cont.h2o + 3 * cont.n_h2o, l);
    }
    if (cont.mask & 2) {
        const Lerp l = lerp_at(cont.co2, cont.n_co2, nu);
        Se = lerp_val(cont.co2 + cont.n_co2, l);
        td = lerp_val(cont.co2 + 2 * cont.n_co2, l);
    }
    CiaPoint cp;
    if (CIA) cia_prepare(cont.cia, cont.mask, nu, cp);
    const ProfileRT pr = prt[p];
    const LayerRT* lr = lrt + (size_t)p * L;
    const TT* tp = tau + (size_t)p * L * n_nu;
    double Tr_up = 1.0;   // transmittance of the level above (TOA = 1)
    double I_atm = 0.0;
    for (int k = L - 1; k >= 0; --k) {
        const LayerRT r = lr[k];
        const double s = layer_tau<CIA>(tp + (size_t)k * n_nu, i, nu, r, cont, Cs, Cf, te, Se, td, cp) / pr.mu;
        const double Tr_k = Tr_up * exp(-s);
        const double dT = Tr_up - Tr_k;
        if (src == 0) {
            const double Ba = planck64(nu, r.T_ave), Bt = planck64(nu, r.T_top);
            I_atm += Ba * dT + (Bt - Ba) * (dT * cim_corr(s));
        } else {
            const double Bb = planck64(nu, r.T_bot), Bt = planck64(nu, r.T_top);
            I_atm += Bt * dT + (Bb - Bt) * (Tr_up * lit_corr(s));
        }
        Tr_up = Tr_k;
    }
    const double Tr0 = Tr_up;
    double Iv = pr.eps * planck64(nu, pr.T_sfc) * Tr0 + I_atm;
    if (pr.eps < 1.0) {
        double Id = 0.0, g = 1.0;
        for (int k = 0; k < L; ++k) {
            const LayerRT r = lr[k];
            const double s = layer_tau<CIA>(tp + (size_t)k * n_nu, i, nu, r, cont, Cs, Cf, te, Se, td, cp) / pr.mu;
            double em;
            if (src == 0) {
                const double Ba = planck64(nu, r.T_ave), Bb = planck64(nu, r.T_bot);
                em = (1.0 - exp(-s)) * (Ba + (Bb - Ba) * cim_corr(s));
            } else {
                const double Bb = planck64(nu, r.T_bot), Bt = planck64(nu, r.T_top);
                em = Bb * (1.0 - exp(-s)) + (Bt - Bb) * lit_corr(s);
            }
            Id += g * em;
            g *= exp(-s);
        }
        Iv += (1.0 - pr.eps) * Id * Tr0;
    }
    I[(size_t)p * n_nu + i] = Iv;
}

// ------------------------------------------------------- RTE, mixed precision
// rte_mixed_kernel: the same radiative transfer as rte_kernel for the FP32 optical
// depths of the mixed path, with FP64 kept only where the result needs it: the
// cumulative layer-to-space optical depth and the transmittances exp(-OD) (and the
// surface-to-layer transmittance of the reflected term).  Planck radiances, the CIM /
// Toon corrections and the MT-CKD continua are FP32, and the radiance is summed in
// FP32 with Kahan compensation.  Per (grid point, layer) it reads the FP32 tau once.
//
// Per-layer FP32 constants, computed once per CTA from LayerRT into shared memory:
struct RteLayerF {
    float c2_ave, c2_top, c2_bot, c2_mid;  // c2 / T
    float h2o_self, h2o_for, l2_296, co2;  // continuum column factors, log2(296/T_mid)
    float l2_246, pad0, pad1, pad2;        // log2(T_mid / 246)
};
constexpr float kC1 = 1.191042953e-5f, kC2 = 1.4387769f;

// planck_radiance (planck.jl:22-24) with c1 nu^3 and c2/T given: c1 nu^3 / expm1(c2 nu / T);
// above x = 0.5 exp(x) - 1 loses under one bit, so the cheaper expf serves there
__device__ __forceinline__ float planck32(float c1nu3, float nu, float c2T) {
    const float x = nu * c2T;
    return c1nu3 * __frcp_rn(x > 0.5f ? expf(x) - 1.0f : expm1f(x));
}
// _cim_correction (schwarzschild.jl:59-63): s/6 below 0.06 as the reference, then the
// series 1 - 2 (1/s - 1/(e^s - 1)) = s/6 - s^3/360 + s^5/15120 - ... (next term below
// 2e-7 of the value for s < 0.5, where the direct form loses digits in FP32), then the
// direct form
__device__ __forceinline__ float cim_corr32(float s) {
    if (s < 0.06f) return s * (1.0f / 6.0f);
    if (s < 0.5f) {
        const float s2 = s * s;
        return s * fmaf(s2, fmaf(s2, 1.0f / 15120.0f, -1.0f / 360.0f), 1.0f / 6.0f);
    }
    return 1.0f - 2.0f * (1.0f / s - 1.0f / expm1f(s));
}
// _lit_correction (schwarzschild.jl:43-47): (1 - e^-s)/s - e^-s; the reference's series
// below 1e-4, continued to s^5 below 0.1 (next term s^6/840), then the direct form
__device__ __forceinline__ float lit_corr32(float s) {
    if (s < 1e-4f) return s * (0.5f - s * (1.0f / 3.0f - s * 0.125f));
    if (s < 0.1f)
        return s * fmaf(s, fmaf(s, fmaf(s, fmaf(s, 1.0f / 144.0f, -1.0f / 30.0f), 0.125f), -1.0f / 3.0f), 0.5f);
    const float e = __expf(-s);
    return -expm1f(-s) / s - e;
}
// radfn (continuum.jl:169-174) with c2/T given
__device__ __forceinline__ float radfn32(float nu, float c2T) {
    const float x = nu * c2T;
    if (x <= 0.01f) return 0.5f * x * nu;
    if (x <= 10.0f) {
        const float e = __expf(-x);
        return nu * (1.0f - e) / (1.0f + e);
    }
    return nu;
}

template <bool CIA>
__global__ void __launch_bounds__(256) rte_mixed_kernel(const float* __restrict__ tau, const LayerRT* __restrict__ lrt,
                                                        const ProfileRT* __restrict__ prt, int L,
                                                        const double* __restrict__ grid, long long n_nu, int src,
                                                        ContDev cont, double* __restrict__ I) {
    extern __shared__ __align__(16) unsigned char rte_smem[];
    RteLayerF* lc = reinterpret_cast<RteLayerF*>(rte_smem);
    const int p = blockIdx.y;
    const LayerRT* lr = lrt + (size_t)p * L;
    for (int k = threadIdx.x; k < L; k += blockDim.x) {  // layer constants (FP64 -> FP32)
        const LayerRT r = lr[k];
        RteLayerF c;
        c.c2_ave = (float)(1.4387769 / r.T_ave);
        c.c2_top = (float)(1.4387769 / r.T_top);
        c.c2_bot = (float)(1.4387769 / r.T_bot);
        c.c2_mid = (float)(1.4387769 / r.T_mid);
        const double rho = (r.p_mid / 1013.0) * (296.0 / r.T_mid);
        const double nh = r.vmr_h2o * r.p_mid * 100.0 / (1.380649e-23 * r.T_mid) * 1e-6;
        const double nc = r.vmr_co2 * r.p_mid * 100.0 / (1.380649e-23 * r.T_mid) * 1e-6;
        c.h2o_self = (float)(r.vmr_h2o * rho * nh * r.dz_cm);
        c.h2o_for = (float)((1.0 - r.vmr_h2o) * rho * nh * r.dz_cm);
        c.l2_296 = (float)log2(296.0 / r.T_mid);
        c.co2 = (float)(1e-20 * nc * rho * r.dz_cm);
        c.l2_246 = (float)log2(r.T_mid / 246.0);
        c.pad0 = c.pad1 = c.pad2 = 0.f;
        lc[k] = c;
    }
    __syncthreads();
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_nu) return;
    const double nud = grid[i];
    const float nu = (float)nud;
    const float c1nu3 = kC1 * nu * nu * nu;
    float Cs = 0.f, Cf = 0.f, te = 0.f, Se = 0.f, td = 0.f;
    if (cont.mask & 1) {
        const Lerp l = lerp_at(cont.h2o, cont.n_h2o, nud);
        Cs = (float)lerp_val(cont.h2o + cont.n_h2o, l);
        Cf = (float)lerp_val(cont.h2o + 2 * cont.n_h2o, l);
        te = (float)lerp_val(cont.h2o + 3 * cont.n_h2o, l);
    }
    if (cont.mask & 2) {
        const Lerp l = lerp_at(cont.co2, cont.n_co2, nud);
        Se = (float)lerp_val(cont.co2 + cont.n_co2, l);
        td = (float)lerp_val(cont.co2 + 2 * cont.n_co2, l);
    }
    CiaPoint cp;
    if (CIA) cia_prepare(cont.cia, cont.mask, nud, cp);
    const ProfileRT pr = prt[p];
    const float imu = (float)(1.0 / pr.mu);
    const float* tp = tau + (size_t)p * L * n_nu + i;
    // the layer's optical depth along the path (FP32)
    auto slant = [&](int k) -> float {
        const RteLayerF& c = lc[k];
        float t = tp[(size_t)k * n_nu];
        if (CIA) {
            const LayerRT r = lr[k];
            t += (float)cia_tau(cont, cp, nud, r.vmr_h2o, r.vmr_co2, r.p_mid, r.T_mid, r.dz_cm);
        }
        if (cont.mask & 3) {
            const float rad = radfn32(nu, c.c2_mid);
            float k_c = 0.f;
            if (cont.mask & 1) k_c = fmaf(Cs * exp2f(te * c.l2_296), c.h2o_self, Cf * c.h2o_for);
            if (cont.mask & 2) k_c = fmaf(Se * (td == 0.f ? 1.f : exp2f(td * c.l2_246)), c.co2, k_c);
            t = fmaf(k_c, rad, t);
        }
        return t * imu;
    };
    double od = 0.0;        // cumulative optical depth from the top of the atmosphere
    double Tr_up = 1.0;     // transmittance of the level above
    float Is = 0.f, Ic = 0.f;  // radiance, Kahan-compensated
    float B_up = planck32(c1nu3, nu, lc[L - 1].c2_top);  // B at the top level of the current layer
    for (int k = L - 1; k >= 0; --k) {
        const RteLayerF& c = lc[k];
        const float s = slant(k);
        od += (double)s;
        const double Tr_k = exp(-od);
        const float dT = (float)(Tr_up - Tr_k);
        const float B_bot = planck32(c1nu3, nu, c.c2_bot);
        float v;
        if (src == 0) {
            const float Ba = planck32(c1nu3, nu, c.c2_ave);
            v = fmaf(Ba, dT, (B_up - Ba) * (dT * cim_corr32(s)));
        } else {
            v = fmaf(B_up, dT, (B_bot - B_up) * ((float)Tr_up * lit_corr32(s)));
        }
        kahan_add32(Is, Ic, v);
        B_up = B_bot;
        Tr_up = Tr_k;
    }
    const double Tr0 = Tr_up;
    double Iv = (double)(Is - Ic) + pr.eps * (double)planck32(c1nu3, nu, kC2 / (float)pr.T_sfc) * Tr0;
    if (pr.eps < 1.0) {  // add_reflected_downwelling!: layers from the surface up
        float Ds = 0.f, Dc = 0.f;
        double od_s = 0.0;  // optical depth from the surface to the bottom of layer k
        for (int k = 0; k < L; ++k) {
            const RteLayerF& c = lc[k];
            const float s = slant(k);
            const float one_m = -expm1f(-s);
            float em;
            if (src == 0) {
                const float Ba = planck32(c1nu3, nu, c.c2_ave), Bb = planck32(c1nu3, nu, c.c2_bot);
                em = one_m * fmaf(Bb - Ba, cim_corr32(s), Ba);
            } else {
                const float Bb = planck32(c1nu3, nu, c.c2_bot), Bt = planck32(c1nu3, nu, c.c2_top);
                em = fmaf(Bb, one_m, (Bt - Bb) * lit_corr32(s));
            }
            kahan_add32(Ds, Dc, (float)exp(-od_s) * em);
            od_s += (double)s;
        }
        Iv += (1.0 - pr.eps) * (double)(Ds - Dc) * Tr0;
    }
    I[(size_t)p * n_nu + i] = Iv;
}

// ---------------------------------------------------------------- ILS
// ils.jl:80-114: raw taps, then area normalisation
__global__ void ils_taps_kernel(double dnu, double opd_max, double fwhm, int apod, long long n_half,
                                double* __restrict__ kern) {
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k > 2 * n_half) return;
    const int n_pts = 2048;
    const double dL = opd_max / (n_pts - 1);
    const double dv = double(k - n_half) * dnu;
    const double sg = fwhm / (2.0 * sqrt(2.0 * log(2.0)));
    const double nb[3][3] = {{0.384093, 0.087577, 0.528330},
                             {0.152442, 0.136176, 0.711382},
                             {0.045335, 0.554883, 0.399782}};
    double s = 0.0;
    for (int j = 0; j < n_pts; ++j) {
        const double L = (double(j) / double(n_pts - 1)) * opd_max;
        double A;
        if (apod == 0) A = exp(-(2.0 * (M_PI * M_PI)) * (sg * sg) * (L * L));
        else {
            const double x = L / opd_max;
            const double t = 1.0 - x * x;
            A = fabs(x) > 1.0 ? 0.0 : nb[apod - 1][0] + nb[apod - 1][1] * t * t + nb[apod - 1][2] * (t * t) * (t * t);
        }
        s += A * cos(2.0 * M_PI * L * dv);
    }
    kern[k] = 2.0 * s * dL;
}
__global__ void ils_normalise_kernel(double* kern, long long n, double dnu) {
    __shared__ double part[1024];
    double s = 0.0;
    for (long long k = threadIdx.x; k < n; k += blockDim.x) s += kern[k];
    part[threadIdx.x] = s;
    __syncthreads();
    for (int d = blockDim.x / 2; d; d >>= 1) {
        if ((int)threadIdx.x < d) part[threadIdx.x] += part[threadIdx.x + d];
        __syncthreads();
    }
    const double tot = part[0] * dnu;
    __syncthreads();
    for (long long k = threadIdx.x; k < n; k += blockDim.x) kern[k] /= tot;
}

__device__ double apod_at(const double* __restrict__ Ip, long long n_nu, const double* __restrict__ kern,
                          long long n_taps, long long i, int lane) {
    const long long half = (n_taps - 1) / 2;
    double acc = 0.0;
    for (long long k = lane; k < n_taps; k += 32) {
        const long long j = i + k - half;
        if (j >= 0 && j < n_nu) acc = fma(Ip[j], kern[k], acc);
    }
    for (int d = 16; d; d >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, d);
    return acc;
}

__global__ void __launch_bounds__(256) ils_bt_kernel(const double* __restrict__ I, long long n_nu,
                                                     const double* __restrict__ kern, long long n_taps,
                                                     double dnu_hi, GridDev g, GridDev ch, int with_ils,
                                                     double* __restrict__ R, double* __restrict__ BT) {
    const long long wid = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const int p = blockIdx.y;
    if (wid >= ch.n) return;
    const double nu = ch.at(wid);
    const double* Ip = I + (size_t)p * n_nu;
    auto value = [&](long long i) -> double {
        if (!with_ils) return Ip[i];
        return apod_at(Ip, n_nu, kern, n_taps, i, lane) * dnu_hi;
    };
    double Rv;
    const double g0 = g.at(0), gl = g.at(n_nu - 1);
    if (nu <= g0) Rv = value(0);
    else if (nu >= gl) Rv = value(n_nu - 1);
    else {
        long long i = (long long)floor((nu - g0) / dnu_hi);
        i = max(0LL, min(i, n_nu - 2));
        while (i > 0 && g.at(i) > nu) --i;
        while (i + 2 < n_nu && g.at(i + 1) <= nu) ++i;
        const double a = g.at(i), b = g.at(i + 1);
        const double w = (nu - a) / (b - a);
        const double r0 = value(i);
        Rv = w == 0.0 ? r0 : r0 * (1.0 - w) + value(i + 1) * w;
    }
    if (lane == 0) {
        R[(size_t)p * ch.n + wid] = Rv;
        BT[(size_t)p * ch.n + wid] =
            Rv <= 0.0 ? 0.0 : 1.4387769 * nu / log1p(1.191042953e-5 * (nu * nu * nu) / Rv);
    }
}

}  // namespace irs
