// irs_host.cpp -- host-side per-profile setup of libirs_b200 (C++, no CUDA).
//
// This is the small amount of per-profile work the reference does on the host
// before its kernels: the internal grid, Curtis-Godson layer properties and the
// Faddeeva series coefficients.  It is O(levels x species) per profile.
#include <algorithm>
#include <cmath>
#include <memory>
#include <numeric>
#include <string>
#include <vector>

#include "faddeeva.cuh"
#include "irs_internal.h"

namespace irs {

namespace {
thread_local std::string t_err;
}
void set_error(const std::string& m) { t_err = m; }
const char* last_error() { return t_err.c_str(); }

// ---------------------------------------------------------------- grids
static int64_t rat_den(double x) {
    for (int64_t d = 1; d <= 1000000; ++d) {
        const double n = std::nearbyint(x * double(d));
        if (n / double(d) == x) return d;
    }
    return 0;
}

GridSpec make_grid(double a, double b, double s) {
    IRS_REQUIRE(s > 0.0 && std::isfinite(a) && std::isfinite(b), "grid step must be positive");
    GridSpec g;
    g.start = a;
    g.step = s;
    const int64_t ds = rat_den(s), da = rat_den(a), db = rat_den(b);
    if (ds && da && db) {
        int64_t den = std::lcm(std::lcm(da, ds), db);
        g.den = den;
        g.a_n = std::nearbyint(a * double(den));
        g.s_n = std::nearbyint(s * double(den));
        const double b_n = std::nearbyint(b * double(den));
        g.n = (int64_t)std::floor((b_n - g.a_n) / g.s_n) + 1;
    } else {
        const double lf = (b - a) / s;
        g.n = (int64_t)std::nearbyint(lf) + 1;
        if (a + double(g.n - 1) * s > b) g.n -= 1;
    }
    IRS_REQUIRE(g.n >= 1, "empty wavenumber grid");
    return g;
}

InternalGrid internal_grid(const irs_sounder& s, const irs_fm_options& o) {
    IRS_REQUIRE(s.dnu > 0 && s.nu_max >= s.nu_min, "invalid sounder grid");
    InternalGrid ig;
    if (o.high_res_factor > 0) ig.hrf = o.high_res_factor;
    else if (o.internal_dnu > 0) ig.hrf = std::max<int64_t>(1, (int64_t)std::ceil(s.dnu / o.internal_dnu));
    else ig.hrf = 4;
    ig.dnu_hi = s.dnu / double(ig.hrf);
    if (o.with_ils) {
        const double pad = std::ceil(16.0 / ig.dnu_hi) * ig.dnu_hi;  // ILS_HALFWIDTH_CM
        ig.g = make_grid(s.nu_min - pad, s.nu_max + pad, ig.dnu_hi);
    } else {
        ig.g = make_grid(s.nu_min, s.nu_max, ig.dnu_hi);
    }
    return ig;
}

// ----------------------------------------------------------- atmosphere
static bool approx_eq(double a, double b) {  // Julia isapprox, rtol = sqrt(eps)
    return std::fabs(a - b) <= 1.4901161193847656e-8 * std::max(std::fabs(a), std::fabs(b));
}
static double cg_column_vmr(double v1, double v2, double p1, double p2) {  // layers.jl:36-45
    if (v1 <= 0.0 || v2 <= 0.0) return 0.5 * (v1 + v2);
    if (approx_eq(v1, v2)) return v1;
    const double al = std::log(v2 / v1) / std::log(p2 / p1), r = p2 / p1, be = al + 1;
    if (std::fabs(be) < 1e-8) return (v1 - v2) / std::log(v1 / v2);
    return v1 * p1 * (1.0 - std::pow(r, be)) / (be * std::fabs(p1 - p2));
}
static double cg_pressure(double v1, double v2, double p1, double p2) {  // layers.jl:60-72
    if (v1 <= 0.0 || v2 <= 0.0) return 0.5 * (p1 + p2);
    if (approx_eq(v1, v2)) return 0.5 * (p1 + p2);
    const double al = std::log(v2 / v1) / std::log(p2 / p1), r = p2 / p1;
    const double b1 = al + 1, b2 = al + 2;
    if (std::fabs(b1) < 1e-8) return std::fabs(p1 - p2) / std::log(p1 / p2);
    if (std::fabs(b2) < 1e-8) return p2 * std::log(p2 / p1) / (p2 / p1 - 1.0);
    return p1 * b1 / b2 * (1.0 - std::pow(r, b2)) / (1.0 - std::pow(r, b1));
}
static double cg_temperature_mass(double T1, double T2, double p1, double p2) {  // :93-106
    if (approx_eq(T1, T2)) return T1;
    if (approx_eq(p1, p2)) return 0.5 * (T1 + T2);
    const double al = std::log(p2 / p1);
    double fr;
    if (std::fabs(al) < 1e-3) fr = 0.5 + al / 12.0;
    else { const double be = p2 / p1; fr = ((al - 1.0) * be + 1.0) / (al * (be - 1.0)); }
    return T1 + (T2 - T1) * fr;
}

// interpolation.jl:10-22: linear in log(p), flat outside the knots
namespace {
struct LogPInterp {
    std::vector<double> k, v;
    LogPInterp(int n, const double* p, const double* x) {
        std::vector<std::pair<double, double>> kv(n);
        for (int i = 0; i < n; ++i) kv[i] = {std::log(p[i]), x[i]};
        std::stable_sort(kv.begin(), kv.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
        for (auto& e : kv) { k.push_back(e.first); v.push_back(e.second); }
    }
    double operator()(double p) const {
        const double x = std::log(p);
        const size_t n = k.size();
        if (x <= k[0]) return v[0];
        if (x >= k[n - 1]) return v[n - 1];
        size_t i = std::upper_bound(k.begin(), k.end(), x) - k.begin() - 1;
        if (i >= n - 1) i = n - 2;
        const double w = (x - k[i]) / (k[i + 1] - k[i]);
        return v[i] * (1.0 - w) + v[i + 1] * w;
    }
};
}  // namespace

void layer_setup(const irs_profile& P, int pi, const irs_fm_options& o,
                 const std::vector<int>& list_species, const std::vector<double>& list_max_shift,
                 double dnu_grid, std::vector<Segment>& segs, std::vector<LayerRT>& lrt,
                 ProfileRT& prt) {
    const int nl = P.n_lev;
    IRS_REQUIRE(nl >= 2 && P.pressure && P.temperature, "profile needs >= 2 levels");
    IRS_REQUIRE(P.n_species >= 0 && (P.n_species == 0 || (P.species && P.vmr)), "profile species/vmr missing");
    IRS_REQUIRE(P.mu > 0.0 && P.mu <= 1.0, "mu must be in (0, 1]");
    IRS_REQUIRE(P.eps_sfc >= 0.0 && P.eps_sfc <= 1.0, "eps_sfc must be in [0, 1]");
    for (int k = 0; k < nl; ++k)
        IRS_REQUIRE(P.pressure[k] > 0.0 && P.temperature[k] > 0.0, "pressures and temperatures must be positive");
    const double* p = P.pressure;
    const double* T = P.temperature;
    const int L = nl - 1;
    LogPInterp Ti(nl, p, T);
    auto find_sp = [&](int sp) -> const double* {
        for (int q = 0; q < P.n_species; ++q) if (P.species[q] == sp) return P.vmr + (size_t)q * nl;
        return nullptr;
    };
    const double* vh = find_sp(1);
    const double* vc = find_sp(2);
    std::unique_ptr<LogPInterp> vhi, vci;
    if (vh) vhi.reset(new LogPInterp(nl, p, vh));
    if (vc) vci.reset(new LogPInterp(nl, p, vc));
    for (int k = 0; k < L; ++k) {
        const double p_mid = 0.5 * (p[k] + p[k + 1]);
        const double dp = std::fabs(p[k] - p[k + 1]);
        const double T_mass = cg_temperature_mass(T[k], T[k + 1], p[k], p[k + 1]);
        LayerRT r;
        r.T_ave = T_mass;
        r.T_top = T[k + 1];
        r.T_bot = T[k];
        r.p_mid = p_mid;
        r.T_mid = Ti(p_mid);
        // optical_depth.jl:123-130
        r.dz_cm = 8.314462 * r.T_mid / (0.028964 * 9.80665) * dp / p_mid * 100.0;
        r.vmr_h2o = vh ? (*vhi)(p_mid) : 0.0;
        r.vmr_co2 = vc ? (*vci)(p_mid) : 4.15e-4;
        lrt.push_back(r);
        for (size_t li = 0; li < list_species.size(); ++li) {
            const int sp = list_species[li];
            const double* v = find_sp(sp);
            if (!v) continue;
            const double vmr = cg_column_vmr(v[k], v[k + 1], p[k], p[k + 1]);
            if (vmr == 0.0) continue;
            const double pcg = cg_pressure(v[k], v[k + 1], p[k], p[k + 1]);
            Segment s;
            s.p_atm = pcg / 1013.25;
            s.T = o.T_method == 1 ? T_mass : Ti(pcg);
            s.vmr_self = sp == 1 ? vmr : 0.0;
            s.coef = vmr * dp * 2.1209e22;
            s.list = (int)li;
            // sounder.jl:294-300: DPTMIN is skipped for CO2 under any line-mixing model
            const bool lm_co2 = sp == 2 && o.line_mixing != IRS_LM_NONE;
            s.flags = (o.dptmn > 0.0 && !lm_co2 ? SEG_DPTMIN : 0) |
                      (lm_co2 && o.line_mixing == IRS_LM_PER_LINE_Y ? SEG_LM : 0);
            s.margin_g = list_max_shift[li] * s.p_atm / dnu_grid + 2.0;
            s.prof = pi;
            s.layer = k;
            s.out_off = 0;
            segs.push_back(s);
        }
    }
    prt.T_sfc = std::isnan(P.T_sfc) ? T[0] : P.T_sfc;
    prt.mu = P.mu;
    prt.eps = P.eps_sfc;
}

// ------------------------------------------------------ Jacobian chains
// schwarzschild_jacobian.jl:47-53
double cg_mass_frac(double p1, double p2) {
    if (approx_eq(p1, p2)) return 0.5;
    const double al = std::log(p2 / p1);
    if (std::fabs(al) < 1e-3) return 0.5 + al / 12.0;
    const double be = p2 / p1;
    return ((al - 1.0) * be + 1.0) / (al * (be - 1.0));
}
// vmr_jacobian.jl:81-107
static void cg_column_vmr_grad(double v1, double v2, double p1, double p2, double& g1, double& g2) {
    if (v1 <= 0.0 || v2 <= 0.0) { g1 = g2 = 0.5; return; }
    if (approx_eq(v1, v2)) { const double fr = cg_mass_frac(p1, p2); g1 = 1.0 - fr; g2 = fr; return; }
    const double Lg = std::log(p2 / p1), al = std::log(v2 / v1) / Lg, be = al + 1.0, dp = std::fabs(p1 - p2);
    if (std::fabs(be) < 1e-6) {
        const double h1 = std::max(std::fabs(v1), 1e-300) * 1e-6, h2 = std::max(std::fabs(v2), 1e-300) * 1e-6;
        g1 = (cg_column_vmr(v1 + h1, v2, p1, p2) - cg_column_vmr(v1 - h1, v2, p1, p2)) / (2 * h1);
        g2 = (cg_column_vmr(v1, v2 + h2, p1, p2) - cg_column_vmr(v1, v2 - h2, p1, p2)) / (2 * h2);
        return;
    }
    const double r = p2 / p1, rb = std::pow(r, be);
    const double c = v1 * p1 * (1.0 - rb) / (be * dp);
    const double J = (v1 * p1 / Lg) * ((rb - 1.0) / (be * be) - rb * Lg / be);
    g1 = c / v1 - J / (v1 * dp);
    g2 = J / (v2 * dp);
}

// Weights of one (profile, layer, species) segment onto the layer Jacobian channels
// (vmr_jacobian.jl:230-290, 392-430): channel 0 tau; 1/2 the T_cg derivative split
// onto the layer's lower/upper level; 3+2r/4+2r the retrieved species r's level
// derivatives (column amount, CG pressure, CG temperature, self broadening).
void jacobian_weights(const irs_profile& P, const irs_fm_options& o, int species, int layer,
                      const irs_state_spec& sp, float w[][4]) {
    const int k = layer;
    const double p1 = P.pressure[k], p2 = P.pressure[k + 1];
    const double* v = nullptr;
    for (int q = 0; q < P.n_species; ++q) if (P.species[q] == species) v = P.vmr + (size_t)q * P.n_lev;
    const double pcg = cg_pressure(v[k], v[k + 1], p1, p2);
    w[0][0] = 1.f;
    if (sp.include_temperature) {
        const double wT = o.T_method == 1 ? cg_mass_frac(p1, p2) : std::log(pcg / p1) / std::log(p2 / p1);
        w[1][1] = (float)(1.0 - wT);
        w[2][1] = (float)wT;
    }
    for (int r = 0; r < sp.n_retrieved; ++r) {
        if (sp.retrieved[r] != species) continue;
        const double v1 = v[k], v2 = v[k + 1];
        const double vcg = cg_column_vmr(v1, v2, p1, p2);
        double gV1, gV2;
        cg_column_vmr_grad(v1, v2, p1, p2, gV1, gV2);
        double gP1 = 0, gP2 = 0, gT1 = 0, gT2 = 0;
        if (sp.vmr_coupling) {
            const double h1 = std::max(std::fabs(v1), 1e-300) * 1e-6, h2 = std::max(std::fabs(v2), 1e-300) * 1e-6;
            gP1 = (cg_pressure(v1 + h1, v2, p1, p2) - cg_pressure(v1 - h1, v2, p1, p2)) / (2 * h1);
            gP2 = (cg_pressure(v1, v2 + h2, p1, p2) - cg_pressure(v1, v2 - h2, p1, p2)) / (2 * h2);
            if (o.T_method != 1) {
                const double dTdp = (P.temperature[k + 1] - P.temperature[k]) / (pcg * std::log(p2 / p1));
                gT1 = dTdp * gP1;
                gT2 = dTdp * gP2;
            }
        }
        const bool self = species == 1 && sp.vmr_coupling;
        float* lo = w[3 + 2 * r];
        float* hi = w[4 + 2 * r];
        lo[0] = (float)(gV1 / vcg); lo[1] = (float)gT1; lo[2] = (float)(gP1 / 1013.25); lo[3] = self ? (float)gV1 : 0.f;
        hi[0] = (float)(gV2 / vcg); hi[1] = (float)gT2; hi[2] = (float)(gP2 / 1013.25); hi[3] = self ? (float)gV2 : 0.f;
    }
}

// --------------------------------------------------- Faddeeva constants
static void weideman_coefficients(int N, double* L_out, double* a_out) {
    const int M = 2 * N, M2 = 2 * M;
    const long double Lw = std::sqrt((long double)N / std::sqrt(2.0L));
    std::vector<long double> f(M2, 0.0L), g(M2);
    for (int k = -M + 1; k <= M - 1; ++k) {
        const long double th = (long double)k * (long double)M_PI / M;
        const long double t = Lw * std::tan(th / 2.0L);
        f[k + M] = std::exp(-t * t) * (Lw * Lw + t * t);
    }
    for (int m = 0; m < M2; ++m) g[(m + M) % M2] = f[m];
    for (int n = 1; n <= N; ++n) {
        long double s = 0.0L;
        for (int m = 0; m < M2; ++m) s += g[m] * std::cos(2.0L * (long double)M_PI * n * m / M2);
        a_out[N - n] = (double)(s / M2);
    }
    *L_out = (double)Lw;
}

void compute_faddeeva_consts(FaddeevaConsts* c) {
    weideman_coefficients(kW64N, &c->w64_L, c->w64_a);
    double L32, a32[kW32N];
    weideman_coefficients(kW32N, &L32, a32);
    c->w32_L = (float)L32;
    for (int i = 0; i < kW32N; ++i) c->w32_a[i] = (float)a32[i];
    // voigt.jl:56-70
    const int N = 24;
    const double L = std::sqrt(double(N) / std::log(2.0));
    for (int n = 1; n <= N; ++n) {
        const double t = L * std::tan(double(2 * n - 1 - N) * M_PI / double(2 * N));
        const double w = L * L + t * t;
        c->wd_t[n - 1] = t;
        c->wd_w[n - 1] = w;
        c->wd_c[n - 1] = w * std::exp(-t * t);
        c->wf_t[n - 1] = (float)t;
        c->wf_w[n - 1] = (float)w;
        c->wf_c[n - 1] = (float)(w * std::exp(-t * t));
    }
    c->wd_scale = double(N) * L;
    c->wf_scale = (float)c->wd_scale;
}

}  // namespace irs
