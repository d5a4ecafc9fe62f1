// irs_oracle.cpp -- TEST INFRASTRUCTURE ONLY (see irs_oracle.h).
//
// FP64 C++ restatement of IRSounderLBL.jl's line-by-line forward path.  Each
// function names the reference file:line it restates.  OpenMP parallelises the
// loops over grid points exactly where the reference's KernelAbstractions CPU
// backend does (one work item per grid point), so per-point arithmetic order is
// the reference's.
#include "irs_oracle.h"

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include <map>
#include <numeric>
#include <string>
#include <utility>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

using cplx = std::complex<double>;
thread_local std::string g_err;

int fail(const std::string& m) { g_err = m; return -1; }

// ---------------------------------------------------------------- constants
const double SQRT_LN2 = std::sqrt(std::log(2.0));          // voigt.jl:4
const double INV_SQRT_PI = 1.0 / std::sqrt(M_PI);          // voigt.jl:5
const double C2_LINE = 1.4387752;                           // broadening.jl:10
const double T_REF = 296.0;                                 // partition.jl:6
const double PLANCK_C1 = 1.191042953e-5;                    // planck.jl:11
const double PLANCK_C2 = 1.4387769;                         // planck.jl:12
const double ILS_HALFWIDTH_CM = 16.0;                       // ils.jl:24
const double NAIR_PER_VMR = 2.1209e22;                      // sounder.jl:280

// broadening.jl:17-24 (species-average n_self, delta_self)
double n_self_of(int mol, double n_air) {
    if (mol == 1) return 0.95;
    if (mol == 2) return 0.75;
    return n_air;
}
double delta_self_of(int mol) {
    if (mol == 1) return 0.002;
    if (mol == 2) return -0.003;
    return 0.0;
}
// broadening.jl:131-148
double molecular_mass_amu(int mol) {
    static const double m[11] = {18.010, 44.010, 47.998, 44.013, 28.010, 16.043,
                                 31.999, 34.015, 64.065, 36.461, 17.031};
    if (mol < 1 || mol > 11) return 30.0;
    return m[mol - 1];
}

// ------------------------------------------------------------------ tables
struct Tips { int tmin; std::vector<double> q; };
std::map<std::pair<int, int>, Tips> g_tips;
struct Table1D { std::vector<double> x; std::vector<std::vector<double>> y; };
Table1D g_ckd_h2o;  // y: Cs, Cf, texp
Table1D g_ckd_co2;  // y: S*xfac, tdep
bool g_have_h2o = false, g_have_co2 = false;

// Interpolations.jl linear_interpolation(knots, v; extrapolation_bc=Flat()),
// as used at continuum.jl:64-66, :94-95 and interpolation.jl:20.
double interp_flat(const std::vector<double>& k, const std::vector<double>& v, double x) {
    const size_t n = k.size();
    if (x <= k[0]) return v[0];
    if (x >= k[n - 1]) return v[n - 1];
    size_t i = std::upper_bound(k.begin(), k.end(), x) - k.begin() - 1;
    if (i >= n - 1) i = n - 2;
    const double w = (x - k[i]) / (k[i + 1] - k[i]);
    return v[i] * (1.0 - w) + v[i + 1] * w;
}

// partition.jl:10-18 (_tips_lookup: linear at 1 K, clamped indices)
double tips_lookup(const Tips& t, double T) {
    const long n = (long)t.q.size();
    long i_lo = (long)std::floor(T) - t.tmin + 1;  // 1-based
    long i_hi = i_lo + 1;
    i_lo = std::min(std::max(i_lo, 1L), n);
    i_hi = std::min(std::max(i_hi, 1L), n);
    const double frac = T - std::floor(T);
    return t.q[i_lo - 1] * (1.0 - frac) + t.q[i_hi - 1] * frac;
}

// ------------------------------------------------------------ Faddeeva w(z)
// The reference evaluates Re/Im erfcx(y - i x) = w(x + i y) through
// SpecialFunctions.jl -> OpenSpecFun (voigt.jl:158-160, line_mixing.jl:1182).
// Restated here from two published methods (no third-party source):
//   * |x| + y >= 8: Laplace continued fraction
//       w(z) = (i/sqrt(pi)) / (z - (1/2)/(z - 1/(z - (3/2)/(z - ...)))), 24 levels;
//   * otherwise: Weideman, SIAM J. Numer. Anal. 31 (1994) 1497-1518, rational
//       series with N = 40 terms, w = 2 p(Z)/(L - i z)^2 + (1/sqrt(pi))/(L - i z),
//       Z = (L + i z)/(L - i z), L = sqrt(N/sqrt(2)); the coefficients of p are
//       the DFT of exp(-t^2)(L^2 + t^2) at t = L tan(theta/2).
// Checked against scipy.special.wofz to ~2e-14 of |w| in tests/test_oracle_pins.py.
struct WeidemanW {
    static const int N = 40;
    double L;
    double a[N];  // highest power first (polyval order)
    WeidemanW() {
        const int M = 2 * N, M2 = 2 * M;
        L = std::sqrt(N / std::sqrt(2.0));
        // f sampled at k = -M+1..M-1, prefixed with 0 -> length 2M; fftshift;
        // real part of the DFT divided by 2M; keep entries 1..N reversed.
        std::vector<double> f(M2, 0.0);
        for (int k = -M + 1; k <= M - 1; ++k) {
            const double th = k * M_PI / M;
            const double t = L * std::tan(th / 2.0);
            f[k + M] = std::exp(-t * t) * (L * L + t * t);
        }
        // fftshift of length-2M vector: element m moves to (m + M) mod 2M
        std::vector<double> g(M2);
        for (int m = 0; m < M2; ++m) g[(m + M) % M2] = f[m];
        for (int n = 1; n <= N; ++n) {
            long double s = 0.0L;
            for (int m = 0; m < M2; ++m)
                s += (long double)g[m] * std::cos(2.0L * (long double)M_PI * n * m / M2);
            a[N - n] = (double)(s / M2);
        }
    }
    cplx eval(cplx z) const {
        const cplx iz(-z.imag(), z.real());
        const cplx den = L - iz;
        const cplx Z = (L + iz) / den;
        cplx p = a[0];
        for (int n = 1; n < N; ++n) p = p * Z + a[n];
        return 2.0 * p / (den * den) + INV_SQRT_PI / den;
    }
};
const WeidemanW& weid_w() { static const WeidemanW w; return w; }

cplx faddeeva(double x, double y) {
    if (std::fabs(x) + y >= 8.0) {
        const cplx z(x, y);
        cplx r = 0.0;
        for (int k = 24; k >= 1; --k) r = (0.5 * k) / (z - r);
        return cplx(0.0, INV_SQRT_PI) / (z - r);
    }
    return weid_w().eval(cplx(x, y));
}

// voigt.jl:56-64, 89-117: the reference's "Weideman" evaluator -- a 24-node
// trapezoid rule on the tan-substituted integral with a two-sum correction.
struct Weid24 {
    double t[24], w[24], c[24], scale;
    float t32[24], w32[24], c32[24], scale32;
    Weid24() {
        const int N = 24;
        const double L = std::sqrt(double(N) / std::log(2.0));
        for (int n = 1; n <= N; ++n) {
            t[n - 1] = L * std::tan(double(2 * n - 1 - N) * M_PI / double(2 * N));
            w[n - 1] = L * L + t[n - 1] * t[n - 1];
            c[n - 1] = w[n - 1] * std::exp(-t[n - 1] * t[n - 1]);
            t32[n - 1] = (float)t[n - 1]; w32[n - 1] = (float)w[n - 1]; c32[n - 1] = (float)c[n - 1];
        }
        scale = double(N) * L;
        scale32 = (float)scale;
    }
};
const Weid24& weid24() { static const Weid24 w; return w; }

double weideman_voigt(double x, double y) {
    const Weid24& W = weid24();
    double A = 0.0, B = 0.0;
    for (int n = 0; n < 24; ++n) {
        const double d = (x - W.t[n]) * (x - W.t[n]) + y * y;
        A += W.c[n] / d;
        B += W.w[n] / d;
    }
    const double sc = y / W.scale;
    return std::max(0.0, std::exp(-(x * x)) * (1.0 - B * sc) + A * sc);
}
float weideman_voigt32(float x, float y) {
    const Weid24& W = weid24();
    float A = 0.0f, B = 0.0f;
    for (int n = 0; n < 24; ++n) {
        const float dx = x - W.t32[n];
        const float d = dx * dx + y * y;
        A += W.c32[n] / d;
        B += W.w32[n] / d;
    }
    const float sc = y / W.scale32;
    return std::max(0.0f, std::exp(-(x * x)) * (1.0f - B * sc) + A * sc);
}

double faddeeva_voigt(double x, double y) { return faddeeva(x, y).real(); }

// voigt.jl:134-147
double pseudo_voigt_profile(double nu, double nu0, double gl, double gd) {
    const double fG = 2.0 * gd, fL = 2.0 * gl;
    const double fV = std::pow(std::pow(fG, 5) + 2.69269 * std::pow(fG, 4) * fL +
                               2.42843 * std::pow(fG, 3) * fL * fL +
                               4.47163 * fG * fG * std::pow(fL, 3) +
                               0.07842 * fG * std::pow(fL, 4) + std::pow(fL, 5), 0.2);
    const double gV = 0.5 * fV, r = fL / fV;
    const double eta = 1.36603 * r - 0.47719 * r * r + 0.11116 * r * r * r;
    const double d = nu - nu0;
    const double G = std::sqrt(std::log(2.0) / M_PI) / gV * std::exp(-std::log(2.0) * d * d / (gV * gV));
    const double Lz = gV / (M_PI * (d * d + gV * gV));
    return eta * Lz + (1.0 - eta) * G;
}

// --------------------------------------------------------- line parameters
struct LineParams { double nu0, S, gl, gd; };

// broadening.jl:40-53 (pressure_broadened_width), :89-99 (S(T)),
// :156-160 (pressure_shift); partition.jl:41-47 (Q_ratio)
double Q_ratio(int mol, int iso, double T) {
    auto it = g_tips.find({mol, iso});
    if (it == g_tips.end()) return T_REF / T;
    return tips_lookup(it->second, T_REF) / tips_lookup(it->second, T);
}
double partition_function(int mol, int iso, double T) {
    auto it = g_tips.find({mol, iso});
    if (it == g_tips.end()) return T / T_REF;
    return tips_lookup(it->second, T);
}
LineParams line_params(const orc_line& l, double T, double p, double vs) {
    LineParams o;
    const int mol = l.mol_id;
    const double n_air = (double)l.temp_depend;
    const double n_self = n_self_of(mol, n_air);
    const double tr = T_REF / T;
    o.gl = std::pow(tr, n_air) * (double)l.air_broad * (1.0 - vs) * p +
           std::pow(tr, n_self) * (double)l.self_broad * vs * p;
    o.gd = l.wavenumber * 3.58126e-7 * std::sqrt(T / molecular_mass_amu(mol));
    const double Qr = Q_ratio(mol, l.iso_id, T);
    const double stim = (1.0 - std::exp(-C2_LINE * l.wavenumber / T)) /
                        (1.0 - std::exp(-C2_LINE * l.wavenumber / T_REF));
    const double boltz = std::exp(-C2_LINE * l.lower_energy * (1.0 / T - 1.0 / T_REF));
    o.S = l.intensity * Qr * boltz * stim;
    o.nu0 = l.wavenumber + ((double)l.pressure_shift * (1.0 - vs) + delta_self_of(mol) * vs) * p;
    return o;
}

// voigt.jl:220-236 (1-based lower/upper bound on possibly unsorted shifted centres)
long lower_bound1(const double* a, double v, long n) {
    long lo = 1, hi = n + 1;
    while (lo < hi) { long mid = (lo + hi) >> 1; if (a[mid - 1] < v) lo = mid + 1; else hi = mid; }
    return lo;
}
long upper_bound1(const double* a, double v, long n) {
    long lo = 0, hi = n;
    while (lo < hi) { long mid = (lo + hi + 1) >> 1; if (a[mid - 1] > v) hi = mid - 1; else lo = mid; }
    return lo;
}

// voigt.jl:375-462 compute_voigt_cross_sections (host prep + kernels :243-313)
void voigt_xsec(const orc_line* lines, long nL, const double* grid, long n_nu, double T,
                double p, double vs, double cutoff, int method, double x_far, double* sigma) {
    std::vector<double> nu0(nL), S(nL), gl(nL), gd(nL), f(nL), y(nL), Sn(nL);
    for (long j = 0; j < nL; ++j) {
        LineParams lp = line_params(lines[j], T, p, vs);
        nu0[j] = lp.nu0;
        S[j] = lp.S;
        gl[j] = lp.gl;
        gd[j] = std::max(lp.gd, 1e-10);
        f[j] = SQRT_LN2 / gd[j];
        y[j] = lp.gl * f[j];
        Sn[j] = lp.S * f[j] * INV_SQRT_PI;
    }
    const double rc = 1.0 / cutoff;
    if (method == 2) {  // PseudoVoigt, voigt.jl:422-441, kernel :281-313
        std::vector<double> gV(nL), eta(nL), base(nL);
        const double cG = std::sqrt(std::log(2.0) / M_PI);
        for (long j = 0; j < nL; ++j) {
            const double fG = 2 * gd[j], fL = 2 * gl[j];
            const double fV = std::pow(std::pow(fG, 5) + 2.69269 * std::pow(fG, 4) * fL +
                                       2.42843 * std::pow(fG, 3) * (fL * fL) +
                                       4.47163 * (fG * fG) * std::pow(fL, 3) +
                                       0.07842 * fG * std::pow(fL, 4) + std::pow(fL, 5), 0.2);
            const double r = fL / fV;
            gV[j] = 0.5 * fV;
            eta[j] = 1.36603 * r - 0.47719 * (r * r) + 0.11116 * (r * r * r);
            const double Gc = cG / gV[j] * std::exp(-std::log(2.0) * (cutoff * cutoff) / (gV[j] * gV[j]));
            const double Lc = gV[j] * (1.0 / M_PI) / (cutoff * cutoff + gV[j] * gV[j]);
            base[j] = S[j] * (eta[j] * Lc + (1.0 - eta[j]) * Gc);
        }
        const double cln2 = std::log(2.0), invpi = 1.0 / M_PI;
#pragma omp parallel for schedule(static)
        for (long i = 0; i < n_nu; ++i) {
            const double nu = grid[i];
            const long jlo = lower_bound1(nu0.data(), nu - cutoff, nL);
            const long jhi = upper_bound1(nu0.data(), nu + cutoff, nL);
            double acc = 0.0;
            for (long j = jlo; j <= jhi; ++j) {
                const long q = j - 1;
                const double d = nu - nu0[q];
                const double G = cG / gV[q] * std::exp(-cln2 * d * d / (gV[q] * gV[q]));
                const double Lz = gV[q] * invpi / (d * d + gV[q] * gV[q]);
                const double zr = d * rc;
                acc += S[q] * (eta[q] * Lz + (1.0 - eta[q]) * G) - (2.0 - zr * zr) * base[q];
            }
            sigma[i] = std::max(acc, 0.0);
        }
        return;
    }
    // Weideman (1) or FullFaddeeva (3): voigt.jl:442-458, kernel :243-277
    auto Hcore = [method](double x, double yy) {
        return method == 3 ? faddeeva_voigt(x, yy) : weideman_voigt(x, yy);
    };
    std::vector<double> Hc(nL);
    for (long j = 0; j < nL; ++j) {
        const double xc = cutoff * f[j];
        Hc[j] = std::fabs(xc) > x_far ? y[j] * INV_SQRT_PI / (xc * xc + y[j] * y[j]) : Hcore(xc, y[j]);
    }
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n_nu; ++i) {
        const double nu = grid[i];
        const long jlo = lower_bound1(nu0.data(), nu - cutoff, nL);
        const long jhi = upper_bound1(nu0.data(), nu + cutoff, nL);
        double acc = 0.0;
        for (long j = jlo; j <= jhi; ++j) {
            const long q = j - 1;
            const double d = nu - nu0[q];
            const double x = d * f[q];
            const double yy = y[q];
            const double zr = d * rc;
            const double ped = (2.0 - zr * zr) * Hc[q];
            const double H = (std::fabs(x) > x_far ? yy * INV_SQRT_PI / (x * x + yy * yy) : Hcore(x, yy)) - ped;
            acc += Sn[q] * H;
        }
        sigma[i] = std::max(acc, 0.0);
    }
}

// voigt.jl:333-355 (_reject_weak_lines; DPTMIN)
long reject_weak(const orc_line* lines, long nL, double T, double p, double coef, double vs,
                 double dptmn, uint8_t* keep) {
    long nk = 0;
    for (long j = 0; j < nL; ++j) {
        if (dptmn <= 0.0) { keep[j] = 1; ++nk; continue; }
        LineParams lp = line_params(lines[j], T, p, vs);
        const double gd = std::max(lp.gd, 1e-10);
        const double f = SQRT_LN2 / gd;
        const double peak = (lp.S * f * INV_SQRT_PI) * faddeeva_voigt(0.0, lp.gl * f);
        keep[j] = (peak * coef > dptmn) ? 1 : 0;
        nk += keep[j];
    }
    return nk;
}

// line_mixing.jl:1166-1236 (dispersive kernel and its flat SoA build), with the
// relaxation-matrix Y replaced by a per-line Y(T) = y0 (296/T)^0.75 and the
// per-line centre, widths and S(T) of the Voigt line itself.
void lm_dispersive(const orc_line* lines, long nL, const double* y0, const double* grid,
                   long n_nu, double T, double p, double cutoff, double x_far, double* ds) {
    struct DL { double nu0, f, y, ysn; };
    std::vector<DL> dl;
    dl.reserve(nL);
    for (long j = 0; j < nL; ++j) {
        const double Y = y0[j] * std::pow(T_REF / T, 0.75);
        if (Y == 0.0) continue;
        LineParams lp = line_params(lines[j], T, p, 0.0);
        if (lp.S <= 0.0) continue;
        const double f = SQRT_LN2 / std::max(lp.gd, 1e-10);
        dl.push_back({lp.nu0, f, lp.gl * f, Y * p * lp.S * f * INV_SQRT_PI});
    }
    std::stable_sort(dl.begin(), dl.end(), [](const DL& a, const DL& b) { return a.nu0 < b.nu0; });
    const long n = (long)dl.size();
    std::vector<double> c(n);
    for (long j = 0; j < n; ++j) c[j] = dl[j].nu0;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n_nu; ++i) {
        const double nu = grid[i];
        const long jlo = lower_bound1(c.data(), nu - cutoff, n);
        const long jhi = upper_bound1(c.data(), nu + cutoff, n);
        double acc = 0.0;
        for (long j = jlo; j <= jhi; ++j) {
            const DL& L = dl[j - 1];
            const double x = (nu - L.nu0) * L.f;
            const double imw = std::fabs(x) > x_far ? x * INV_SQRT_PI / (x * x + L.y * L.y)
                                                    : faddeeva(x, L.y).imag();
            acc += L.ysn * imw;
        }
        ds[i] = acc;
    }
}

// ------------------------------------------------------------ atmosphere
bool approx_eq(double a, double b) {  // Julia isapprox default rtol = sqrt(eps)
    return std::fabs(a - b) <= 1.4901161193847656e-8 * std::max(std::fabs(a), std::fabs(b));
}
// layers.jl:36-45
double cg_column_vmr(double v1, double v2, double p1, double p2) {
    if (v1 <= 0.0 || v2 <= 0.0) return 0.5 * (v1 + v2);
    if (approx_eq(v1, v2)) return v1;
    const double a = std::log(v2 / v1) / std::log(p2 / p1);
    const double r = p2 / p1, b = a + 1;
    if (std::fabs(b) < 1e-8) return (v1 - v2) / std::log(v1 / v2);
    return v1 * p1 * (1.0 - std::pow(r, b)) / (b * std::fabs(p1 - p2));
}
// layers.jl:60-72
double cg_pressure(double v1, double v2, double p1, double p2) {
    if (v1 <= 0.0 || v2 <= 0.0) return 0.5 * (p1 + p2);
    if (approx_eq(v1, v2)) return 0.5 * (p1 + p2);
    const double a = std::log(v2 / v1) / std::log(p2 / p1);
    const double r = p2 / p1, b1 = a + 1, b2 = a + 2;
    if (std::fabs(b1) < 1e-8) return std::fabs(p1 - p2) / std::log(p1 / p2);
    if (std::fabs(b2) < 1e-8) return p2 * std::log(p2 / p1) / (p2 / p1 - 1.0);
    return p1 * b1 / b2 * (1.0 - std::pow(r, b2)) / (1.0 - std::pow(r, b1));
}
// layers.jl:93-106
double cg_temperature_mass(double T1, double T2, double p1, double p2) {
    if (approx_eq(T1, T2)) return T1;
    if (approx_eq(p1, p2)) return 0.5 * (T1 + T2);
    const double a = std::log(p2 / p1);
    double frac;
    if (std::fabs(a) < 1e-3) frac = 0.5 + a / 12.0;
    else { const double b = p2 / p1; frac = ((a - 1.0) * b + 1.0) / (a * (b - 1.0)); }
    return T1 + (T2 - T1) * frac;
}
// interpolation.jl:10-22 (linear in log p, flat outside)
struct LogPInterp {
    std::vector<double> k, v;
    LogPInterp(int n, const double* p, const double* x) {
        std::vector<std::pair<double, double>> kv(n);
        for (int i = 0; i < n; ++i) kv[i] = {std::log(p[i]), x[i]};
        bool sorted = true;
        for (int i = 1; i < n; ++i) if (kv[i].first < kv[i - 1].first) sorted = false;
        if (!sorted) std::stable_sort(kv.begin(), kv.end(),
                                      [](auto& a, auto& b) { return a.first < b.first; });
        for (auto& e : kv) { k.push_back(e.first); v.push_back(e.second); }
    }
    double operator()(double p) const { return interp_flat(k, v, std::log(p)); }
};

// ------------------------------------------------------------ continua
// continuum.jl:169-174
double radfn(double nu, double T) {
    const double x = 1.4387769 * nu / T;
    if (x <= 0.01) return 0.5 * x * nu;
    if (x <= 10.0) return nu * (1.0 - std::exp(-x)) / (1.0 + std::exp(-x));
    return nu;
}
// optical_depth.jl:123-130
double dp_to_dz_cm(double dp, double pmid, double T) {
    const double H = 8.314462 * T / (0.028964 * 9.80665);
    return H * dp / pmid * 100.0;
}
// continuum.jl:183-209
void h2o_continuum_add(const double* grid, long n, double vmr, double p, double T, double dz, double* tau) {
    if (!g_have_h2o) return;  // missing table: zeros (continuum.jl:190-194)
    const double rho = (p / 1013.0) * (296.0 / T);
    const double nh2o = vmr * p * 100.0 / (1.380649e-23 * T) * 1e-6;
    for (long i = 0; i < n; ++i) {
        const double nu = grid[i];
        const double Cs = interp_flat(g_ckd_h2o.x, g_ckd_h2o.y[0], nu);
        const double Cf = interp_flat(g_ckd_h2o.x, g_ckd_h2o.y[1], nu);
        const double te = interp_flat(g_ckd_h2o.x, g_ckd_h2o.y[2], nu);
        const double rad = radfn(nu, T);
        const double ks = Cs * std::pow(296.0 / T, te) * vmr * rho * rad * nh2o;
        const double kf = Cf * (1.0 - vmr) * rho * rad * nh2o;
        tau[i] += (ks + kf) * dz;
    }
}
// continuum.jl:227-250
void co2_continuum_add(const double* grid, long n, double vmr, double p, double T, double dz, double* tau) {
    if (!g_have_co2) return;
    const double rho = (p / 1013.0) * (296.0 / T);
    const double nco2 = vmr * p * 100.0 / (1.380649e-23 * T) * 1e-6;
    const double pref = 1e-20 * nco2 * rho;
    const double tr = T / 246.0;
    for (long i = 0; i < n; ++i) {
        const double nu = grid[i];
        const double td = interp_flat(g_ckd_co2.x, g_ckd_co2.y[1], nu);
        const double tc = td == 0.0 ? 1.0 : std::pow(tr, td);
        tau[i] += interp_flat(g_ckd_co2.x, g_ckd_co2.y[0], nu) * tc * pref * radfn(nu, T) * dz;
    }
}

// HITRAN CIA tables (continuum.jl:104-160): blocks of (T, nu range, sigma(nu)),
// nu ascending within a block, sigma clamped at 0 when loaded.
struct CiaBlock {
    double T, numin, numax;
    std::vector<double> nu, sg;
};
std::vector<CiaBlock> g_cia[3];  // 0 CO2-CO2, 1 N2-N2, 2 O2-O2

// linear interpolation inside a block (the block's own knots)
double cia_block_value(const CiaBlock& b, double nu) {
    const std::vector<double>& x = b.nu;
    const long n = (long)x.size();
    if (n == 1) return b.sg[0];
    long i = (long)(std::upper_bound(x.begin(), x.end(), nu) - x.begin()) - 1;
    i = std::max(0L, std::min(i, n - 2));
    const double w = (nu - x[i]) / (x[i + 1] - x[i]);
    return b.sg[i] * (1.0 - w) + b.sg[i + 1] * w;
}
// _cia_sigma (continuum.jl:333-362): blocks containing nu, T bracketed linearly,
// the nearest block's value outside the bracketed range
double cia_sigma(const std::vector<CiaBlock>& B, double nu, double T) {
    double T_lo = -INFINITY, s_lo = 0.0, T_hi = INFINITY, s_hi = 0.0;
    bool any = false;
    for (const CiaBlock& b : B) {
        if (nu < b.numin || nu > b.numax) continue;
        any = true;
        const double s = cia_block_value(b, nu);
        if (b.T <= T && b.T > T_lo) { T_lo = b.T; s_lo = s; }
        if (b.T >= T && b.T < T_hi) { T_hi = b.T; s_hi = s; }
    }
    if (!any) return 0.0;
    if (!std::isfinite(T_lo)) return s_hi;
    if (!std::isfinite(T_hi)) return s_lo;
    if (T_lo == T_hi) return s_lo;
    const double w = (T - T_lo) / (T_hi - T_lo);
    return (1.0 - w) * s_lo + w * s_hi;
}
// co2_cia / n2_cia / o2_cia (continuum.jl:252-331): sigma * pair densities * dz
void cia_add(const double* grid, long n, int continua, double vh, double vc, double p, double T, double dz,
             double* tau) {
    const double nair = p * 100.0 / (1.380649e-23 * T) * 1e-6;
    const double vdry = 1.0 - vh;
    const double nn[3] = {vc * nair * nair, (0.78084 * vdry * nair) * (0.78084 * vdry * nair),
                          (0.20946 * vdry * nair) * (0.20946 * vdry * nair)};
    for (int t = 0; t < 3; ++t) {
        if (!(continua & (4 << t)) || g_cia[t].empty()) continue;
        for (long i = 0; i < n; ++i) tau[i] += cia_sigma(g_cia[t], grid[i], T) * nn[t] * dz;
    }
}

// ------------------------------------------------------------- solver
double planck(double nu, double T) { return PLANCK_C1 * (nu * nu * nu) / std::expm1(PLANCK_C2 * nu / T); }
double bt(double nu, double R) {
    if (R <= 0.0) return 0.0;
    return PLANCK_C2 * nu / std::log1p(PLANCK_C1 * (nu * nu * nu) / R);
}
// schwarzschild.jl:43-63
double lit_corr(double s) {
    if (s < 1e-4) return s * (0.5 - s * (1.0 / 3.0 - s * 0.125));
    const double e = std::exp(-s);
    return (1.0 - e) / s - e;
}
double cim_corr(double s) {
    if (s < 0.06) return s / 6.0;
    const double e = std::exp(-s);
    return 1.0 - 2.0 * (e / (e - 1.0) + 1.0 / s);
}

// transmittance.jl:26-43 and schwarzschild.jl:130-274, for one grid point.
// tau is [layer][nu] with stride n_nu.
double rte_point(double nu, long i, long n_nu, int L, const double* tau, const double* T_lev,
                 double T_sfc, double mu, double eps, int src, const double* T_ave) {
    std::vector<double> Tr(L + 1);
    Tr[L] = 1.0;
    for (int k = L - 1; k >= 0; --k) Tr[k] = Tr[k + 1] * std::exp(-tau[(long)k * n_nu + i] / mu);
    double I = eps * planck(nu, T_sfc) * Tr[0];
    for (int k = 0; k < L; ++k) {
        const double s = tau[(long)k * n_nu + i] / mu;
        const double dT = Tr[k + 1] - Tr[k];
        if (src == 1) {  // :toon
            const double Bb = planck(nu, T_lev[k]), Bt = planck(nu, T_lev[k + 1]);
            const double C = Tr[k + 1] * lit_corr(s);
            I += Bt * dT + (Bb - Bt) * C;
        } else {  // :cim
            const double Ba = planck(nu, T_ave[k]), Bt = planck(nu, T_lev[k + 1]);
            const double C = dT * cim_corr(s);
            I += Ba * dT + (Bt - Ba) * C;
        }
    }
    if (eps < 1.0) {  // schwarzschild.jl:203-206, 228-274
        double Id = 0.0, g = 1.0;
        for (int k = 0; k < L; ++k) {
            const double s = tau[(long)k * n_nu + i] / mu;
            double em;
            if (src == 1) {
                const double Bb = planck(nu, T_lev[k]), Bt = planck(nu, T_lev[k + 1]);
                em = Bb * (1.0 - std::exp(-s)) + (Bt - Bb) * lit_corr(s);
            } else {
                const double Ba = planck(nu, T_ave[k]), Bb = planck(nu, T_lev[k]);
                em = (1.0 - std::exp(-s)) * (Ba + (Bb - Ba) * cim_corr(s));
            }
            Id += g * em;
            g *= std::exp(-s);
        }
        I += (1.0 - eps) * Id * Tr[0];
    }
    return I;
}

// ils.jl:38-44, 80-114
const double NB[3][3] = {{0.384093, 0.087577, 0.528330},
                         {0.152442, 0.136176, 0.711382},
                         {0.045335, 0.554883, 0.399782}};
void ils_kernel(double dnu, double opd_max, double fwhm, int apod, std::vector<double>& kern) {
    const int n_pts = 2048;
    const double dL = opd_max / (n_pts - 1);
    std::vector<double> opd(n_pts), A(n_pts);
    for (int j = 0; j < n_pts; ++j) {
        // LinRange(0, opd_max, n): (1 - t)*0 + t*opd_max with t = j/(n-1)
        opd[j] = (double(j) / double(n_pts - 1)) * opd_max;
        if (apod == 0) {
            const double sg = fwhm / (2.0 * std::sqrt(2.0 * std::log(2.0)));
            A[j] = std::exp(-(2.0 * (M_PI * M_PI)) * (sg * sg) * (opd[j] * opd[j]));
        } else {
            const double x = opd[j] / opd_max;
            const double* c = NB[apod - 1];
            if (std::fabs(x) > 1.0) A[j] = 0.0;
            else { const double t = 1.0 - x * x; A[j] = c[0] + c[1] * t * t + c[2] * (t * t) * (t * t); }
        }
    }
    const long n_half = (long)std::ceil(ILS_HALFWIDTH_CM / dnu);
    kern.assign(2 * n_half + 1, 0.0);
    double tot = 0.0;
    for (long k = -n_half; k <= n_half; ++k) {
        const double dv = double(k) * dnu;
        double s = 0.0;
        for (int j = 0; j < n_pts; ++j) s += A[j] * std::cos(2.0 * M_PI * opd[j] * dv);
        kern[k + n_half] = 2.0 * s * dL;
    }
    for (double v : kern) tot += v;
    for (double& v : kern) v /= (tot * dnu);
}

// ------------------------------------------------------------- grid
// Julia's float range a:s:b (utils/wavenumber_grid.jl:23-26) rationalises
// start, step and stop and evaluates (a_n + i s_n)/den in extended precision.
long rat_den(double x) {
    for (long d = 1; d <= 1000000; ++d) {
        const double n = std::nearbyint(x * d);
        if (n / d == x) return d;
    }
    return 0;
}
struct Grid { double start, step; long den, n; double a_n, s_n; };
Grid make_grid(double a, double b, double s) {
    Grid g{a, s, 0, 0, 0, 0};
    const long ds = rat_den(s), da = rat_den(a), db = rat_den(b);
    if (ds && da && db) {
        long den = std::lcm(da, ds);
        den = std::lcm(den, db);
        g.den = den;
        g.a_n = std::nearbyint(a * den);
        g.s_n = std::nearbyint(s * den);
        const double b_n = std::nearbyint(b * den);
        g.n = (long)std::floor((b_n - g.a_n) / g.s_n) + 1;
    } else {
        const double lf = (b - a) / s;
        g.n = (long)std::nearbyint(lf) + 1;
        if (a + (g.n - 1) * s > b) g.n -= 1;
    }
    return g;
}
double grid_at(const Grid& g, long i) {
    if (g.den) return (g.a_n + double(i) * g.s_n) / double(g.den);
    return g.start + double(i) * g.step;
}

struct InternalGrid { Grid g; double dnu_hi; };
InternalGrid internal_grid(const orc_sounder& s, const orc_fm_options& o) {
    // sounder.jl:263-271, :155-161
    long hrf;
    if (o.high_res_factor > 0) hrf = o.high_res_factor;
    else if (o.internal_dnu > 0) hrf = std::max(1L, (long)std::ceil(s.dnu / o.internal_dnu));
    else hrf = 4;
    const double dhi = s.dnu / double(hrf);
    InternalGrid ig;
    ig.dnu_hi = dhi;
    if (o.with_ils) {
        const double pad = std::ceil(ILS_HALFWIDTH_CM / dhi) * dhi;
        ig.g = make_grid(s.nu_min - pad, s.nu_max + pad, dhi);
    } else {
        ig.g = make_grid(s.nu_min, s.nu_max, dhi);
    }
    return ig;
}

// ======================================================== Jacobian pieces
// partition.jl:52-66 (staircase slope of the 1 K TIPS table)
double partition_derivative(int mol, int iso, double T) {
    auto it = g_tips.find({mol, iso});
    if (it == g_tips.end()) return 1.0 / T_REF;
    const Tips& t = it->second;
    const long i_lo = (long)std::floor(T) - t.tmin + 1, i_hi = i_lo + 1;
    if (i_lo < 1 || i_hi > (long)t.q.size()) return 0.0;
    return t.q[i_hi - 1] - t.q[i_lo - 1];
}

// schwarzschild.jl:71-90
double lit_corr_deriv(double s) {
    if (s < 1e-4) return 0.5 - s * (2.0 / 3.0 - s * 0.375);
    const double e = std::exp(-s);
    return (e * (s + 1.0) - 1.0) / (s * s) + e;
}
double cim_corr_deriv(double s) {
    if (s < 0.06) return 1.0 / 6.0;
    const double w = std::exp(-s);
    return 2.0 / (s * s) - 2.0 * w / ((w - 1.0) * (w - 1.0));
}
double dB_dT(double nu, double T) {  // planck.jl:67-71
    const double x = PLANCK_C2 * nu / T, ex = std::exp(x);
    return PLANCK_C1 * PLANCK_C2 * (nu * nu * nu * nu) * ex / ((T * T) * (ex - 1.0) * (ex - 1.0));
}
// schwarzschild_jacobian.jl:47-53
double cg_mass_frac(double p1, double p2) {
    if (approx_eq(p1, p2)) return 0.5;
    const double a = std::log(p2 / p1);
    if (std::fabs(a) < 1e-3) return 0.5 + a / 12.0;
    const double b = p2 / p1;
    return ((a - 1.0) * b + 1.0) / (a * (b - 1.0));
}
// vmr_jacobian.jl:81-107
void cg_column_vmr_grad(double v1, double v2, double p1, double p2, double& g1, double& g2) {
    if (v1 <= 0.0 || v2 <= 0.0) { g1 = g2 = 0.5; return; }
    if (approx_eq(v1, v2)) { const double fr = cg_mass_frac(p1, p2); g1 = 1.0 - fr; g2 = fr; return; }
    const double L = std::log(p2 / p1), al = std::log(v2 / v1) / L, be = al + 1.0, dp = std::fabs(p1 - p2);
    if (std::fabs(be) < 1e-6) {
        const double h1 = std::max(std::fabs(v1), 1e-300) * 1e-6, h2 = std::max(std::fabs(v2), 1e-300) * 1e-6;
        g1 = (cg_column_vmr(v1 + h1, v2, p1, p2) - cg_column_vmr(v1 - h1, v2, p1, p2)) / (2 * h1);
        g2 = (cg_column_vmr(v1, v2 + h2, p1, p2) - cg_column_vmr(v1, v2 - h2, p1, p2)) / (2 * h2);
        return;
    }
    const double r = p2 / p1, rb = std::pow(r, be);
    const double c = v1 * p1 * (1.0 - rb) / (be * dp);
    const double J = (v1 * p1 / L) * ((rb - 1.0) / (be * be) - rb * L / be);
    g1 = c / v1 - J / (v1 * dp);
    g2 = J / (v2 * dp);
}
// vmr_jacobian.jl:120-125
double dBT_dR(double nu, double R) {
    if (R <= 0.0) return 0.0;
    const double A = PLANCK_C1 * (nu * nu * nu), L = std::log1p(A / R);
    return PLANCK_C2 * nu * A / ((L * L) * R * (R + A));
}

// cross_section_jacobian.jl:43-56
void voigt_H_and_grad(double x, double y, double x_far, double& H, double& Hx, double& Hy) {
    if (std::fabs(x) > x_far) {
        const double d = x * x + y * y, d2 = d * d;
        H = y * INV_SQRT_PI / d;
        Hx = -2.0 * x * y * INV_SQRT_PI / d2;
        Hy = INV_SQRT_PI * (x * x - y * y) / d2;
        return;
    }
    const cplx w = faddeeva(x, y);
    const double K = w.real(), L = w.imag();
    H = K;
    Hx = -2.0 * x * K + 2.0 * y * L;
    Hy = 2.0 * (x * L + y * K) - 2.0 * INV_SQRT_PI;
}

struct Grad { std::vector<double> s, dT, dp, dv; };

// cross_section_jacobian.jl:155-240 (sigma, dsigma/dT, dsigma/dp_atm, dsigma/dvmr_self)
void voigt_xsec_grad(const orc_line* lines, long nL, const double* grid, long n_nu, double T, double p,
                     double vs, double cutoff, double x_far, Grad& g) {
    std::vector<double> nu0(nL), f(nL), df(nL), y(nL), dyT(nL), dyp(nL), dyv(nL), dn0p(nL), dn0v(nL),
        Sn(nL), dSnT(nL), Hc(nL), dHcT(nL), dHcp(nL), dHcv(nL);
    for (long j = 0; j < nL; ++j) {
        const orc_line& l = lines[j];
        const int mol = l.mol_id;
        const double n_air = (double)l.temp_depend, n_self = n_self_of(mol, n_air);
        const double d_air = (double)l.pressure_shift, d_self = delta_self_of(mol);
        LineParams lp = line_params(l, T, p, vs);
        nu0[j] = lp.nu0;
        dn0p[j] = d_air * (1.0 - vs) + d_self * vs;
        dn0v[j] = (d_self - d_air) * p;
        // temperature_scaled_intensity_deriv, broadening.jl:112-128
        const double QT = partition_function(mol, l.iso_id, T), dQT = partition_derivative(mol, l.iso_id, T);
        const double a = C2_LINE * l.wavenumber;
        const double dlnS = -dQT / QT + C2_LINE * l.lower_energy / (T * T) - (a / (T * T)) / (std::exp(a / T) - 1.0);
        const double S = lp.S, dS = S * dlnS;
        // pressure_broadened_width_deriv, broadening.jl:62-78
        const double tr = T_REF / T;
        const double A = std::pow(tr, n_air) * (double)l.air_broad * (1.0 - vs) * p;
        const double B = std::pow(tr, n_self) * (double)l.self_broad * vs * p;
        const double gl = A + B, dglT = -(n_air * A + n_self * B) / T;
        double gd = lp.gd;
        const double dgd = gd / (2.0 * T);
        gd = std::max(gd, 1e-10);
        const double fj = SQRT_LN2 / gd, dfj = -fj * (dgd / gd);
        const double ac = std::pow(tr, n_air) * (double)l.air_broad, bc = std::pow(tr, n_self) * (double)l.self_broad;
        const double dglp = gl / p, dglv = (bc - ac) * p;
        f[j] = fj; df[j] = dfj; y[j] = gl * fj;
        dyT[j] = dglT * fj + gl * dfj; dyp[j] = dglp * fj; dyv[j] = dglv * fj;
        Sn[j] = S * fj * INV_SQRT_PI;
        dSnT[j] = (dS * fj + S * dfj) * INV_SQRT_PI;
        double hc, hx, hy;
        voigt_H_and_grad(cutoff * fj, y[j], x_far, hc, hx, hy);
        Hc[j] = hc;
        dHcT[j] = hx * (cutoff * dfj) + hy * dyT[j];
        dHcp[j] = hy * dyp[j];
        dHcv[j] = hy * dyv[j];
    }
    g.s.assign(n_nu, 0.0); g.dT.assign(n_nu, 0.0); g.dp.assign(n_nu, 0.0); g.dv.assign(n_nu, 0.0);
    const double invc = 1.0 / cutoff, invc2 = invc * invc;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n_nu; ++i) {
        const double nu = grid[i];
        const long jlo = lower_bound1(nu0.data(), nu - cutoff, nL), jhi = upper_bound1(nu0.data(), nu + cutoff, nL);
        double acc = 0, aT = 0, ap = 0, av = 0;
        for (long jj = jlo; jj <= jhi; ++jj) {
            const long j = jj - 1;
            const double d = nu - nu0[j], fj = f[j], x = d * fj;
            double H, Hx, Hy;
            voigt_H_and_grad(x, y[j], x_far, H, Hx, Hy);
            const double dHt = Hx * (d * df[j]) + Hy * dyT[j];
            const double dHp = Hx * (-dn0p[j] * fj) + Hy * dyp[j];
            const double dHv = Hx * (-dn0v[j] * fj) + Hy * dyv[j];
            const double pedfac = 2.0 - (d * invc) * (d * invc);
            const double dpfp = 2.0 * d * dn0p[j] * invc2, dpfv = 2.0 * d * dn0v[j] * invc2;
            const double dpedT = pedfac * dHcT[j];
            const double dpedp = dpfp * Hc[j] + pedfac * dHcp[j];
            const double dpedv = dpfv * Hc[j] + pedfac * dHcv[j];
            const double Hm = H - pedfac * Hc[j];
            acc += Sn[j] * Hm;
            aT += dSnT[j] * Hm + Sn[j] * (dHt - dpedT);
            ap += Sn[j] * (dHp - dpedp);
            av += Sn[j] * (dHv - dpedv);
        }
        if (acc > 0.0) { g.s[i] = acc; g.dT[i] = aT; g.dp[i] = ap; g.dv[i] = av; }
    }
}

// cross_section_jacobian.jl:255-322 for VP_Y: analytic Voigt baseline plus the
// dispersive perturbation central-differenced in (T, p)
void species_grad(const orc_line* ll, long nL, const double* y0, bool lm, const double* grid, long n,
                  double T, double p, double vs, double cutoff, double lm_cutoff, double x_far, Grad& g) {
    voigt_xsec_grad(ll, nL, grid, n, T, p, vs, cutoff, x_far, g);
    if (!lm || !y0) return;
    std::vector<double> d0(n), a(n), b(n);
    lm_dispersive(ll, nL, y0, grid, n, T, p, lm_cutoff, x_far, d0.data());
    const double hT = 0.02;
    lm_dispersive(ll, nL, y0, grid, n, T + hT, p, lm_cutoff, x_far, a.data());
    lm_dispersive(ll, nL, y0, grid, n, T - hT, p, lm_cutoff, x_far, b.data());
    std::vector<double> dT(n);
    for (long i = 0; i < n; ++i) dT[i] = (a[i] - b[i]) / (2 * hT);
    const double hp = std::max(p, 1e-6) * 1e-4;
    lm_dispersive(ll, nL, y0, grid, n, T, p + hp, lm_cutoff, x_far, a.data());
    lm_dispersive(ll, nL, y0, grid, n, T, p - hp, lm_cutoff, x_far, b.data());
    for (long i = 0; i < n; ++i) {
        const double s = g.s[i] + d0[i];
        if (s <= 0.0) { g.s[i] = 0; g.dT[i] = 0; g.dp[i] = 0; }
        else { g.s[i] = s; g.dT[i] += dT[i]; g.dp[i] += (a[i] - b[i]) / (2 * hp); }
    }
}

}  // namespace

// =================================================================== C ABI
// The lines of a list (sorted by wavenumber) that can reach grid [lo, hi]: centres
// within the cutoff plus 1 cm^-1 (more than any pressure shift) of it.  Lines beyond
// contribute nothing to the window, so leaving them out of a windowed run changes no
// result; an unsorted list is used whole.
static void reach_range(const orc_line* ll, long nL, double lo, double hi, double reach, long& a, long& b) {
    a = 0;
    b = nL;
    for (long j = 1; j < nL; ++j)
        if (ll[j].wavenumber < ll[j - 1].wavenumber) return;
    const double vlo = lo - reach - 1.0, vhi = hi + reach + 1.0;
    a = (long)(std::lower_bound(ll, ll + nL, vlo, [](const orc_line& l, double v) { return l.wavenumber < v; }) - ll);
    b = (long)(std::upper_bound(ll, ll + nL, vhi, [](double v, const orc_line& l) { return v < l.wavenumber; }) - ll);
}

extern "C" {

const char* orc_last_error(void) { return g_err.c_str(); }
int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void orc_clear_tables(void) {
    g_tips.clear();
    g_have_h2o = g_have_co2 = false;
}
int orc_set_tips(int mol, int iso, int tmin, int n, const double* q) {
    if (n < 2) return fail("TIPS table needs at least 2 points");
    g_tips[{mol, iso}] = Tips{tmin, std::vector<double>(q, q + n)};
    return 0;
}
int orc_set_ckd_h2o(int n, const double* nu, const double* cs, const double* cf, const double* te) {
    g_ckd_h2o.x.assign(nu, nu + n);
    g_ckd_h2o.y = {std::vector<double>(cs, cs + n), std::vector<double>(cf, cf + n),
                   std::vector<double>(te, te + n)};
    g_have_h2o = true;
    return 0;
}
int orc_set_ckd_co2(int n, const double* nu, const double* s, const double* xf, const double* td) {
    g_ckd_co2.x.assign(nu, nu + n);
    std::vector<double> se(n);
    for (int i = 0; i < n; ++i) se[i] = s[i] * xf[i];
    g_ckd_co2.y = {se, std::vector<double>(td, td + n)};
    g_have_co2 = true;
    return 0;
}

void orc_faddeeva(double x, double y, double* re, double* im) {
    cplx w = faddeeva(x, y);
    *re = w.real();
    *im = w.imag();
}
double orc_weideman_voigt(double x, double y) { return weideman_voigt(x, y); }
float orc_weideman_voigt32(float x, float y) { return weideman_voigt32(x, y); }
double orc_pseudo_voigt_profile(double nu, double nu0, double gl, double gd) {
    return pseudo_voigt_profile(nu, nu0, gl, gd);
}
double orc_voigt_profile(double nu, double nu0, double gl, double gd, int method) {
    if (method == 2) return pseudo_voigt_profile(nu, nu0, gl, gd);
    const double f = SQRT_LN2 / gd, x = (nu - nu0) * f, y = gl * f;
    const double H = method == 1 ? weideman_voigt(x, y) : faddeeva_voigt(x, y);
    return f * H * INV_SQRT_PI;
}
double orc_Q_ratio(int mol, int iso, double T) { return Q_ratio(mol, iso, T); }
double orc_partition_function(int mol, int iso, double T) { return partition_function(mol, iso, T); }
void orc_line_params(const orc_line* l, double T, double p, double vs, double* nu0, double* S,
                     double* gl, double* gd) {
    LineParams lp = line_params(*l, T, p, vs);
    *nu0 = lp.nu0; *S = lp.S; *gl = lp.gl; *gd = lp.gd;
}
double orc_planck(double nu, double T) { return planck(nu, T); }
double orc_bt(double nu, double R) { return bt(nu, R); }
double orc_dB_dT(double nu, double T) {  // planck.jl:67-71
    const double x = PLANCK_C2 * nu / T, ex = std::exp(x);
    return PLANCK_C1 * PLANCK_C2 * (nu * nu * nu * nu) * ex / ((T * T) * (ex - 1.0) * (ex - 1.0));
}
double orc_cim_correction(double s) { return cim_corr(s); }
double orc_lit_correction(double s) { return lit_corr(s); }
void orc_layer_cg(double v1, double v2, double p1, double p2, double* vc, double* pc) {
    *vc = cg_column_vmr(v1, v2, p1, p2);
    *pc = cg_pressure(v1, v2, p1, p2);
}
double orc_cg_temperature_mass(double T1, double T2, double p1, double p2) {
    return cg_temperature_mass(T1, T2, p1, p2);
}
double orc_scan_angle_to_local_zenith(double scan) {  // geometry.jl:92-101
    const double s = (6371.0 + 817.0) / 6371.0 * std::sin(std::fabs(scan) * M_PI / 180.0);
    if (s > 1.0) return NAN;
    return std::asin(s) * 180.0 / M_PI;
}

int64_t orc_internal_grid(const orc_sounder* s, const orc_fm_options* o, double* nu0,
                          double* dnu_hi, int64_t* den) {
    InternalGrid ig = internal_grid(*s, *o);
    *nu0 = grid_at(ig.g, 0);
    *dnu_hi = ig.dnu_hi;
    *den = ig.g.den;
    return ig.g.n;
}
void orc_grid_values(double nu_start, double dnu_hi, int64_t den, int64_t i0, int64_t n, double* out) {
    Grid g{nu_start, dnu_hi, den, 0, 0, 0};
    if (den) { g.a_n = std::nearbyint(nu_start * den); g.s_n = std::nearbyint(dnu_hi * den); }
    for (int64_t i = 0; i < n; ++i) out[i] = grid_at(g, i0 + i);
}

int orc_voigt_xsec(const orc_line* lines, int64_t nL, const double* grid, int64_t n_nu, double T,
                   double p, double vs, double cutoff, int method, double x_far, double* sigma) {
    if (method < 1 || method > 3) return fail("method must be 1 (Weideman), 2 (PseudoVoigt) or 3 (FullFaddeeva)");
    voigt_xsec(lines, nL, grid, n_nu, T, p, vs, cutoff, method, x_far, sigma);
    return 0;
}
int64_t orc_reject_weak_lines(const orc_line* lines, int64_t nL, double T, double p, double coef,
                              double vs, double dptmn, uint8_t* keep) {
    return reject_weak(lines, nL, T, p, coef, vs, dptmn, keep);
}
int orc_lm_dispersive(const orc_line* lines, int64_t nL, const double* y0, const double* grid,
                      int64_t n_nu, double T, double p, double cutoff, double x_far, double* ds) {
    lm_dispersive(lines, nL, y0, grid, n_nu, T, p, cutoff, x_far, ds);
    return 0;
}
int orc_ils_kernel(double dnu, double opd, double fwhm, int apod, int64_t n_taps, double* out) {
    if (apod < 0 || apod > 3) return fail("unknown apodization");
    std::vector<double> k;
    ils_kernel(dnu, opd, fwhm, apod, k);
    if ((int64_t)k.size() != n_taps) return fail("n_taps mismatch");
    std::copy(k.begin(), k.end(), out);
    return 0;
}
int orc_rte(const double* grid, int64_t n_nu, int L, const double* tau, const double* T_lev,
            double T_sfc, double mu, double eps, int src, const double* T_ave, double* I) {
    if (!(mu > 0.0 && mu <= 1.0)) return fail("mu must be in (0, 1]");
    if (src != 0 && src != 1) return fail("source_function must be :cim or :toon");
    if (src == 0 && !T_ave) return fail(":cim source_function requires T_ave");
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n_nu; ++i)
        I[i] = rte_point(grid[i], i, n_nu, L, tau, T_lev, T_sfc, mu, eps, src, T_ave);
    return 0;
}

// sounder.jl:233-360
int orc_set_cia(int pair, int n_blocks, const double* T, const int64_t* off, const double* nu, const double* sg) {
    if (pair < 1 || pair > 3) return fail("CIA pair must be 1 (CO2-CO2), 2 (N2-N2) or 3 (O2-O2)");
    std::vector<CiaBlock> B;
    for (int b = 0; b < n_blocks; ++b) {
        CiaBlock c;
        c.T = T[b];
        c.nu.assign(nu + off[b], nu + off[b + 1]);
        c.sg.assign(sg + off[b], sg + off[b + 1]);
        if (c.nu.empty()) continue;
        c.numin = c.nu.front();
        c.numax = c.nu.back();
        B.push_back(std::move(c));
    }
    g_cia[pair - 1] = std::move(B);
    return 0;
}

static orc_lm_cb g_lm_cb = nullptr;
static void* g_lm_user = nullptr;
static int g_lm_species = 0;

int orc_set_lm_callback(int species, orc_lm_cb cb, void* user) {
    g_lm_cb = cb;
    g_lm_user = user;
    g_lm_species = species;
    return 0;
}

int orc_forward_model(int n_lev, const double* p_lev, const double* T_lev, int nps,
                      const int* psp, const double* pvmr, int n_lists, const int* lsp,
                      const int64_t* loff, const orc_line* lines, const double* y0,
                      const orc_sounder* s, const orc_fm_options* o, int64_t ch_begin,
                      int64_t ch_end, double* R_out, double* BT_out, double* tau_out,
                      int64_t* n_nu_window) {
    if (n_lev < 2) return fail("profile needs at least 2 levels");
    if (!(o->mu > 0.0 && o->mu <= 1.0)) return fail("mu must be in (0, 1]");
    if (o->T_method != 0 && o->T_method != 1) return fail("T_method must be :logp_at_pcg or :mass_weighted");
    if (o->source_function != 0 && o->source_function != 1) return fail("source_function must be :cim or :toon");
    if (o->apodization < 0 || o->apodization > 3) return fail("unknown apodization");
    const int L = n_lev - 1;
    InternalGrid ig = internal_grid(*s, *o);
    const Grid ch = make_grid(s->nu_min, s->nu_max, s->dnu);
    if (ch_end <= 0) { ch_begin = 0; ch_end = ch.n; }
    if (ch_begin < 0 || ch_end > ch.n || ch_begin >= ch_end) return fail("bad channel window");
    // channel wavenumbers and the hi-res index interval the window needs
    std::vector<double> nu_ch(ch_end - ch_begin);
    for (long c = ch_begin; c < ch_end; ++c) nu_ch[c - ch_begin] = grid_at(ch, c);
    const double dhi = ig.dnu_hi;
    const long n_hi = ig.g.n;
    const double nu_first = grid_at(ig.g, 0);
    auto idx_floor = [&](double nu) {
        long i = (long)std::floor((nu - nu_first) / dhi);
        i = std::max(0L, std::min(i, n_hi - 1));
        while (i > 0 && grid_at(ig.g, i) > nu) --i;
        while (i + 1 < n_hi && grid_at(ig.g, i + 1) <= nu) ++i;
        return i;
    };
    std::vector<double> kern;
    long n_half = 0;
    if (o->with_ils) {
        ils_kernel(dhi, s->opd_max, s->fwhm_gauss, o->apodization, kern);
        n_half = ((long)kern.size() - 1) / 2;
    }
    const long i_lo_ch = idx_floor(nu_ch.front());
    const long i_hi_ch = std::min(n_hi - 1, idx_floor(nu_ch.back()) + 1);
    const long w0 = std::max(0L, i_lo_ch - n_half);
    const long w1 = std::min(n_hi - 1, i_hi_ch + n_half);
    const long nw = w1 - w0 + 1;
    std::vector<double> grid(nw);
    for (long i = 0; i < nw; ++i) grid[i] = grid_at(ig.g, w0 + i);
    if (n_nu_window) *n_nu_window = nw;

    // layers.jl:133-178
    std::vector<double> p_mid(L), dp(L);
    for (int k = 0; k < L; ++k) { p_mid[k] = 0.5 * (p_lev[k] + p_lev[k + 1]); dp[k] = std::fabs(p_lev[k] - p_lev[k + 1]); }
    LogPInterp Ti(n_lev, p_lev, T_lev);
    std::vector<double> T_mid(L);
    for (int k = 0; k < L; ++k) T_mid[k] = Ti(p_mid[k]);
    std::vector<double> T_mass(L);
    for (int k = 0; k < L; ++k) T_mass[k] = cg_temperature_mass(T_lev[k], T_lev[k + 1], p_lev[k], p_lev[k + 1]);
    auto prof_index = [&](int sp) { for (int q = 0; q < nps; ++q) if (psp[q] == sp) return q; return -1; };

    std::vector<double> tau((size_t)L * nw, 0.0), sig(nw), ds(nw);
    for (int k = 0; k < L; ++k) {
        double* tk = tau.data() + (size_t)k * nw;
        for (int li = 0; li < n_lists; ++li) {
            const int sp = lsp[li];
            const int q = prof_index(sp);
            if (q < 0) continue;
            const double* v = pvmr + (size_t)q * n_lev;
            const double vmr = cg_column_vmr(v[k], v[k + 1], p_lev[k], p_lev[k + 1]);
            if (vmr == 0.0) continue;
            const double pcg = cg_pressure(v[k], v[k + 1], p_lev[k], p_lev[k + 1]);
            const double p_atm = pcg / 1013.25;
            const double Tcg = o->T_method == 1 ? T_mass[k] : Ti(pcg);
            const double vs = sp == 1 ? vmr : 0.0;
            const double coef = vmr * dp[k] * NAIR_PER_VMR;
            long ja = 0, jb = 0;
            reach_range(lines + loff[li], (long)(loff[li + 1] - loff[li]), grid.front(), grid.back(),
                        std::max(o->cutoff, o->lm_cutoff), ja, jb);
            const orc_line* ll = lines + loff[li] + ja;
            const long nL = jb - ja;
            const double* y0l = y0 ? y0 + loff[li] + ja : nullptr;
            // sounder.jl:294-300: DPTMIN is skipped for CO2 under any line-mixing model
            const bool lm_co2 = sp == 2 && o->line_mixing == 1;
            const bool no_dpt = sp == 2 && o->line_mixing != 0;
            const bool relmat = (o->line_mixing == 2 || o->line_mixing == 3) && g_lm_cb && sp == g_lm_species;
            std::vector<orc_line> kept;
            const orc_line* use = ll;
            long nuse = nL;
            if (o->dptmn > 0.0 && !no_dpt) {
                std::vector<uint8_t> keep(nL);
                reject_weak(ll, nL, Tcg, p_atm, coef, vs, o->dptmn, keep.data());
                for (long j = 0; j < nL; ++j) if (keep[j]) kept.push_back(ll[j]);
                use = kept.data();
                nuse = (long)kept.size();
            }
            if (lm_co2) {
                voigt_xsec(use, nuse, grid.data(), nw, Tcg, p_atm, 0.0, o->cutoff, 3, o->x_far, sig.data());
                if (y0) {
                    lm_dispersive(use, nuse, y0l, grid.data(), nw, Tcg, p_atm, o->lm_cutoff, o->x_far, ds.data());
                    for (long i = 0; i < nw; ++i) sig[i] = std::max(sig[i] + ds[i], 0.0);
                }
            } else if (relmat) {  // compute_voigt_{lm,vpw}_cross_sections, line_mixing.jl:1093-1110, 1351-1369
                voigt_xsec(use, nuse, grid.data(), nw, Tcg, p_atm, 0.0, o->cutoff, 3, o->x_far, sig.data());
                if (g_lm_cb(g_lm_user, Tcg, p_atm, grid.data(), nw, ds.data()) != 0) return fail("line-mixing callback failed");
                for (long i = 0; i < nw; ++i) sig[i] = std::max(sig[i] + ds[i], 0.0);
            } else if (nuse > 0) {
                voigt_xsec(use, nuse, grid.data(), nw, Tcg, p_atm, vs, o->cutoff, o->method, o->x_far, sig.data());
            } else {
                std::fill(sig.begin(), sig.end(), 0.0);
            }
            for (long i = 0; i < nw; ++i) tk[i] += sig[i] * coef;
        }
    }
    if (o->apply_continuum) {  // sounder.jl:310-322
        const int qh = prof_index(1), qc = prof_index(2);
        for (int k = 0; k < L; ++k) {
            double* tk = tau.data() + (size_t)k * nw;
            LogPInterp* dummy = nullptr; (void)dummy;
            auto vmid = [&](int q) {
                const double* v = pvmr + (size_t)q * n_lev;
                LogPInterp vi(n_lev, p_lev, v);
                return vi(p_mid[k]);
            };
            const double vh = qh >= 0 ? vmid(qh) : 0.0;
            const double vc = qc >= 0 ? vmid(qc) : 4.15e-4;
            const double dz = dp_to_dz_cm(dp[k], p_mid[k], T_mid[k]);
            if (o->continua & 1) h2o_continuum_add(grid.data(), nw, vh, p_mid[k], T_mid[k], dz, tk);
            if (o->continua & 2) co2_continuum_add(grid.data(), nw, vc, p_mid[k], T_mid[k], dz, tk);
            // CIA (:co2_cia, :n2, :o2) from the tables of orc_set_cia; zeros without them,
            // as the reference does when the data is absent (continuum.jl:268-272)
            cia_add(grid.data(), nw, o->continua, vh, vc, p_mid[k], T_mid[k], dz, tk);
        }
    }
    if (tau_out) std::copy(tau.begin(), tau.end(), tau_out);

    std::vector<double> T_ave(L);
    for (int k = 0; k < L; ++k) T_ave[k] = cg_temperature_mass(T_lev[k], T_lev[k + 1], p_lev[k], p_lev[k + 1]);
    const double Tsfc = std::isnan(o->T_sfc) ? T_lev[0] : o->T_sfc;
    std::vector<double> I(nw);
#pragma omp parallel for schedule(static)
    for (long i = 0; i < nw; ++i)
        I[i] = rte_point(grid[i], i, nw, L, tau.data(), T_lev, Tsfc, o->mu, o->eps_sfc,
                         o->source_function, T_ave.data());

    // ils.jl:131-153 evaluated at the nodes the channel interpolation reads,
    // then sounder.jl:372-377 (linear interpolation, flat outside) and planck.jl:53-57
    auto ils_at = [&](long ig_idx) {
        if (!o->with_ils) return I[ig_idx - w0];
        double acc = 0.0;
        for (long k = 0; k < (long)kern.size(); ++k) {
            const long j = ig_idx + (k - n_half);
            if (j < 0 || j >= n_hi) continue;
            acc += I[j - w0] * kern[k];
        }
        return acc * dhi;
    };
    const long nch = ch_end - ch_begin;
#pragma omp parallel for schedule(static)
    for (long c = 0; c < nch; ++c) {
        const double nu = nu_ch[c];
        double R;
        if (nu <= nu_first) R = ils_at(0);
        else if (nu >= grid_at(ig.g, n_hi - 1)) R = ils_at(n_hi - 1);
        else {
            const long i = idx_floor(nu);
            const double a = grid_at(ig.g, i), b = grid_at(ig.g, i + 1);
            const double w = (nu - a) / (b - a);
            const double r0 = ils_at(i);
            R = w == 0.0 ? r0 : r0 * (1.0 - w) + ils_at(i + 1) * w;
        }
        R_out[c] = R;
        BT_out[c] = bt(nu, R);
    }
    return 0;
}

// vmr_jacobian.jl:152-505 (analytic_jacobian) with schwarzschild_jacobian.jl:66-266
// on channels [ch_begin, ch_end).  State layout (state_vector.jl:253-309):
// [T (n_lev) if include_T][per retrieved species: VMR or log VMR (n_lev)][T_sfc][eps].
// K is [n_state][n_window_channels] (the column-major n_ch x n_state Jacobian.K).
int orc_analytic_jacobian(int n_lev, const double* p_lev, const double* T_lev, int nps, const int* psp,
                          const double* pvmr, int n_lists, const int* lsp, const int64_t* loff,
                          const orc_line* lines, const double* y0, const orc_sounder* s,
                          const orc_fm_options* o, int n_retr, const int* retr, int include_T,
                          int include_tsfc, int include_eps, int log_vmr, int vmr_coupling, int observable,
                          int64_t ch_begin, int64_t ch_end, double* K, double* y_out) {
    if (n_lev < 2) return fail("profile needs at least 2 levels");
    if (!(o->mu > 0.0 && o->mu <= 1.0)) return fail("mu must be in (0, 1]");
    const int L = n_lev - 1;
    const int src = o->source_function;
    InternalGrid ig = internal_grid(*s, *o);
    const Grid ch = make_grid(s->nu_min, s->nu_max, s->dnu);
    if (ch_end <= 0) { ch_begin = 0; ch_end = ch.n; }
    if (ch_begin < 0 || ch_end > ch.n || ch_begin >= ch_end) return fail("bad channel window");
    const double dhi = ig.dnu_hi;
    const long n_hi = ig.g.n;
    const double nu_first = grid_at(ig.g, 0);
    auto idx_floor = [&](double nu) {
        long i = (long)std::floor((nu - nu_first) / dhi);
        i = std::max(0L, std::min(i, n_hi - 1));
        while (i > 0 && grid_at(ig.g, i) > nu) --i;
        while (i + 1 < n_hi && grid_at(ig.g, i + 1) <= nu) ++i;
        return i;
    };
    std::vector<double> kern;
    long n_half = 0;
    if (o->with_ils) { ils_kernel(dhi, s->opd_max, s->fwhm_gauss, o->apodization, kern); n_half = ((long)kern.size() - 1) / 2; }
    const long nch = ch_end - ch_begin;
    std::vector<double> nu_ch(nch);
    for (long c = 0; c < nch; ++c) nu_ch[c] = grid_at(ch, ch_begin + c);
    const long w0 = std::max(0L, idx_floor(nu_ch.front()) - n_half);
    const long w1 = std::min(n_hi - 1, std::min(n_hi - 1, idx_floor(nu_ch.back()) + 1) + n_half);
    const long nw = w1 - w0 + 1;
    std::vector<double> grid(nw);
    for (long i = 0; i < nw; ++i) grid[i] = grid_at(ig.g, w0 + i);

    // layer properties (layers.jl:133-178)
    std::vector<double> p_mid(L), dp(L), T_mid(L), T_ave(L), fracs(L);
    LogPInterp Ti(n_lev, p_lev, T_lev);
    for (int k = 0; k < L; ++k) {
        p_mid[k] = 0.5 * (p_lev[k] + p_lev[k + 1]);
        dp[k] = std::fabs(p_lev[k] - p_lev[k + 1]);
        T_mid[k] = Ti(p_mid[k]);
        T_ave[k] = cg_temperature_mass(T_lev[k], T_lev[k + 1], p_lev[k], p_lev[k + 1]);
        fracs[k] = cg_mass_frac(p_lev[k], p_lev[k + 1]);
    }
    auto prof_index = [&](int sp) { for (int q = 0; q < nps; ++q) if (psp[q] == sp) return q; return -1; };
    auto is_retr = [&](int sp) { for (int r = 0; r < n_retr; ++r) if (retr[r] == sp) return true; return false; };

    const size_t NL = (size_t)L * nw;
    std::vector<double> tau(NL, 0.0);
    std::map<int, std::vector<double>> tau_sp, dTcg, dtdp, dtdTc, dtdvs, wT;
    for (int li = 0; li < n_lists; ++li) {
        const int sp = lsp[li];
        if (include_T) { dTcg[sp].assign(NL, 0.0); wT[sp].assign(L, 0.0); }
        if (is_retr(sp)) {
            tau_sp[sp].assign(NL, 0.0);
            if (vmr_coupling) { dtdp[sp].assign(NL, 0.0); dtdTc[sp].assign(NL, 0.0); dtdvs[sp].assign(NL, 0.0); }
        }
    }
    for (int k = 0; k < L; ++k) {
        for (int li = 0; li < n_lists; ++li) {
            const int sp = lsp[li];
            const int q = prof_index(sp);
            if (q < 0) continue;
            const double* v = pvmr + (size_t)q * n_lev;
            const double vmr = cg_column_vmr(v[k], v[k + 1], p_lev[k], p_lev[k + 1]);
            if (vmr == 0.0) continue;
            const double pcg = cg_pressure(v[k], v[k + 1], p_lev[k], p_lev[k + 1]);
            const double p_atm = pcg / 1013.25;
            const double Tcg = o->T_method == 1 ? T_ave[k] : Ti(pcg);
            const double vs = sp == 1 ? vmr : 0.0;
            const double coef = vmr * dp[k] * NAIR_PER_VMR;
            long ja = 0, jb = 0;
            reach_range(lines + loff[li], (long)(loff[li + 1] - loff[li]), grid.front(), grid.back(),
                        std::max(o->cutoff, o->lm_cutoff), ja, jb);
            const orc_line* ll = lines + loff[li] + ja;
            const long nL = jb - ja;
            const bool lm = sp == 2 && o->line_mixing == 1;
            Grad g;
            species_grad(ll, nL, y0 ? y0 + loff[li] + ja : nullptr, lm, grid.data(), nw, Tcg, p_atm, vs, o->cutoff,
                         o->lm_cutoff, o->x_far, g);
            const size_t base = (size_t)k * nw;
            if (include_T) {
                for (long i = 0; i < nw; ++i) dTcg[sp][base + i] = g.dT[i] * coef;
                wT[sp][k] = o->T_method == 1 ? cg_mass_frac(p_lev[k], p_lev[k + 1])
                                             : std::log(pcg / p_lev[k]) / std::log(p_lev[k + 1] / p_lev[k]);
            }
            if (vmr_coupling && is_retr(sp))
                for (long i = 0; i < nw; ++i) {
                    dtdp[sp][base + i] = g.dp[i] * (coef / 1013.25);
                    dtdTc[sp][base + i] = g.dT[i] * coef;
                    dtdvs[sp][base + i] = g.dv[i] * coef;
                }
            for (long i = 0; i < nw; ++i) {
                const double c = g.s[i] * coef;
                tau[base + i] += c;
                if (is_retr(sp)) tau_sp[sp][base + i] = c;
            }
        }
    }
    // continua and their central differences (vmr_jacobian.jl:294-345)
    const int qh = prof_index(1), qc = prof_index(2);
    auto vmid = [&](int q, int k, double dflt) {
        if (q < 0) return dflt;
        LogPInterp vi(n_lev, p_lev, pvmr + (size_t)q * n_lev);
        return vi(p_mid[k]);
    };
    auto cont_layer = [&](int k, double vh, double vc, double Tm, std::vector<double>& out) {
        out.assign(nw, 0.0);
        const double dz = dp_to_dz_cm(dp[k], p_mid[k], Tm);
        if (o->continua & 1) h2o_continuum_add(grid.data(), nw, vh, p_mid[k], Tm, dz, out.data());
        if (o->continua & 2) co2_continuum_add(grid.data(), nw, vc, p_mid[k], Tm, dz, out.data());
        cia_add(grid.data(), nw, o->continua, vh, vc, p_mid[k], Tm, dz, out.data());
    };
    const bool cvh = o->apply_continuum && vmr_coupling && is_retr(1);
    const bool cvc = o->apply_continuum && vmr_coupling && is_retr(2);
    const bool cT = o->apply_continuum && include_T;
    std::vector<double> dcvh(cvh ? NL : 0), dcvc(cvc ? NL : 0), dcT(cT ? NL : 0), wM(L, 0.0), t1, t2;
    if (o->apply_continuum)
        for (int k = 0; k < L; ++k) {
            const double vh = vmid(qh, k, 0.0), vc = vmid(qc, k, 4.15e-4);
            cont_layer(k, vh, vc, T_mid[k], t1);
            for (long i = 0; i < nw; ++i) tau[(size_t)k * nw + i] += t1[i];
            wM[k] = std::log(p_mid[k] / p_lev[k]) / std::log(p_lev[k + 1] / p_lev[k]);
            if (cvh) {
                const double h = std::max(std::fabs(vh), 1e-30) * 1e-6;
                cont_layer(k, vh + h, vc, T_mid[k], t1); cont_layer(k, vh - h, vc, T_mid[k], t2);
                for (long i = 0; i < nw; ++i) dcvh[(size_t)k * nw + i] = (t1[i] - t2[i]) / (2 * h);
            }
            if (cvc) {
                const double h = std::max(std::fabs(vc), 1e-30) * 1e-6;
                cont_layer(k, vh, vc + h, T_mid[k], t1); cont_layer(k, vh, vc - h, T_mid[k], t2);
                for (long i = 0; i < nw; ++i) dcvc[(size_t)k * nw + i] = (t1[i] - t2[i]) / (2 * h);
            }
            if (cT) {
                const double h = 0.05;
                cont_layer(k, vh, vc, T_mid[k] + h, t1); cont_layer(k, vh, vc, T_mid[k] - h, t2);
                for (long i = 0; i < nw; ++i) dcT[(size_t)k * nw + i] = (t1[i] - t2[i]) / (2 * h);
            }
        }

    // schwarzschild_rte_jacobian (schwarzschild_jacobian.jl:66-266)
    const double Tsfc = std::isnan(o->T_sfc) ? T_lev[0] : o->T_sfc;
    const double mu = o->mu, eps = o->eps_sfc, invmu = 1.0 / mu;
    std::vector<double> I(nw), dIdtau(NL), dIdTl((size_t)n_lev * nw, 0.0), dIdTs(nw), dIde(nw);
#pragma omp parallel for schedule(static)
    for (long i = 0; i < nw; ++i) {
        const double nu = grid[i];
        std::vector<double> Tr(L + 1), gk(L), em(L), dem(L);
        Tr[L] = 1.0;
        for (int k = L - 1; k >= 0; --k) Tr[k] = Tr[k + 1] * std::exp(-tau[(size_t)k * nw + i] / mu);
        const double Bs = planck(nu, Tsfc);
        double Ii = eps * Bs * Tr[0];
        dIde[i] = Bs * Tr[0];
        dIdTs[i] = eps * dB_dT(nu, Tsfc) * Tr[0];
        double Ib = eps * Bs * Tr[0];
        for (int m = 0; m < L; ++m) {
            const double a = tau[(size_t)m * nw + i] * invmu, w = std::exp(-a), u = 1.0 - w, Tt = Tr[m + 1];
            double e, dea;
            if (src == 0) {
                const double Ba = planck(nu, T_ave[m]), Bt = planck(nu, T_lev[m + 1]);
                const double f = cim_corr(a), fp = cim_corr_deriv(a), core = Ba + (Bt - Ba) * f;
                e = u * core;
                dea = w * core + u * (Bt - Ba) * fp;
                const double cavg = Tt * u * (1.0 - f) * dB_dT(nu, T_ave[m]);
                dIdTl[(size_t)m * nw + i] += cavg * (1.0 - fracs[m]);
                dIdTl[(size_t)(m + 1) * nw + i] += cavg * fracs[m] + Tt * u * f * dB_dT(nu, T_lev[m + 1]);
            } else {
                const double Bb = planck(nu, T_lev[m]), Bt = planck(nu, T_lev[m + 1]);
                const double fl = lit_corr(a), flp = lit_corr_deriv(a);
                e = Bt * u + (Bb - Bt) * fl;
                dea = Bt * w + (Bb - Bt) * flp;
                dIdTl[(size_t)m * nw + i] += Tt * fl * dB_dT(nu, T_lev[m]);
                dIdTl[(size_t)(m + 1) * nw + i] += Tt * (u - fl) * dB_dT(nu, T_lev[m + 1]);
            }
            dIdtau[(size_t)m * nw + i] = invmu * (-Ib + Tt * dea);
            Ii += Tt * e;
            Ib += Tt * e;
        }
        if (eps < 1.0) {  // schwarzschild_jacobian.jl:189-266
            const double refl = 1.0 - eps, T1 = Tr[0];
            double g = 1.0, Id = 0.0;
            for (int k = 0; k < L; ++k) {
                const double a = tau[(size_t)k * nw + i] * invmu, w = std::exp(-a), u = 1.0 - w;
                gk[k] = g;
                if (src == 0) {
                    const double Ba = planck(nu, T_ave[k]), Bb = planck(nu, T_lev[k]);
                    const double f = cim_corr(a), fp = cim_corr_deriv(a), core = Ba + (Bb - Ba) * f;
                    em[k] = u * core;
                    dem[k] = w * core + u * (Bb - Ba) * fp;
                    const double cavg = refl * T1 * g * u * (1.0 - f) * dB_dT(nu, T_ave[k]);
                    dIdTl[(size_t)k * nw + i] += cavg * (1.0 - fracs[k]) + refl * T1 * g * u * f * dB_dT(nu, T_lev[k]);
                    dIdTl[(size_t)(k + 1) * nw + i] += cavg * fracs[k];
                } else {
                    const double Bb = planck(nu, T_lev[k]), Bt = planck(nu, T_lev[k + 1]);
                    const double fl = lit_corr(a), flp = lit_corr_deriv(a);
                    em[k] = Bb * u + (Bt - Bb) * fl;
                    dem[k] = Bb * w + (Bt - Bb) * flp;
                    dIdTl[(size_t)k * nw + i] += refl * T1 * g * (u - fl) * dB_dT(nu, T_lev[k]);
                    dIdTl[(size_t)(k + 1) * nw + i] += refl * T1 * g * fl * dB_dT(nu, T_lev[k + 1]);
                }
                Id += g * em[k];
                g *= w;
            }
            Ii += refl * Id * T1;
            dIde[i] += -Id * T1;
            double above = 0.0;
            for (int m = L - 1; m >= 0; --m) {
                dIdtau[(size_t)m * nw + i] += refl * invmu * T1 * (-above + gk[m] * dem[m] - Id);
                above += gk[m] * em[m];
            }
        }
        I[i] = Ii;
    }

    // channel tail (vmr_jacobian.jl:359-380): ILS at the nodes the resampling reads
    std::vector<long> c_i(nch);
    std::vector<double> c_w(nch);
    for (long c = 0; c < nch; ++c) {
        const double nu = nu_ch[c];
        if (nu <= nu_first) { c_i[c] = 0; c_w[c] = -1; }
        else if (nu >= grid_at(ig.g, n_hi - 1)) { c_i[c] = n_hi - 1; c_w[c] = -1; }
        else {
            const long i = idx_floor(nu);
            const double a = grid_at(ig.g, i), b = grid_at(ig.g, i + 1);
            c_i[c] = i;
            c_w[c] = (nu - a) / (b - a);
        }
    }
    auto ils_at = [&](const std::vector<double>& col, long gi) {
        if (!o->with_ils) return col[gi - w0];
        double acc = 0.0;
        for (long k = 0; k < (long)kern.size(); ++k) {
            const long j = gi + (k - n_half);
            if (j < 0 || j >= n_hi) continue;
            acc += col[j - w0] * kern[k];
        }
        return acc * dhi;
    };
    auto resample = [&](const std::vector<double>& col, long c) {
        const double r0 = ils_at(col, c_i[c]);
        if (c_w[c] <= 0.0) return r0;
        return r0 * (1.0 - c_w[c]) + ils_at(col, c_i[c] + 1) * c_w[c];
    };
    std::vector<double> Rc(nch), dbt(nch);
    for (long c = 0; c < nch; ++c) {
        Rc[c] = resample(I, c);
        dbt[c] = observable == 0 ? dBT_dR(nu_ch[c], Rc[c]) : 1.0;
        y_out[c] = observable == 0 ? bt(nu_ch[c], Rc[c]) : Rc[c];
    }
    int col = 0;
    auto emit = [&](const std::vector<double>& dI, double scale) {
#pragma omp parallel for schedule(static)
        for (long c = 0; c < nch; ++c) K[(size_t)col * nch + c] = resample(dI, c) * dbt[c] * scale;
        ++col;
    };
    std::vector<double> dI(nw);
    if (include_T) {
        for (int j = 0; j < n_lev; ++j) {
            for (long i = 0; i < nw; ++i) dI[i] = dIdTl[(size_t)j * nw + i];
            for (auto& e : dTcg) {
                const std::vector<double>& M = e.second;
                const std::vector<double>& w = wT[e.first];
                if (j < L) for (long i = 0; i < nw; ++i) dI[i] += dIdtau[(size_t)j * nw + i] * M[(size_t)j * nw + i] * (1.0 - w[j]);
                if (j >= 1) for (long i = 0; i < nw; ++i) dI[i] += dIdtau[(size_t)(j - 1) * nw + i] * M[(size_t)(j - 1) * nw + i] * w[j - 1];
            }
            if (cT) {
                if (j < L) for (long i = 0; i < nw; ++i) dI[i] += dIdtau[(size_t)j * nw + i] * dcT[(size_t)j * nw + i] * (1.0 - wM[j]);
                if (j >= 1) for (long i = 0; i < nw; ++i) dI[i] += dIdtau[(size_t)(j - 1) * nw + i] * dcT[(size_t)(j - 1) * nw + i] * wM[j - 1];
            }
            emit(dI, 1.0);
        }
    }
    for (int r = 0; r < n_retr; ++r) {
        const int sp = retr[r];
        const int q = prof_index(sp);
        if (q < 0) return fail("profile is missing a retrieved species");
        const double* vl = pvmr + (size_t)q * n_lev;
        const bool has_lbl = tau_sp.count(sp) > 0;
        std::vector<double> vcg(L), gV1(L), gV2(L), gP1(L, 0.0), gP2(L, 0.0), gT1(L, 0.0), gT2(L, 0.0);
        for (int k = 0; k < L; ++k) {
            const double v1 = vl[k], v2 = vl[k + 1], p1 = p_lev[k], p2 = p_lev[k + 1];
            vcg[k] = cg_column_vmr(v1, v2, p1, p2);
            cg_column_vmr_grad(v1, v2, p1, p2, gV1[k], gV2[k]);
            if (vmr_coupling) {
                const double h1 = std::max(std::fabs(v1), 1e-300) * 1e-6, h2 = std::max(std::fabs(v2), 1e-300) * 1e-6;
                gP1[k] = (cg_pressure(v1 + h1, v2, p1, p2) - cg_pressure(v1 - h1, v2, p1, p2)) / (2 * h1);
                gP2[k] = (cg_pressure(v1, v2 + h2, p1, p2) - cg_pressure(v1, v2 - h2, p1, p2)) / (2 * h2);
                if (o->T_method != 1) {
                    const double dTdp = (T_lev[k + 1] - T_lev[k]) / (cg_pressure(v1, v2, p1, p2) * std::log(p2 / p1));
                    gT1[k] = dTdp * gP1[k];
                    gT2[k] = dTdp * gP2[k];
                }
            }
        }
        const std::vector<double>* dcv = sp == 1 ? (cvh ? &dcvh : nullptr) : (sp == 2 ? (cvc ? &dcvc : nullptr) : nullptr);
        for (int j = 0; j < n_lev; ++j) {
            std::fill(dI.begin(), dI.end(), 0.0);
            auto add_layer = [&](int k, double gV, double gP, double gT) {
                if (!has_lbl || vcg[k] == 0.0) return;
                const std::vector<double>& ts = tau_sp[sp];
                for (long i = 0; i < nw; ++i) dI[i] += dIdtau[(size_t)k * nw + i] * ts[(size_t)k * nw + i] * (gV / vcg[k]);
                if (vmr_coupling) {
                    for (long i = 0; i < nw; ++i)
                        dI[i] += dIdtau[(size_t)k * nw + i] * (dtdp[sp][(size_t)k * nw + i] * gP + dtdTc[sp][(size_t)k * nw + i] * gT);
                    if (sp == 1)
                        for (long i = 0; i < nw; ++i) dI[i] += dIdtau[(size_t)k * nw + i] * dtdvs[sp][(size_t)k * nw + i] * gV;
                }
            };
            if (j < L) add_layer(j, gV1[j], gP1[j], gT1[j]);
            if (j >= 1) add_layer(j - 1, gV2[j - 1], gP2[j - 1], gT2[j - 1]);
            if (dcv) {
                if (j < L) for (long i = 0; i < nw; ++i) dI[i] += dIdtau[(size_t)j * nw + i] * (*dcv)[(size_t)j * nw + i] * (1.0 - wM[j]);
                if (j >= 1) for (long i = 0; i < nw; ++i) dI[i] += dIdtau[(size_t)(j - 1) * nw + i] * (*dcv)[(size_t)(j - 1) * nw + i] * wM[j - 1];
            }
            emit(dI, log_vmr ? vl[j] : 1.0);
        }
    }
    if (include_tsfc) emit(dIdTs, 1.0);
    if (include_eps) emit(dIde, 1.0);
    return 0;
}

}  // extern "C"
