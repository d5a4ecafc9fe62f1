// relmat.cpp -- host side of relaxation-matrix line mixing: the relmat data model,
// the temperature-dependent relaxation matrix W(T), first-order Y(T), the VP_W
// eigenmodes, and the pole lists the device pole sum evaluates.
//
// Follows src/CrossSections/line_mixing.jl of IRSounderLBL.jl:
//   _build_coupling                  :530-578   (once per band, at upload)
//   _build_W_matrix                  :607-700
//   _calc_W_and_Y                    :712-738
//   _band_eff_strength               :804-811
//   band_modes                       :892-955
//   _diagonal_band_modes             :1030-1052
//   _append_dispersive_lines!        :1193-1220
//   _vpw_perturbation, compute_lm_dispersive_correction band filters :1120-1154, :1303-1337
//
// The eigendecomposition of M = diag(nu) + i p W (complex, non-Hermitian) is our own:
// Householder reduction to Hessenberg form, complex single-shift QR with Wilkinson
// shifts and deflation to the Schur form, eigenvectors by back substitution on the
// triangular factor, then the amplitudes a = X^T d and b = X^-1 (rho d) by an LU solve
// with partial pivoting.  Amplitudes A = a b do not depend on how the eigenvector
// columns are scaled.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <complex>
#include <map>
#include <numeric>
#include <tuple>

#include "irs_internal.h"

namespace irs {

using cd = std::complex<double>;

namespace {

constexpr double kT0 = 296.0;         // line_mixing.jl:30
constexpr double kCT = 1.4388;        // line_mixing.jl:31
constexpr double kCtGamD = 3.5812e-7; // line_mixing.jl:755
constexpr double kSqrtLn2 = 0.83255461115769775635;
constexpr double kInvSqrtPi = 0.56418958354775628695;

// isotopologue masses (amu), line_mixing.jl:743-753; unknown -> 44
double mass_amu(int mol, int iso) {
    static const std::map<std::pair<int, int>, double> m = {
        {{2, 1}, 43.98983}, {{2, 2}, 44.99318}, {{2, 3}, 45.99398}, {{2, 4}, 44.99403},
        {{2, 5}, 45.99706}, {{2, 6}, 44.99706}, {{2, 7}, 47.99832}, {{2, 8}, 47.00134},
        {{2, 9}, 48.00196}, {{2, 10}, 47.00427}, {{6, 1}, 16.031300}, {{6, 2}, 17.034655},
        {{6, 3}, 17.037475}, {{6, 4}, 18.040830}};
    auto it = m.find({mol, iso});
    return it == m.end() ? 44.0 : it->second;
}

bool decoupled(int li, int lf) { return li > 8 || lf > 8 || std::abs(li - lf) > 1; }

int branch_type(int j, int jf) { return j > jf ? 0 : (j == jf ? 1 : 2); }  // P, Q, R

// lower-state populations at T (line_mixing.jl:619-624)
void populations(const RelmatBandHost& b, double T, double q_ratio, std::vector<double>& popu) {
    const size_t n = b.lines.size();
    popu.resize(n);
    for (size_t i = 0; i < n; ++i)
        popu[i] = b.lines[i].popu_t0 * q_ratio * std::exp(-kCT * b.lines[i].e_lower * (1.0 / T - 1.0 / kT0));
}

double gamma_T(const irs_relmat_line& l, double T) { return l.gv_air * std::pow(kT0 / T, (double)l.n_air); }

// _build_W_matrix (:607-700).  W row-major, W[i*n + j] = the reference's W[i, j].
void build_w(const RelmatBandHost& b, double T, double q_ratio, std::vector<double>& W, std::vector<double>& popu) {
    const int n = (int)b.lines.size();
    populations(b, T, q_ratio, popu);
    W.assign((size_t)n * n, 0.0);
    if (decoupled(b.li, b.lf)) {
        for (int i = 0; i < n; ++i) W[(size_t)i * n + i] = gamma_T(b.lines[i], T);
        return;
    }
    // intensity order, descending, stable (sortperm(S_eff, rev=true))
    std::vector<double> s_eff(n);
    for (int i = 0; i < n; ++i) s_eff[i] = b.lines[i].nu * popu[i] * b.lines[i].dipo_t * b.lines[i].dipo_t;
    std::vector<int> ord(n);
    std::iota(ord.begin(), ord.end(), 0);
    std::stable_sort(ord.begin(), ord.end(), [&](int a, int c) { return s_eff[a] > s_eff[c]; });
    const double dlg = std::log(kT0 / T);
    for (int ir = 0; ir < n; ++ir) {  // pair loop in intensity order (last writer wins)
        const int i = ord[ir];
        for (int t = b.row_ptr[i]; t < b.row_ptr[i + 1]; ++t) {
            const int j = b.col[t];
            const double ycal = std::exp(b.w0r[t] - b.b0r[t] * dlg);
            W[(size_t)j * n + i] = ycal;
            W[(size_t)i * n + j] = ycal * popu[i] / popu[j];
        }
    }
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j)
            if (i != j) W[(size_t)i * n + j] = -std::fabs(W[(size_t)i * n + j]);
    for (int i = 0; i < n; ++i) W[(size_t)i * n + i] = gamma_T(b.lines[i], T);
    // sum-rule renormalisation in intensity order (:676-697)
    const bool sym = b.isot > 2 && b.isot != 7 && b.isot != 10;
    for (int ir = 0; ir < n; ++ir) {
        const int i = ord[ir];
        const int ji = b.lines[i].ji;
        double sum_lw = 0.0, sum_up = 0.0;
        for (int irp = 0; irp < n; ++irp) {
            const int j = ord[irp];
            if (sym && std::abs(ji - (int)b.lines[j].ji) % 2 != 0) continue;
            const double v = std::fabs(b.lines[j].dipo0) * W[(size_t)j * n + i];
            if (irp > ir) sum_lw += v; else sum_up += v;
        }
        if (sum_lw == 0.0) continue;
        const double ratio = -sum_up / sum_lw;
        for (int irp = ir + 1; irp < n; ++irp) {
            const int j = ord[irp];
            W[(size_t)j * n + i] *= ratio;
            W[(size_t)i * n + j] = W[(size_t)j * n + i] * popu[i] / popu[j];
        }
    }
}

// _calc_W_and_Y (:712-738)
void calc_y(const RelmatBandHost& b, double T, double q_ratio, std::vector<double>& Y) {
    const int n = (int)b.lines.size();
    Y.assign(n, 0.0);
    if (n == 0 || decoupled(b.li, b.lf)) return;
    std::vector<double> W, popu;
    build_w(b, T, q_ratio, W, popu);
    for (int i = 0; i < n; ++i) {
        double s = 0.0;
        for (int j = 0; j < n; ++j) {
            if (j == i) continue;
            double dn = b.lines[i].nu - b.lines[j].nu;
            if (std::fabs(dn) < 1e-4) dn = (dn >= 0.0 ? 1.0 : -1.0) * 1e-4;
            s += 2.0 * std::fabs(b.lines[j].dipo_t) / std::fabs(b.lines[i].dipo_t) * (1.0 / dn) * W[(size_t)j * n + i];
        }
        Y[i] = s;
    }
}

// ------------------------------------------------------------ complex eigenproblem
inline double abs1(cd z) { return std::fabs(z.real()) + std::fabs(z.imag()); }

// A (row-major n x n) -> upper Hessenberg H = Q^H A Q by Householder reflections.
// Qt holds Q transposed (Qt[j*n + r] = Q[r][j]) so that every update below runs along
// contiguous memory.
void hessenberg(int n, std::vector<cd>& A, std::vector<cd>& Qt) {
    Qt.assign((size_t)n * n, cd(0.0));
    for (int i = 0; i < n; ++i) Qt[(size_t)i * n + i] = 1.0;
    std::vector<cd> v(n), s(n);
    for (int k = 0; k + 2 < n; ++k) {
        const int m = n - k - 1;
        double xn2 = 0.0;
        for (int i = 0; i < m; ++i) xn2 += std::norm(A[(size_t)(k + 1 + i) * n + k]);
        if (xn2 == 0.0) continue;
        const double xn = std::sqrt(xn2);
        const cd x0 = A[(size_t)(k + 1) * n + k];
        const cd ph = std::abs(x0) > 0.0 ? x0 / std::abs(x0) : cd(1.0);
        const cd alpha = -ph * xn;
        for (int i = 0; i < m; ++i) v[i] = A[(size_t)(k + 1 + i) * n + k];
        v[0] -= alpha;
        double vn2 = 0.0;
        for (int i = 0; i < m; ++i) vn2 += std::norm(v[i]);
        if (vn2 == 0.0) continue;
        const double tau = 2.0 / vn2;
        // A := (I - tau v v^H) A on rows k+1.., columns k..: s = tau v^H A, then A -= v s
        std::fill(s.begin() + k, s.end(), cd(0.0));
        for (int i = 0; i < m; ++i) {
            const cd cv = std::conj(v[i]) * tau;
            const cd* row = &A[(size_t)(k + 1 + i) * n];
            for (int j = k; j < n; ++j) s[j] += cv * row[j];
        }
        for (int i = 0; i < m; ++i) {
            cd* row = &A[(size_t)(k + 1 + i) * n];
            for (int j = k; j < n; ++j) row[j] -= v[i] * s[j];
        }
        // A := A (I - tau v v^H) on all rows, columns k+1..
        for (int r = 0; r < n; ++r) {
            cd* row = &A[(size_t)r * n + k + 1];
            cd t = 0.0;
            for (int i = 0; i < m; ++i) t += row[i] * v[i];
            t *= tau;
            for (int i = 0; i < m; ++i) row[i] -= t * std::conj(v[i]);
        }
        // Q := Q (I - tau v v^H), i.e. rows k+1.. of Qt: Qt -= conj(v) (tau v^T Qt)
        std::fill(s.begin(), s.end(), cd(0.0));
        for (int i = 0; i < m; ++i) {
            const cd cv = v[i] * tau;
            const cd* row = &Qt[(size_t)(k + 1 + i) * n];
            for (int r = 0; r < n; ++r) s[r] += cv * row[r];
        }
        for (int i = 0; i < m; ++i) {
            const cd cv = std::conj(v[i]);
            cd* row = &Qt[(size_t)(k + 1 + i) * n];
            for (int r = 0; r < n; ++r) row[r] -= cv * s[r];
        }
        A[(size_t)(k + 1) * n + k] = alpha;
        for (int i = 1; i < m; ++i) A[(size_t)(k + 1 + i) * n + k] = 0.0;
    }
}

// Rotation G = [c s; -conj(s) c] with G (x, y)^T = (r, 0)^T.
inline void givens(cd x, cd y, double& c, cd& s) {
    const double ax = std::abs(x), ay = std::abs(y);
    if (ay == 0.0) { c = 1.0; s = 0.0; return; }
    if (ax == 0.0) { c = 0.0; s = std::conj(y) / ay; return; }
    const double nr = std::hypot(ax, ay);
    c = ax / nr;
    s = (x / ax) * std::conj(y) / nr;
}

// Hessenberg H -> upper triangular T = Z^H A Z; Zt (Z transposed) enters holding Q.
bool schur(int n, std::vector<cd>& H, std::vector<cd>& Zt) {
    const double eps = DBL_EPSILON;
    double hnorm = 0.0;
    for (auto& h : H) hnorm = std::max(hnorm, abs1(h));
    if (hnorm == 0.0) return true;
    int hi = n - 1, its = 0, total = 0;
    while (hi > 0) {
        int l = hi;
        for (; l > 0; --l) {
            double s = abs1(H[(size_t)(l - 1) * n + l - 1]) + abs1(H[(size_t)l * n + l]);
            if (s == 0.0) s = hnorm;
            if (abs1(H[(size_t)l * n + l - 1]) <= eps * s) break;
        }
        if (l > 0) H[(size_t)l * n + l - 1] = 0.0;
        if (l == hi) { --hi; its = 0; continue; }
        if (++total > 100 * n) return false;
        ++its;
        cd mu;
        if (its % 10 == 0) {  // exceptional shift
            mu = H[(size_t)hi * n + hi] + 0.75 * std::fabs(H[(size_t)hi * n + hi - 1].real()) +
                 0.75 * std::fabs(H[(size_t)hi * n + hi - 1].imag());
        } else {  // eigenvalue of the trailing 2x2 block nearer its last diagonal element
            const cd a = H[(size_t)(hi - 1) * n + hi - 1], b = H[(size_t)(hi - 1) * n + hi];
            const cd c = H[(size_t)hi * n + hi - 1], d = H[(size_t)hi * n + hi];
            const cd half = 0.5 * (a - d);
            const cd disc = std::sqrt(half * half + b * c);
            const cd m1 = d + half + disc, m2 = d + half - disc;
            mu = std::abs(m1 - d) < std::abs(m2 - d) ? m1 : m2;
        }
        for (int k = l; k < hi; ++k) {  // implicit single-shift QR sweep (bulge chase)
            cd x, y;
            if (k == l) { x = H[(size_t)l * n + l] - mu; y = H[(size_t)(l + 1) * n + l]; }
            else { x = H[(size_t)k * n + k - 1]; y = H[(size_t)(k + 1) * n + k - 1]; }
            double c;
            cd s;
            givens(x, y, c, s);
            const cd sc = std::conj(s);
            cd* r0 = &H[(size_t)k * n];
            cd* r1 = &H[(size_t)(k + 1) * n];
            for (int j = (k == l ? l : k - 1); j < n; ++j) {
                const cd h1 = r0[j], h2 = r1[j];
                r0[j] = c * h1 + s * h2;
                r1[j] = -sc * h1 + c * h2;
            }
            const int rmax = std::min(k + 2, hi);
            for (int r = 0; r <= rmax; ++r) {
                cd* row = &H[(size_t)r * n + k];
                const cd h1 = row[0], h2 = row[1];
                row[0] = h1 * c + h2 * sc;
                row[1] = -h1 * s + h2 * c;
            }
            cd* z0 = &Zt[(size_t)k * n];
            cd* z1 = &Zt[(size_t)(k + 1) * n];
            for (int r = 0; r < n; ++r) {
                const cd a = z0[r], b = z1[r];
                z0[r] = a * c + b * sc;
                z1[r] = -a * s + b * c;
            }
            if (k > l) H[(size_t)(k + 1) * n + k - 1] = 0.0;
        }
    }
    return true;
}

// Eigen-decomposition of M: lam[k], X[i*n + k] (column k = eigenvector k).
bool eig(int n, std::vector<cd> M, std::vector<cd>& lam, std::vector<cd>& X) {
    std::vector<cd> Zt;
    hessenberg(n, M, Zt);
    if (!schur(n, M, Zt)) return false;
    lam.resize(n);
    for (int k = 0; k < n; ++k) lam[k] = M[(size_t)k * n + k];
    const double eps = DBL_EPSILON, small = DBL_MIN * (n / eps);
    std::vector<cd> V((size_t)n * n, cd(0.0)), v(n);
    for (int k = n - 1; k >= 0; --k) {  // T v = lam_k v, v upper part of column k
        v[k] = 1.0;
        const cd lk = lam[k];
        const double smin = std::max(eps * abs1(lk), small);
        for (int i = k - 1; i >= 0; --i) {
            const cd* row = &M[(size_t)i * n];
            cd s = 0.0;
            for (int j = i + 1; j <= k; ++j) s += row[j] * v[j];
            cd d = row[i] - lk;
            if (abs1(d) < smin) d = smin;
            v[i] = -s / d;
            if (abs1(v[i]) > 1e50) {  // rescale the vector built so far
                const double sc = 1.0 / abs1(v[i]);
                for (int q = i; q <= k; ++q) v[q] *= sc;
            }
        }
        for (int i = 0; i <= k; ++i) V[(size_t)i * n + k] = v[i];
    }
    // X = Z V, row by row: X[i][:] = sum_j Z[i][j] V[j][:] (V upper triangular)
    X.assign((size_t)n * n, cd(0.0));
    for (int j = 0; j < n; ++j) {
        const cd* vr = &V[(size_t)j * n];
        const cd* zc = &Zt[(size_t)j * n];  // column j of Z
        for (int i = 0; i < n; ++i) {
            const cd z = zc[i];
            cd* xr = &X[(size_t)i * n];
            for (int k = j; k < n; ++k) xr[k] += z * vr[k];
        }
    }
    return true;
}

// Solve X b = r (LU with partial pivoting); X is overwritten.
bool lu_solve(int n, std::vector<cd> X, std::vector<cd>& r) {
    for (int k = 0; k < n; ++k) {
        int p = k;
        double best = std::abs(X[(size_t)k * n + k]);
        for (int i = k + 1; i < n; ++i)
            if (std::abs(X[(size_t)i * n + k]) > best) { best = std::abs(X[(size_t)i * n + k]); p = i; }
        if (best == 0.0) return false;
        if (p != k) {
            for (int j = 0; j < n; ++j) std::swap(X[(size_t)k * n + j], X[(size_t)p * n + j]);
            std::swap(r[k], r[p]);
        }
        const cd piv = X[(size_t)k * n + k];
        for (int i = k + 1; i < n; ++i) {
            const cd m = X[(size_t)i * n + k] / piv;
            if (m == cd(0.0)) continue;
            for (int j = k + 1; j < n; ++j) X[(size_t)i * n + j] -= m * X[(size_t)k * n + j];
            r[i] -= m * r[k];
        }
    }
    for (int i = n - 1; i >= 0; --i) {
        cd s = r[i];
        for (int j = i + 1; j < n; ++j) s -= X[(size_t)i * n + j] * r[j];
        r[i] = s / X[(size_t)i * n + i];
    }
    return true;
}

// ------------------------------------------------------------ complex symmetric path
// W satisfies detailed balance (W_ij rho_j = W_ji rho_i, build_w), so with D = diag(rho)
// the matrix S = D^-1/2 M D^1/2 = diag(nu) + i p D^-1/2 W D^1/2 is complex symmetric and,
// when diagonalizable, S = Q Lam Q^T with Q^T Q = I.  Then X = D^1/2 Q, and the two
// amplitude vectors of band_modes, a = X^T d and b = X^-1 (rho d), are both
// w = Q^T (sqrt(rho) d): A_k = w_k^2.  Q itself is never formed: every reflection of
// the tridiagonal reduction and every rotation of the QL sweeps is applied to w only,
// so the cost is the reduction's ~n^3 plus O(n^2), against ~15 n^3 for the Schur path.
// Complex orthogonal transformations break down on (near-)isotropic vectors
// (x^T x ~ 0 with x != 0); the functions below then return false and band_modes takes
// the Schur path.

// S (row-major, symmetric, overwritten) -> tridiagonal d (diagonal) and e (e[i] = the
// (i+1, i) element, e[n-1] = 0) by reflections H = I - tau u u^T (H^T H = I), w := H w.
bool csym_tridiag(int n, std::vector<cd>& S, std::vector<cd>& d, std::vector<cd>& e, std::vector<cd>& w) {
    std::vector<cd> u(n), q(n);
    for (int k = 0; k + 2 < n; ++k) {
        const int m = n - k - 1;
        double xn2 = 0.0, tail = 0.0;
        cd sig = 0.0;
        for (int i = 0; i < m; ++i) {
            const cd x = S[(size_t)(k + 1 + i) * n + k];
            xn2 += std::norm(x);
            if (i > 0) tail += std::norm(x);
            sig += x * x;
        }
        if (tail == 0.0) continue;                     // already tridiagonal in this column
        if (std::abs(sig) <= 1e-10 * xn2) return false;  // (near-)isotropic column
        const cd x0 = S[(size_t)(k + 1) * n + k];
        cd alpha = std::sqrt(sig);
        if (std::real(std::conj(x0) * alpha) > 0.0) alpha = -alpha;  // x0 - alpha without cancellation
        const cd utu = 2.0 * alpha * (alpha - x0);   // u^T u for u = x - alpha e1
        if (std::abs(utu) <= 1e-12 * xn2) return false;
        const cd tau = 2.0 / utu;
        for (int i = 0; i < m; ++i) u[i] = S[(size_t)(k + 1 + i) * n + k];
        u[0] -= alpha;
        // trailing block A: H A H = A - u q^T - q u^T, q = p - K u, p = tau A u, K = tau u^T p / 2
        cd K = 0.0;
        for (int i = 0; i < m; ++i) {
            const cd* row = &S[(size_t)(k + 1 + i) * n + k + 1];
            cd t = 0.0;
            for (int j = 0; j < m; ++j) t += row[j] * u[j];
            q[i] = tau * t;
            K += u[i] * q[i];
        }
        K *= 0.5 * tau;
        for (int i = 0; i < m; ++i) q[i] -= K * u[i];
        for (int i = 0; i < m; ++i) {
            cd* row = &S[(size_t)(k + 1 + i) * n + k + 1];
            const cd ui = u[i], qi = q[i];
            for (int j = 0; j < m; ++j) row[j] -= ui * q[j] + qi * u[j];
        }
        S[(size_t)(k + 1) * n + k] = S[(size_t)k * n + k + 1] = alpha;
        for (int i = 1; i < m; ++i) S[(size_t)(k + 1 + i) * n + k] = S[(size_t)k * n + k + 1 + i] = 0.0;
        cd t = 0.0;
        for (int i = 0; i < m; ++i) t += u[i] * w[k + 1 + i];
        t *= tau;
        for (int i = 0; i < m; ++i) w[k + 1 + i] -= t * u[i];
    }
    d.resize(n);
    e.assign(n, cd(0.0));
    for (int i = 0; i < n; ++i) d[i] = S[(size_t)i * n + i];
    for (int i = 0; i + 1 < n; ++i) e[i] = S[(size_t)(i + 1) * n + i];
    return true;
}

// Eigenvalues of the complex symmetric tridiagonal (d, e) by QL sweeps with implicit
// shifts (the order of EISPACK's tql2, in complex arithmetic: r = sqrt(p^2 + 1) and
// sqrt(p^2 + e^2) with complex square roots, rotations c^2 + s^2 = 1), each rotation
// applied to w.  On return d holds the eigenvalues, w[k] pairs with d[k].
bool csym_ql(int n, std::vector<cd>& d, std::vector<cd>& e, std::vector<cd>& w) {
    const double eps = DBL_EPSILON;
    double tst1 = 0.0;
    cd f = 0.0;
    for (int l = 0; l < n; ++l) {
        tst1 = std::max(tst1, std::abs(d[l]) + std::abs(e[l]));
        int m = l;
        while (m < n - 1 && std::abs(e[m]) > eps * tst1) ++m;  // e[n-1] = 0 ends the search
        int iter = 0;
        while (m > l) {
            if (++iter > 60) return false;
            cd g = d[l];
            cd p = (d[l + 1] - g) / (2.0 * e[l]);
            cd r = std::sqrt(p * p + 1.0);
            if (std::real(std::conj(p) * r) < 0.0) r = -r;  // |p + r| >= |p - r|
            if (std::abs(p + r) == 0.0) return false;
            d[l] = e[l] / (p + r);
            d[l + 1] = e[l] * (p + r);
            const cd dl1 = d[l + 1];
            cd h = g - d[l];
            for (int i = l + 2; i < n; ++i) d[i] -= h;
            f += h;
            p = d[m];
            cd c = 1.0, c2 = 1.0, c3 = 1.0, sn = 0.0, s2 = 0.0;
            const cd el1 = e[l + 1];
            for (int i = m - 1; i >= l; --i) {
                c3 = c2;
                c2 = c;
                s2 = sn;
                g = c * e[i];
                h = c * p;
                r = std::sqrt(p * p + e[i] * e[i]);
                if (!(std::abs(r) > 1e-12 * (std::abs(p) + std::abs(e[i])))) return false;  // breakdown
                e[i + 1] = sn * r;
                sn = e[i] / r;
                c = p / r;
                p = c * d[i] - sn * g;
                d[i + 1] = h + sn * (c * g + sn * d[i]);
                const cd w1 = w[i + 1];
                w[i + 1] = sn * w[i] + c * w1;
                w[i] = c * w[i] - sn * w1;
            }
            p = -sn * s2 * c3 * el1 * e[l] / dl1;
            e[l] = sn * p;
            d[l] = c * p;
            if (std::abs(e[l]) <= eps * tst1) break;
        }
        d[l] += f;
        e[l] = 0.0;
    }
    for (int i = 0; i < n; ++i)
        if (!std::isfinite(d[i].real()) || !std::isfinite(d[i].imag()) || !std::isfinite(w[i].real()) ||
            !std::isfinite(w[i].imag()))
            return false;
    return true;
}

// Eigenvalues lam and amplitudes A_k = w_k^2 of M = diag(nu) + i p W through S;
// false (nothing usable) when W is not in detailed balance with rho or the complex
// orthogonal reduction breaks down.
bool csym_modes(int n, const std::vector<double>& nu, const std::vector<double>& W, const std::vector<double>& rho,
                const std::vector<cd>& d0, double p_atm, std::vector<cd>& lam, std::vector<cd>& A) {
    std::vector<double> sr(n);
    for (int i = 0; i < n; ++i) {
        if (!(rho[i] > 0.0) || !std::isfinite(rho[i])) return false;
        sr[i] = std::sqrt(rho[i]);
    }
    std::vector<cd> S((size_t)n * n), w(n);
    for (int i = 0; i < n; ++i) {
        S[(size_t)i * n + i] = cd(nu[i], p_atm * W[(size_t)i * n + i]);
        w[i] = sr[i] * d0[i];
        for (int j = 0; j < i; ++j) {
            const double wij = W[(size_t)i * n + j] * rho[j], wji = W[(size_t)j * n + i] * rho[i];
            if (std::fabs(wij - wji) > 1e-10 * std::max(std::fabs(wij), std::fabs(wji))) return false;
            const cd v(0.0, p_atm * W[(size_t)i * n + j] * (sr[j] / sr[i]));  // i p W_ij sqrt(rho_j / rho_i)
            S[(size_t)i * n + j] = S[(size_t)j * n + i] = v;
        }
    }
    std::vector<cd> d, e;
    if (!csym_tridiag(n, S, d, e, w) || !csym_ql(n, d, e, w)) return false;
    lam = d;
    A.resize(n);
    for (int k = 0; k < n; ++k) A[k] = w[k] * w[k];
    return true;
}

// band_modes (:892-955): kept poles and amplitudes, and the band Doppler factor.
void band_modes(const RelmatBandHost& b, double T, double p_atm, double q_ratio, double keep_threshold,
                std::vector<cd>& poles, std::vector<cd>& amps, double& f) {
    const int n = (int)b.lines.size();
    poles.clear();
    amps.clear();
    f = 0.0;
    if (n == 0) return;
    std::vector<double> W, rho;
    build_w(b, T, q_ratio, W, rho);
    std::vector<cd> d(n), M((size_t)n * n);
    double nu_sum = 0.0;
    for (int i = 0; i < n; ++i) {
        const double nu = b.lines[i].nu;
        nu_sum += nu;
        d[i] = b.lines[i].dipo_t * std::sqrt(nu * (1.0 - std::exp(-kCT * nu / T)));
        for (int j = 0; j < n; ++j) M[(size_t)i * n + j] = cd(i == j ? nu : 0.0, p_atm * W[(size_t)i * n + j]);
    }
    std::vector<cd> lam, A;
    std::vector<double> nus(n);
    for (int i = 0; i < n; ++i) nus[i] = b.lines[i].nu;
    if (!csym_modes(n, nus, W, rho, d, p_atm, lam, A)) {  // the general (Schur) path
        std::vector<cd> X;
        if (!eig(n, M, lam, X)) throw Error{IRS_E_ARG, "band_modes: the QR iteration did not converge"};
        std::vector<cd> bvec(n);
        for (int i = 0; i < n; ++i) bvec[i] = rho[i] * d[i];
        if (!lu_solve(n, X, bvec)) throw Error{IRS_E_ARG, "band_modes: singular eigenvector matrix"};
        A.resize(n);
        for (int k = 0; k < n; ++k) {
            cd a = 0.0;
            for (int i = 0; i < n; ++i) a += X[(size_t)i * n + k] * d[i];
            A[k] = a * bvec[k];
        }
    }
    const int iso = b.isot;
    const double gD = kCtGamD * (nu_sum / n) * std::sqrt(T / mass_amu(b.molecule, iso));
    f = kSqrtLn2 / std::max(gD, 1e-10);
    double max_a = 0.0;
    bool any = false;
    for (int k = 0; k < n; ++k)
        if (lam[k].imag() > 0.0) { any = true; max_a = std::max(max_a, std::abs(A[k])); }
    for (int k = 0; k < n; ++k) {
        if (!(lam[k].imag() > 0.0)) continue;
        if (keep_threshold > 0.0 && any && !(std::abs(A[k]) >= keep_threshold * max_a)) continue;
        poles.push_back(lam[k]);
        amps.push_back(A[k]);
    }
}

double band_eff_strength(const RelmatBandHost& b) {  // :804-811
    double S = 0.0;
    for (auto& l : b.lines) S += l.dipo_t * l.dipo_t * l.popu_t0 * l.nu * (1.0 - std::exp(-kCT * l.nu / kT0));
    return S;
}

}  // namespace

double Tables::q_value(int mol, int iso, double T) const {
    auto it = tips.find({mol, iso});
    if (it == tips.end()) return T / kT0;
    const int tmin = it->second.first;
    const std::vector<double>& q = it->second.second;
    const int n = (int)q.size();
    int lo = (int)std::floor(T) - tmin + 1, hi = lo + 1;
    lo = std::min(std::max(lo, 1), n);
    hi = std::min(std::max(hi, 1), n);
    const double fr = T - std::floor(T);
    return q[lo - 1] * (1.0 - fr) + q[hi - 1] * fr;
}

RelmatBandHost make_band(const irs_relmat_band& b, const irs_wtfit_entry* wt, int64_t n_wt) {
    IRS_REQUIRE(b.n_lines >= 0 && (b.n_lines == 0 || b.lines), "relmat band: lines missing");
    RelmatBandHost h;
    h.lines.assign(b.lines, b.lines + b.n_lines);
    h.li = b.li; h.lf = b.lf; h.isot = b.isot; h.molecule = b.molecule;
    h.whitelisted = b.whitelisted != 0;
    h.nu_min = b.nu_min; h.nu_max = b.nu_max;
    h.eff_strength = band_eff_strength(h);
    // the band's W0B0Table: entries of key (min(li,lf), max(li,lf)); later ones overwrite
    const int lli = std::min(b.li, b.lf), llf = std::max(b.li, b.lf);
    std::map<std::tuple<int, int, int>, std::pair<double, double>> tab;
    for (int64_t e = 0; e < n_wt; ++e) {
        if (wt[e].lli != lli || wt[e].llf != llf) continue;
        IRS_REQUIRE(wt[e].sub >= 0 && wt[e].sub < 9, "W0B0 entry: sub must be in 0..8");
        h.has_wtfit = true;
        tab[{wt[e].sub, wt[e].ji, wt[e].jip}] = {wt[e].w0r, wt[e].b0r};
    }
    // _build_coupling (:530-578)
    const int n = (int)h.lines.size();
    const bool sym = h.isot > 2 && h.isot != 7 && h.isot != 10;
    h.row_ptr.assign(n + 1, 0);
    for (int i = 0; i < n; ++i) {
        h.row_ptr[i] = (int)h.col.size();
        const int jji = h.lines[i].ji, jjf = jji + h.lines[i].branch;
        for (int j = 0; j < n; ++j) {
            if (j == i) continue;
            const int jjip = h.lines[j].ji, jjfp = jjip + h.lines[j].branch;
            if (jjip > jji) continue;
            if (sym && std::abs(jji - jjip) % 2 != 0) continue;
            int ji_e = jji, jf_e = jjf, jip_e = jjip, jfp_e = jjfp;
            if (h.li > h.lf) { ji_e = jjf; jf_e = jji; jip_e = jjfp; jfp_e = jjip; }
            const int sub = 3 * branch_type(ji_e, jf_e) + branch_type(jip_e, jfp_e);
            auto it = tab.find({sub, ji_e, jip_e});
            if (it == tab.end()) continue;
            h.col.push_back(j);
            h.w0r.push_back(it->second.first);
            h.b0r.push_back(it->second.second);
        }
    }
    h.row_ptr[n] = (int)h.col.size();
    return h;
}

void lm_poles(const RelmatHost& R, const Tables& tabs, int mode, uint32_t iso_mask, double T, double p_atm,
              double keep_threshold, std::vector<LmPole>& out) {
    out.clear();
    std::vector<double> Y;
    std::vector<cd> poles, amps;
    for (const RelmatBandHost& b : R.bands) {
        if (b.li > 8) continue;
        if (iso_mask && (b.isot < 0 || b.isot > 31 || !((iso_mask >> b.isot) & 1u))) continue;
        if (R.min_band_strength > 0.0 && b.eff_strength < R.min_band_strength) continue;
        if (!b.has_wtfit) continue;
        const double q_ratio = tabs.q_value(b.molecule, b.isot, 296.0) / tabs.q_value(b.molecule, b.isot, T);
        const int n = (int)b.lines.size();
        if (mode == IRS_LM_RELMAT_VPW && b.whitelisted) {
            double f;
            band_modes(b, T, p_atm, q_ratio, keep_threshold, poles, amps, f);
            if (n == 0) continue;
            const double pre = f * kInvSqrtPi;
            for (size_t k = 0; k < poles.size(); ++k)
                out.push_back({poles[k].real(), f, poles[k].imag() * f, amps[k].real() * pre, amps[k].imag() * pre, 0, 0});
            // minus the no-coupling modes at the same f (_diagonal_band_modes, :1030-1052)
            for (int i = 0; i < n; ++i) {
                const irs_relmat_line& l = b.lines[i];
                const double popu = l.popu_t0 * q_ratio * std::exp(-kCT * l.e_lower * (1.0 / T - 1.0 / kT0));
                const double S = l.dipo_t * l.dipo_t * popu * l.nu * (1.0 - std::exp(-kCT * l.nu / T));
                out.push_back({l.nu, f, gamma_T(l, T) * p_atm * f, -S * pre, 0.0, 0, 0});
            }
        } else {  // first-order dispersive lines (_append_dispersive_lines!, :1193-1220)
            calc_y(b, T, q_ratio, Y);
            const double M = mass_amu(b.molecule, b.isot);
            for (int i = 0; i < n; ++i) {
                if (Y[i] == 0.0) continue;
                const irs_relmat_line& l = b.lines[i];
                const double nu0 = l.nu + (double)l.shift * p_atm;
                const double gD = kCtGamD * l.nu * std::sqrt(T / M);
                const double gL = gamma_T(l, T) * p_atm;
                const double f = kSqrtLn2 / std::max(gD, 1e-10);
                const double st0 = 1.0 - std::exp(-kCT * l.nu / kT0);
                const double stT = 1.0 - std::exp(-kCT * l.nu / T);
                const double S0 = l.dipo_t * l.dipo_t * l.popu_t0 * l.nu * st0;
                const double ST = S0 * q_ratio * std::exp(-kCT * l.e_lower * (1.0 / T - 1.0 / kT0)) * stT / st0;
                if (ST <= 0.0) continue;
                out.push_back({nu0, f, gL * f, 0.0, Y[i] * p_atm * ST * f * kInvSqrtPi, 1, 0});
            }
        }
    }
    std::stable_sort(out.begin(), out.end(), [](const LmPole& a, const LmPole& c) { return a.c < c.c; });
}

}  // namespace irs

// ------------------------------------------------------------------ C ABI (host only)
using irs::Error;

namespace {
template <class F>
int guard(F&& f) {
    try {
        f();
        return IRS_OK;
    } catch (const Error& e) {
        irs::set_error(e.msg);
        return e.code;
    } catch (const std::exception& e) {
        irs::set_error(e.what());
        return IRS_E_ARG;
    }
}
}  // namespace

extern "C" int irs_relmat_w_matrix(const irs_relmat_band* band, const irs_wtfit_entry* wt, int64_t n_wt,
                                   double T, double q_ratio, double* W, double* popu) {
    return guard([&] {
        IRS_REQUIRE(band && W && popu && T > 0.0, "irs_relmat_w_matrix: bad arguments");
        const irs::RelmatBandHost b = irs::make_band(*band, wt, n_wt);
        std::vector<double> w, p;
        irs::build_w(b, T, q_ratio, w, p);
        std::copy(w.begin(), w.end(), W);
        std::copy(p.begin(), p.end(), popu);
    });
}

extern "C" int irs_relmat_y(const irs_relmat_band* band, const irs_wtfit_entry* wt, int64_t n_wt, double T,
                            double q_ratio, double* Y) {
    return guard([&] {
        IRS_REQUIRE(band && Y && T > 0.0, "irs_relmat_y: bad arguments");
        const irs::RelmatBandHost b = irs::make_band(*band, wt, n_wt);
        std::vector<double> y;
        irs::calc_y(b, T, q_ratio, y);
        std::copy(y.begin(), y.end(), Y);
    });
}

extern "C" int irs_band_modes(const irs_relmat_band* band, const irs_wtfit_entry* wt, int64_t n_wt, double T,
                              double p_atm, double q_ratio, double keep_threshold, double* poles, double* amps,
                              double* f, int64_t* n_kept) {
    return guard([&] {
        IRS_REQUIRE(band && poles && amps && f && n_kept && T > 0.0, "irs_band_modes: bad arguments");
        const irs::RelmatBandHost b = irs::make_band(*band, wt, n_wt);
        std::vector<irs::cd> lam, A;
        irs::band_modes(b, T, p_atm, q_ratio, keep_threshold, lam, A, *f);
        for (size_t k = 0; k < lam.size(); ++k) {
            poles[2 * k] = lam[k].real(); poles[2 * k + 1] = lam[k].imag();
            amps[2 * k] = A[k].real(); amps[2 * k + 1] = A[k].imag();
        }
        *n_kept = (int64_t)lam.size();
    });
}
