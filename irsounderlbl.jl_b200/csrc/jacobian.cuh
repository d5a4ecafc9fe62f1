// jacobian.cuh -- the analytic Jacobian of forward_model on the GPU.
//
// Restates vmr_jacobian.jl:152-505 with its atoms:
//   cross-section derivatives (sigma, d/dT, d/dp, d/dvmr_self) in one pass
//                                cross_section_jacobian.jl:68-240 (jg_params_kernel,
//                                jg_linesum_kernel); VP_Y dispersive term with its
//                                analytic derivatives (the reference central-
//                                differences it, :255-322)
//   RTE Jacobian                 schwarzschild_jacobian.jl:66-266 (jg_rte_kernel)
//   channel tail K = dBT/dR . resample . ILS . dI/dx      vmr_jacobian.jl:359-503
//                                (jg_channel_kernel)
// The line sum and the channel contraction are FP32 (Kahan-compensated tile sums);
// the optical-depth sums, transmittances and radiance derivatives are FP64.
#pragma once
#include "faddeeva.cuh"
#include "lineparams.cuh"
#include "linesum.cuh"
#include "rte_ils.cuh"

namespace irs {

constexpr int kJgMaxOut = 11;  // tau, T_lo, T_hi, and (lo, hi) for up to 4 retrieved species

// Per-line primitives (FP64 physics, stored FP32 except the centres), grid units.
struct JgOut {
    double *V, *U;          // sorted key, shifted centre
    float4 *q0;             // An, fx, y, Hc
    float4 *q1;             // An_T, fx_T, y_T, Hc_T
    float4 *q2;             // y_p, u_p, Hc_p, dfar
    float4 *q3;             // y_v, u_v, Hc_v, -
    float4 *q4;             // Yw, Yw_T, Yw_p, -
};

// cross_section_jacobian.jl:43-56 in FP64 (H and its x, y gradient)
__device__ __forceinline__ void h_and_grad64(double x, double y, double x_far, double& H, double& Hx, double& Hy) {
    if (fabs(x) > x_far) {
        const double d = x * x + y * y, d2 = d * d;
        H = y * kInvSqrtPi / d;
        Hx = -2.0 * x * y * kInvSqrtPi / d2;
        Hy = kInvSqrtPi * (x * x - y * y) / d2;
        return;
    }
    const double2 w = faddeeva64(x, y);
    H = w.x;
    Hx = -2.0 * x * w.x + 2.0 * y * w.y;
    Hy = 2.0 * (x * w.y + y * w.x) - 2.0 * kInvSqrtPi;
}

// partition.jl:52-66
__device__ __forceinline__ double tips_slope(const TipsDev& t, int idx, double T) {
    const double* q = t.q + (size_t)idx * t.stride;
    const int lo = (int)floor(T) - t.tmin[idx] + 1, hi = lo + 1;
    if (lo < 1 || hi > t.n[idx]) return 0.0;
    return q[hi - 1] - q[lo - 1];
}

// One thread per (line, segment); no DPTMIN (the Jacobian freezes the line set,
// vmr_jacobian.jl:188-201).  cross_section_jacobian.jl:198-236.
__global__ void __launch_bounds__(256) jg_params_kernel(const SegDev* __restrict__ segs,
                                                        const ListDev* __restrict__ lists, TipsDev tp,
                                                        LpConfig cfg, JgOut o, unsigned* __restrict__ core_reach) {
    const SegDev sg = segs[blockIdx.y];
    const ListDev L = lists[sg.list];
    const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= L.n) return;
    const long long slot = sg.off + j;
    const int mol = L.mol;
    const double T = sg.T, p = sg.p_atm, vs = sg.vs, c = cfg.cutoff, dg = cfg.dnu_g, co = sg.coef;
    const double nu = L.nu[j], n_air = L.nair[j];
    const double n_self = mol == 1 ? 0.95 : (mol == 2 ? 0.75 : n_air);
    const double d_air = L.delta[j], d_self = mol == 1 ? 0.002 : (mol == 2 ? -0.003 : 0.0);
    const double nu0 = nu + (d_air * (1.0 - vs) + d_self * vs) * p;
    const double dn0p = d_air * (1.0 - vs) + d_self * vs, dn0v = (d_self - d_air) * p;
    // temperature_scaled_intensity_deriv, broadening.jl:112-128
    const int ti = L.tips[j];
    const double c2 = 1.4387752;
    double Qr, dlnQ;
    if (ti >= 0) {
        const double QT = tips_lookup(tp, ti, T);
        Qr = tips_lookup(tp, ti, 296.0) / QT;
        dlnQ = tips_slope(tp, ti, T) / QT;
    } else {
        Qr = 296.0 / T;
        dlnQ = (1.0 / 296.0) / (T / 296.0);
    }
    const double stim = (1.0 - exp(-c2 * nu / T)) / (1.0 - exp(-c2 * nu / 296.0));
    const double S = L.S296[j] * Qr * exp(-c2 * L.E[j] * (1.0 / T - 1.0 / 296.0)) * stim;
    const double a = c2 * nu;
    const double dS = S * (-dlnQ + c2 * L.E[j] / (T * T) - (a / (T * T)) / (exp(a / T) - 1.0));
    // pressure_broadened_width_deriv, broadening.jl:62-78
    const double tr = 296.0 / T;
    const double ac = pow(tr, n_air) * L.gair[j], bc = pow(tr, n_self) * L.gself[j];
    const double A = ac * (1.0 - vs) * p, B = bc * vs * p;
    const double gl = A + B, dglT = -(n_air * A + n_self * B) / T;
    const double gd0 = nu * 3.58126e-7 * sqrt(T / mol_mass(mol)), dgd = gd0 / (2.0 * T);
    const double gd = fmax(gd0, 1e-10);
    const double f = kSqrtLn2 / gd, df = -f * (dgd / gd);
    const double dglp = p > 0.0 ? gl / p : ac * (1.0 - vs) + bc * vs, dglv = (bc - ac) * p;
    const double y = gl * f, dyT = dglT * f + gl * df, dyp = dglp * f, dyv = dglv * f;
    const double Sn = S * f * kInvSqrtPi, dSnT = (dS * f + S * df) * kInvSqrtPi;
    double Hc, Hcx, Hcy;
    h_and_grad64(c * f, y, cfg.x_far, Hc, Hcx, Hcy);
    const double dHcT = Hcx * (c * df) + Hcy * dyT, dHcp = Hcy * dyp, dHcv = Hcy * dyv;
    double Yw = 0.0, YwT = 0.0, Ywp = 0.0;
    if ((sg.flags & SEG_LM) && L.has_y0) {  // line_mixing.jl:1193-1220 with Y(T) = y0 (296/T)^0.75
        const double Y = L.y0[j] * pow(296.0 / T, 0.75);
        if (Y != 0.0 && S > 0.0) {
            const double YT = -0.75 * Y / T;
            Yw = Y * p * Sn * co;
            YwT = (YT * Sn + Y * dSnT) * p * co;
            Ywp = Y * Sn * co;
        }
    }
    o.V[slot] = (nu - cfg.grid0) / dg;
    o.U[slot] = (nu0 - cfg.grid0) / dg;
    o.q0[slot] = make_float4((float)(Sn * co), (float)(f * dg), (float)y, (float)Hc);
    o.q1[slot] = make_float4((float)(dSnT * co), (float)(df * dg), (float)dyT, (float)dHcT);
    o.q2[slot] = make_float4((float)dyp, (float)(dn0p / dg), (float)dHcp, (float)fmin(cfg.x_far / (f * dg), 1.0e30));
    o.q3[slot] = make_float4((float)dyv, (float)(dn0v / dg), (float)dHcv, 0.f);
    o.q4[slot] = make_float4((float)Yw, (float)YwT, (float)Ywp, 0.f);
    if (core_reach) {  // the segment's largest core half-width (non-negative floats order as their bits)
        const unsigned mask = __activemask();
        const unsigned r = __reduce_max_sync(mask, __float_as_uint((float)fmin(cfg.x_far / (f * dg), 1.0e30)));
        if ((int)(threadIdx.x & 31) == __ffs(mask) - 1) atomicMax(&core_reach[blockIdx.y], r);
    }
}

// ------------------------------------------------------------------ line sum
constexpr int kJgQ = 4;                        // points per lane
constexpr int kJgWarpPts = 32 * kJgQ;          // 128 points per warp
constexpr int kJgWarps = 8;
constexpr int kJgStrip = kJgWarps * kJgWarpPts;

// Per pair: the value and derivative terms of one line at offset d (grid units).
// H-ped and its derivatives; x = d fx, y; c1 = P/cut^2, c0 = -2P with P = An Hc.
// Far wing: H = y/(sqrt(pi)(x^2+y^2)); core: FP32 Faddeeva with w' = -2 z w + 2i/sqrt(pi).
template <bool LM>
__device__ __forceinline__ void jg_pair(float d, bool core, const float4& q0, const float4& q1, const float4& q2,
                                        const float4& q3, const float4& q4, float icut2, float& s, float& sT,
                                        float& sp, float& sv, float& D, float& DT, float& Dp) {
    const float An = q0.x, fx = q0.y, y = q0.z, Hc = q0.w;
    const float x = d * fx;
    const float xT = d * q1.y;          // u_T = 0
    const float xp = -fx * q2.y, xv = -fx * q3.y;
    float H, Hx, Hy, Lw = 0.f, Lx = 0.f, Ly = 0.f;
    if (core) {
        const float2 w = faddeeva32_fast(x, y);
        H = w.x;
        Hx = -2.f * x * w.x + 2.f * y * w.y;
        Hy = 2.f * (x * w.y + y * w.x) - 2.f * (float)kInvSqrtPi;
        if (LM) {
            Lw = w.y;
            Lx = -2.f * (x * w.y + y * w.x) + 2.f * (float)kInvSqrtPi;
            Ly = Hx;
        }
    } else {
        const float e = fmaf(x, x, y * y);
        const float r = rcp_approx32(e);
        const float r2 = r * r;
        const float k = (float)kInvSqrtPi;
        H = y * k * r;
        Hx = -2.f * x * y * k * r2;
        Hy = k * (x * x - y * y) * r2;
        if (LM) {
            Lw = x * k * r;
            Lx = k * (y * y - x * x) * r2;
            Ly = -2.f * x * y * k * r2;
        }
    }
    // pedestal (2 - (d/cut)^2) Hc and its derivatives; the factor moves with the centre
    const float pf = 2.f - d * d * icut2;
    const float pfp = 2.f * d * q2.y * icut2, pfv = 2.f * d * q3.y * icut2;
    const float Hm = H - pf * Hc;
    s += An * Hm;
    sT += q1.x * Hm + An * (Hx * xT + Hy * q1.z - pf * q1.w);
    sp += An * (Hx * xp + Hy * q2.x - (pfp * Hc + pf * q2.z));
    sv += An * (Hx * xv + Hy * q3.x - (pfv * Hc + pf * q3.z));
    if (LM) {
        D += q4.x * Lw;
        DT += q4.y * Lw + q4.x * (Lx * xT + Ly * q1.z);
        Dp += q4.z * Lw + q4.x * (Lx * xp + Ly * q2.x);
    }
}

// Warp-private staging of one 32-line tile, compacted into the two line classes.
// Fast lines (all 128 points of the warp inside the cutoff and outside the Faddeeva
// core) carry closed-form coefficients of the far-wing terms in rho = 1/(d^2 + b2),
// d the offset in grid units and b2 = (y/fx)^2:
//   s  = a_s rho
//   sT = aT1 rho + aT2 rho^2
//   sp = ap1 rho + ap2 rho^2 + ap3 d rho^2        (sv likewise)
//   D  = cD d rho,  DT = cT1 d rho + cT2 d rho^2,
//   Dp = cp1 d rho + cp2 rho + cp3 rho^2 + cp4 d rho^2          (line mixing)
// which follow from H = y/(sqrt(pi)(x^2+y^2)), its x and y derivatives and
// x = d fx (x_T = d fx_T, x_p = -fx u_p); their pedestals are quadratics in the point
// index summed over the tile.  Slow lines keep the general per-pair form (jg_pair).
struct JgTile {
    float4 fu[32];   // fast: uh, ul, b2, a_s
    float4 fT[32];   // fast: aT1, aT2, ap1, ap2
    float4 fp[32];   // fast: ap3, av1, av2, av3
    float4 fL0[32];  // fast, line mixing: cD, cT1, cT2, cp1
    float4 fL1[32];  // fast, line mixing: cp2, cp3, cp4, -
    float4 su[32];   // slow: uh, ul, -, dfar2
    float4 q0[32], q1[32], q2[32], q3[32], q4[32];  // slow: per-line primitives
};

// The far-wing coefficients of one line (the JgTile fast-line layout; fu = (-, -, b2,
// a_s)) and its pedestal scales P[o] (value, d/dT, d/dp, d/dv) of -P pf,
// pf = 2 - (i - u)^2 / c^2 (pf also moves with the centre for d/dp and d/dv).
template <bool LM>
__device__ __forceinline__ void jg_wing_coeffs(const float4& a0, const float4& a1, const float4& a2,
                                               const float4& a3, const float4& a4, float4& fu, float4& fT,
                                               float4& fp, float4& fL0, float4& fL1, float P[4]) {
    constexpr float k = (float)kInvSqrtPi;
    const float An = a0.x, fx = a0.y, y = a0.z, Hc = a0.w;
    const float AnT = a1.x, fxT = a1.y, yT = a1.z, HcT = a1.w;
    const float yp = a2.x, up = a2.y, Hcp = a2.z, yv = a3.x, uv = a3.y, Hcv = a3.z;
    // 1/fx by the MUFU reciprocal (about 1 ulp) instead of IEEE divisions: these are
    // far-wing coefficients of an FP32 sum
    const float ifx = rcp_fast(fx);
    const float gg = ifx * ifx, b2 = y * y * gg, Aky = An * k * y;
    fu = make_float4(0.f, 0.f, b2, Aky * gg);
    const float r_fx = fxT * ifx;
    fT = make_float4(gg * k * (AnT * y + An * yT) - 2.f * Aky * r_fx * gg,
                     2.f * Aky * b2 * r_fx * gg - 2.f * An * k * yT * b2 * gg, An * k * yp * gg,
                     -2.f * An * k * yp * b2 * gg);
    fp = make_float4(2.f * Aky * up * gg, An * k * yv * gg, -2.f * An * k * yv * b2 * gg, 2.f * Aky * uv * gg);
    if (LM) {
        const float Yw = a4.x, YwT = a4.y, Ywp = a4.z;
        fL0 = make_float4(Yw * k * ifx, YwT * k * ifx - Yw * k * gg * fxT,
                          2.f * Yw * k * gg * fxT * b2 - 2.f * Yw * k * y * fx * yT * gg * gg, Ywp * k * ifx);
        fL1 = make_float4(Yw * k * up * ifx, -2.f * Yw * k * up * b2 * ifx, -2.f * Yw * k * y * fx * yp * gg * gg, 0.f);
    }
    // pedestals: -P0 pf, -PT pf, -An Hc pf_p - An Hc_p pf, ... with pf = 2 - (i - u)^2 / c^2
    P[0] = An * Hc;
    P[1] = AnT * Hc + An * HcT;
    P[2] = An * Hcp;
    P[3] = An * Hcv;
}

// A line's pedestals as quadratics in the point index i (value A + B i + C i^2, the
// centre u in the same coordinates as i)
__device__ __forceinline__ void jg_pedestal_quadratics(const float P[4], const float4& a0, const float4& a2,
                                                       const float4& a3, float u, float icut2, float pA[4],
                                                       float pB[4], float pC[4]) {
    const float e0 = 2.f - u * u * icut2, e1 = 2.f * u * icut2;
#pragma unroll
    for (int o = 0; o < 4; ++o) {
        pA[o] = -P[o] * e0;
        pB[o] = -P[o] * e1;
        pC[o] = P[o] * icut2;
    }
    const float shp = 2.f * a0.x * a0.w * icut2;  // pf_p = 2 (i - u) u_p / c^2
    pA[2] += shp * a2.y * u;
    pB[2] -= shp * a2.y;
    pA[3] += shp * a3.y * u;
    pB[3] -= shp * a3.y;
}

// Far field of the Jacobian sums: as in the forward line sum, the fast lines whose
// centres lie kJgFarDist or more points from the centre of the warp's 128-point block
// are summed at the 8 Chebyshev nodes of the block (all seven sums: s, s_T, s_p, s_v
// and the three dispersive ones) and interpolated; kJgFarDist / 64 = 5 gives the same
// 1.6e-7 bound on one line's interpolation error as the forward kernel's 640 / 128.
constexpr float kJgFarDist = 320.f;
constexpr int kJgFarNodes = 8;
struct JgFarTable {
    float L[kJgFarNodes][kJgWarpPts];
};
__device__ __forceinline__ double jg_far_node(int k) {
    return 63.5 + 63.5 * cos((2 * k + 1) * 3.14159265358979323846 / (2 * kJgFarNodes));
}
__device__ __forceinline__ void jg_far_table_init(JgFarTable& F) {
    for (int idx = threadIdx.x; idx < kJgFarNodes * kJgWarpPts; idx += blockDim.x) {
        const int kk = idx / kJgWarpPts, i = idx % kJgWarpPts;
        double v = 1.0;
        for (int j = 0; j < kJgFarNodes; ++j)
            if (j != kk) v *= ((double)i - jg_far_node(j)) / (jg_far_node(kk) - jg_far_node(j));
        F.L[kk][i] = (float)v;
    }
}

// ---------------------------------------------------------- strip far field
// As for the forward line sum (strip_far_kernel): a line whose shifted centre lies
// kJgStripR or more points from the centre of a 1024-point strip (the 8 warps of a CTA),
// whose cutoff covers the strip and whose Faddeeva core stays off it, is evaluated once
// per strip at 16 Chebyshev nodes, for the four sums (seven with VP_Y on the segment),
// pedestals included (quadratics, reproduced by the interpolation); the degree-15
// interpolants go to each warp's 8 nodes through the fixed matrix M and join the
// warp's own far field.  Worst error of one line's term: 1.6e-8 of its largest value
// on the strip (poles 2 half-widths or more from its centre).  Its lines are two index
// ranges per (segment, strip), taken out of every warp's window.
constexpr float kJgStripR = 1024.f;
constexpr double kJgStripCentre = 0.5 * (kJgStrip - 1);  // 511.5
constexpr int kJgStripNodes = 16;
constexpr int kJgStripOut = 7;                                       // s, s_T, s_p, s_v, D, D_T, D_p
constexpr int kJgStripWords = kJgWarps * kJgStripOut * kJgFarNodes;  // per (segment, strip)
constexpr int kJgStripSegs = 4;                                      // segments per block-wide exchange
// the nodes relative to the strip centre, 511.5 cos((2k+1) pi / 32), rounded to FP32
__device__ __forceinline__ float jg_strip_node_f(int k) {
    const int a = k < 8 ? k : 15 - k;
    const float v = a == 0 ? 5.090369873e+02f : a == 1 ? 4.894749756e+02f : a == 2 ? 4.511027222e+02f
                  : a == 3 ? 3.953948364e+02f : a == 4 ? 3.244921570e+02f : a == 5 ? 2.411194305e+02f
                  : a == 6 ? 1.484806061e+02f : 5.013576889e+01f;
    return k < 8 ? v : -v;
}

// M[w][j][k] = L_k(node j of warp w) for the strip nodes k; one thread per entry
__global__ void jg_strip_table_kernel(float* __restrict__ M) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kJgWarps * kJgFarNodes * kJgStripNodes) return;
    const int w = i / (kJgFarNodes * kJgStripNodes), j = (i / kJgStripNodes) % kJgFarNodes, k = i % kJgStripNodes;
    const double x = (double)kJgWarpPts * w + jg_far_node(j) - kJgStripCentre;
    const double xk = (double)jg_strip_node_f(k);
    double v = 1.0;
    for (int l = 0; l < kJgStripNodes; ++l)
        if (l != k) v *= (x - (double)jg_strip_node_f(l)) / (xk - (double)jg_strip_node_f(l));
    M[i] = (float)v;
}

// One CTA per (strip, profile-layer).  Per batch of segments: the index ranges
// (rin = max(kJgStripR, core reach + 513) + margin, rout = cut - 512 - margin), then
// each warp takes tiles warp, warp + 8, ... of the ranges' lines: the lanes stage their
// lines' far-wing coefficients and sum their pedestal quadratics (the centre as offset
// from the strip centre), and lane l evaluates nodes l % 8 and l % 8 + 8 (packed) over
// every fourth staged line;
// the warps' node and pedestal sums meet in shared memory, and each warp takes them
// (the warps in a fixed order, pedestals evaluated at the nodes) through M to its own
// line-sum warp's 8 nodes: far[(segment, strip)][warp][sum][node], and the ranges.
template <bool ANY_LM>
__global__ void __launch_bounds__(kJgWarps * 32, 2) jg_strip_kernel(
    const SegDev* __restrict__ segs, const int* __restrict__ seg_n, const unsigned* __restrict__ core_reach,
    const int2* __restrict__ pl_segs, JgOut g, float cut_g, int n_strips, const float* __restrict__ M,
    float* __restrict__ far, int4* __restrict__ ranges) {
    constexpr int NC = ANY_LM ? 7 : 4;            // sums
    constexpr int kSlot = kJgStripOut * kJgStripNodes + 12;  // node sums, then A, B, C of the 4 pedestals
    __shared__ float4 sfu[kJgWarps][32], sfT[kJgWarps][32], sfp[kJgWarps][32];
    __shared__ float4 sL0[ANY_LM ? kJgWarps : 1][32], sL1[ANY_LM ? kJgWarps : 1][32];
    __shared__ float slot[kJgStripSegs][kJgWarps][kSlot];
    __shared__ int sj[kJgStripSegs][4];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int strip = blockIdx.x, pl = blockIdx.y;
    const double c = (double)strip * kJgStrip + kJgStripCentre;
    const float icut2 = 1.f / (cut_g * cut_g);
    const float xk = jg_strip_node_f(lane & (kJgStripNodes - 1));  // this lane's node (combining)
    // this lane's node pair (np, np + 8), np = lane % 8, for the line evaluations
    const float2 xp = make_float2(jg_strip_node_f(lane & 7), jg_strip_node_f((lane & 7) + 8));
    const float2 xps = make_float2(xp.y, xp.x);
    const int2 rng = pl_segs[pl];
    for (int s0 = rng.x; s0 < rng.x + rng.y; s0 += kJgStripSegs) {  // block-uniform
        const int ns = min(kJgStripSegs, rng.x + rng.y - s0);
        for (int i = warp; i < 4 * ns; i += kJgWarps) {  // search i: bound i % 4 of segment i / 4
            const SegDev sg = segs[s0 + i / 4];
            const double reach = (double)__uint_as_float(core_reach[s0 + i / 4]);
            const double m = sg.margin_g, rin = fmax((double)kJgStripR, reach + 0.5 * kJgStrip + 1.0) + m;
            const double rout = (double)cut_g - 0.5 * kJgStrip - m;
            int j = 0;
            if (rout > rin) {
                const int b = i % 4;
                const double v = b == 0 ? c - rout : b == 1 ? c - rin : b == 2 ? c + rin : c + rout;
                j = (int)warp_lower_bound(g.V + sg.off, v, seg_n[s0 + i / 4], lane);
            }
            if (lane == 0) sj[i / 4][i % 4] = j;
        }
        __syncthreads();
        for (int si = 0; si < ns; ++si) {
            const SegDev sg = segs[s0 + si];
            const bool lm = ANY_LM && (sg.flags & SEG_LM);
            const int jA = sj[si][0], jB = sj[si][1], jC = sj[si][2], jD = sj[si][3];
            const int nL = jB - jA, n = nL + (jD - jC);
            float2 v[7];  // this lane's node pair (np, np + 8), np = lane % 8, over lines lane / 8 + 4 i
#pragma unroll
            for (int cc = 0; cc < 7; ++cc) v[cc] = make_float2(0.f, 0.f);
            float QA[4] = {0.f, 0.f, 0.f, 0.f}, QB[4] = {0.f, 0.f, 0.f, 0.f}, QC[4] = {0.f, 0.f, 0.f, 0.f};
            float QAc = 0.f, QBc = 0.f, QCc = 0.f;
            for (int t0 = warp * 32; t0 < n; t0 += 32 * kJgWarps) {
                const int t = t0 + lane, nt = min(32, n - t0);
                float pA[4] = {0.f, 0.f, 0.f, 0.f}, pB[4] = {0.f, 0.f, 0.f, 0.f}, pC[4] = {0.f, 0.f, 0.f, 0.f};
                if (t < n) {
                    const long long q = sg.off + (t < nL ? jA + t : jC + (t - nL));
                    const double u = g.U[q] - c;
                    const float uh = (float)u, ul = (float)(u - (double)uh);
                    const float4 a0 = g.q0[q], a1 = g.q1[q], a2 = g.q2[q], a3 = g.q3[q];
                    const float4 a4 = lm ? g.q4[q] : make_float4(0.f, 0.f, 0.f, 0.f);
                    float4 fu, fT, fp, fL0, fL1;
                    float P[4];
                    jg_wing_coeffs<ANY_LM>(a0, a1, a2, a3, a4, fu, fT, fp, fL0, fL1, P);
                    sfu[warp][lane] = make_float4(uh, ul, fu.z, fu.w);
                    sfT[warp][lane] = fT;
                    sfp[warp][lane] = fp;
                    if (ANY_LM) {
                        sL0[warp][lane] = fL0;
                        sL1[warp][lane] = fL1;
                    }
                    jg_pedestal_quadratics(P, a0, a2, a3, uh, icut2, pA, pB, pC);
                }
                kahan_add(QA[0], QAc, pA[0]);
                kahan_add(QB[0], QBc, pB[0]);
                kahan_add(QC[0], QCc, pC[0]);
#pragma unroll
                for (int o = 1; o < 4; ++o) {
                    QA[o] += pA[o];
                    QB[o] += pB[o];
                    QC[o] += pC[o];
                }
                __syncwarp();
                for (int kk = lane >> 3; kk < nt; kk += 4) {  // packed: one reciprocal per node pair
                    const float4 f0 = sfu[warp][kk], f1 = sfT[warp][kk], f2 = sfp[warp][kk];
                    const float2 nu_ = make_float2(-f0.x, -f0.x), nl = make_float2(-f0.y, -f0.y);
                    const float2 dn = __fadd2_rn(__fadd2_rn(xp, nu_), nl);     // (d_a, d_b)
                    const float2 dsw = __fadd2_rn(__fadd2_rn(xps, nu_), nl);   // (d_b, d_a)
                    const float2 es = __ffma2_rn(dsw, dsw, make_float2(f0.z, f0.z));  // (e_b, e_a)
                    const float R = rcp_fast(es.x * es.y);
                    const float2 rho = __fmul2_rn(es, make_float2(R, R));     // (1/e_a, 1/e_b)
                    const float2 rho2 = __fmul2_rn(rho, rho), drho2 = __fmul2_rn(dn, rho2);
                    v[0] = __ffma2_rn(make_float2(f0.w, f0.w), rho, v[0]);
                    v[1] = __ffma2_rn(make_float2(f1.x, f1.x), rho, __ffma2_rn(make_float2(f1.y, f1.y), rho2, v[1]));
                    v[2] = __ffma2_rn(make_float2(f1.z, f1.z), rho,
                                      __ffma2_rn(make_float2(f1.w, f1.w), rho2,
                                                 __ffma2_rn(make_float2(f2.x, f2.x), drho2, v[2])));
                    v[3] = __ffma2_rn(make_float2(f2.y, f2.y), rho,
                                      __ffma2_rn(make_float2(f2.z, f2.z), rho2,
                                                 __ffma2_rn(make_float2(f2.w, f2.w), drho2, v[3])));
                    if (ANY_LM) {
                        const float4 l0 = sL0[warp][kk], l1 = sL1[warp][kk];
                        const float2 drho = __fmul2_rn(dn, rho);
                        v[4] = __ffma2_rn(make_float2(l0.x, l0.x), drho, v[4]);
                        v[5] = __ffma2_rn(make_float2(l0.y, l0.y), drho, __ffma2_rn(make_float2(l0.z, l0.z), drho2, v[5]));
                        v[6] = __ffma2_rn(make_float2(l0.w, l0.w), drho,
                                          __ffma2_rn(make_float2(l1.x, l1.x), rho,
                                                     __ffma2_rn(make_float2(l1.y, l1.y), rho2,
                                                                __ffma2_rn(make_float2(l1.z, l1.z), drho2, v[6]))));
                    }
                }
                __syncwarp();
            }
            float* sl = slot[si][warp];
#pragma unroll
            for (int cc = 0; cc < NC; ++cc) {  // the four line groups, then node np and np + 8
                float2 x = v[cc];
                x.x += __shfl_xor_sync(kFull, x.x, 8);
                x.y += __shfl_xor_sync(kFull, x.y, 8);
                x.x += __shfl_xor_sync(kFull, x.x, 16);
                x.y += __shfl_xor_sync(kFull, x.y, 16);
                if (lane < 8) {
                    sl[cc * kJgStripNodes + lane] = x.x;
                    sl[cc * kJgStripNodes + lane + 8] = x.y;
                }
            }
            float wA[4], wB[4], wC[4];
            wA[0] = warp_sum(QA[0] - QAc);
            wB[0] = warp_sum(QB[0] - QBc);
            wC[0] = warp_sum(QC[0] - QCc);
#pragma unroll
            for (int o = 1; o < 4; ++o) {
                wA[o] = warp_sum(QA[o]);
                wB[o] = warp_sum(QB[o]);
                wC[o] = warp_sum(QC[o]);
            }
            if (lane == 0) {
#pragma unroll
                for (int o = 0; o < 4; ++o) {
                    sl[kJgStripOut * kJgStripNodes + 3 * o] = wA[o];
                    sl[kJgStripOut * kJgStripNodes + 3 * o + 1] = wB[o];
                    sl[kJgStripOut * kJgStripNodes + 3 * o + 2] = wC[o];
                }
            }
        }
        __syncthreads();
        const float* Mw = M + ((size_t)warp * kJgFarNodes + (lane & (kJgFarNodes - 1))) * kJgStripNodes;
        for (int si = 0; si < ns; ++si) {
            const size_t cell = (size_t)(s0 + si) * n_strips + strip;
            const bool lm = ANY_LM && (segs[s0 + si].flags & SEG_LM);
#pragma unroll
            for (int cc = 0; cc < NC; ++cc) {
                if (cc >= 4 && !lm) break;
                float fc = 0.f;  // lane k < 16: node k of sum cc, the warps in a fixed order
                float A = 0.f, B = 0.f, C = 0.f;
#pragma unroll
                for (int w = 0; w < kJgWarps; ++w) {
                    fc += slot[si][w][cc * kJgStripNodes + (lane & (kJgStripNodes - 1))];
                    if (cc < 4) {
                        A += slot[si][w][kJgStripOut * kJgStripNodes + 3 * cc];
                        B += slot[si][w][kJgStripOut * kJgStripNodes + 3 * cc + 1];
                        C += slot[si][w][kJgStripOut * kJgStripNodes + 3 * cc + 2];
                    }
                }
                if (cc < 4) fc += fmaf(xk, fmaf(xk, C, B), A);
                float gv = 0.f;
#pragma unroll
                for (int k = 0; k < kJgStripNodes; ++k) gv = fmaf(__ldg(Mw + k), __shfl_sync(kFull, fc, k), gv);
                if (lane < kJgFarNodes) far[cell * kJgStripWords + (warp * kJgStripOut + cc) * kJgFarNodes + lane] = gv;
            }
            if (threadIdx.x == 0) ranges[cell] = make_int4(sj[si][0], sj[si][1], sj[si][2], sj[si][3]);
        }
        if (s0 + kJgStripSegs < rng.x + rng.y) __syncthreads();  // slots and ranges reused by the next batch
    }
}

template <bool LM>
__device__ void jg_segment(const SegDev& sg, long long cnt, const JgOut& g, long long wb, float cut, int lane,
                           JgTile& T, const JgFarTable& FT, float xn, float sum[4][kJgQ], float dsum[3][kJgQ],
                           int4 sx, const float* __restrict__ gfar) {
    constexpr float kCentre = 0.5f * (kJgWarpPts - 1);
    constexpr float kHalf = 0.5f * kJgWarpPts + 0.5f;
    const float cut2 = cut * cut, icut2 = 1.f / cut2;
    const long long jlo = warp_lower_bound(g.V + sg.off, (double)wb - cut - sg.margin_g, cnt, lane);
    const long long jhi =
        warp_lower_bound(g.V + sg.off, (double)(wb + kJgWarpPts - 1) + cut + sg.margin_g + 1e-9, cnt, lane);
    const float pl0 = (float)lane;
    const unsigned lt = (1u << lane) - 1u;
    // packed accumulators over point pairs (q = 2h, 2h + 1)
    float2 S[kJgQ / 2], C[kJgQ / 2], ST[kJgQ / 2], SP[kJgQ / 2], SV[kJgQ / 2];
    float2 SD[kJgQ / 2], CD[kJgQ / 2], SDT[kJgQ / 2], SDP[kJgQ / 2];
#pragma unroll
    for (int h = 0; h < kJgQ / 2; ++h) {
        S[h] = C[h] = ST[h] = SP[h] = SV[h] = make_float2(0.f, 0.f);
        SD[h] = CD[h] = SDT[h] = SDP[h] = make_float2(0.f, 0.f);
    }
    float2 offn[kJgQ / 2], offs[kJgQ / 2];  // natural (32q, 32(q+1)) and swapped offsets
#pragma unroll
    for (int h = 0; h < kJgQ / 2; ++h) {
        offn[h] = make_float2(64.f * h, 64.f * h + 32.f);
        offs[h] = make_float2(64.f * h + 32.f, 64.f * h);
    }
    // far-field node sums: lane l accumulates node l % 8 over every fourth far line
    float fS = 0.f, fC = 0.f, fT_ = 0.f, fP = 0.f, fV = 0.f, fD = 0.f, fDC = 0.f, fDT = 0.f, fDP = 0.f;
    // pedestal quadratics of this lane's fast and far lines (the value sum compensated),
    // reduced over the warp once per segment
    float QA[4] = {0.f, 0.f, 0.f, 0.f}, QB[4] = {0.f, 0.f, 0.f, 0.f}, QC[4] = {0.f, 0.f, 0.f, 0.f};
    float QAc = 0.f, QBc = 0.f, QCc = 0.f;
    // the window without the strip far field's ranges [sx.x, sx.y) and [sx.z, sx.w):
    // [ilo, ra), [rb, rc) and [rd, ihi), walked in turn (indices within a segment fit in int)
    const int ilo = (int)jlo, ihi = (int)jhi;
    const int ra = min(max(sx.x, ilo), ihi), rb = min(max(sx.y, ilo), ihi);
    const int rc = min(max(sx.z, ilo), ihi), rd = min(max(sx.w, ilo), ihi);
    int nt = 0;
    for (int t0 = skip_ranges(ilo, ra, rb, rc, rd); t0 < ihi; t0 = skip_ranges(t0 + nt, ra, rb, rc, rd)) {
        nt = min(32, (t0 < ra ? ra : t0 < rc ? rc : ihi) - t0);
        int cls = 0;
        float uh = 0.f, ul = 0.f;
        float4 a0, a1, a2, a3, a4;
        // pedestal quadratic of a fast line: value at point i is A + B i + Cq i^2
        float pA[4] = {0.f, 0.f, 0.f, 0.f}, pB[4] = {0.f, 0.f, 0.f, 0.f}, pC[4] = {0.f, 0.f, 0.f, 0.f};
        if (lane < nt) {
            const long long q = sg.off + t0 + lane;
            const double u = g.U[q] - (double)wb;
            uh = (float)u;
            ul = (float)(u - (double)uh);
            a0 = g.q0[q];
            a1 = g.q1[q];
            a2 = g.q2[q];
            a3 = g.q3[q];
            if (LM) a4 = g.q4[q];
            const float dist = fabsf(uh - kCentre);
            if (dist > cut + kHalf) cls = 0;
            else if (dist + kHalf <= cut && dist > a2.w + kHalf) cls = dist >= kJgFarDist ? 3 : 1;
            else if (dist > a2.w + kHalf) cls = 4;  // far wing everywhere, the cutoff falls among the points
            else cls = 2;
        }
        const unsigned fm = __ballot_sync(kFull, cls == 1), sm = __ballot_sync(kFull, cls == 2);
        const unsigned xm = __ballot_sync(kFull, cls == 3), em = __ballot_sync(kFull, cls == 4);
        __syncwarp();
        if (cls == 1 || cls == 3 || cls == 4) {  // fast lines first, far lines after them, edge lines from the top
            const int pos = cls == 1 ? __popc(fm & lt) : (cls == 3 ? __popc(fm) + __popc(xm & lt) : 31 - __popc(em & lt));
            float4 fu, fT, fp, fL0, fL1;
            float P[4];
            jg_wing_coeffs<LM>(a0, a1, a2, a3, a4, fu, fT, fp, fL0, fL1, P);
            T.fu[pos] = make_float4(uh, ul, fu.z, fu.w);
            T.fT[pos] = fT;
            T.fp[pos] = fp;
            if (LM) {
                T.fL0[pos] = fL0;
                T.fL1[pos] = fL1;
            }
            if (cls == 4) {  // edge lines: pedestals per point (masked by the cutoff), in the slow arrays' top
                T.q0[pos] = make_float4(P[0], P[1], P[2], P[3]);
                T.q1[pos] = make_float4(2.f * a2.y * icut2 * P[0], 2.f * a3.y * icut2 * P[0], 0.f, 0.f);
            } else {
                jg_pedestal_quadratics(P, a0, a2, a3, uh, icut2, pA, pB, pC);
            }
        } else if (cls == 2) {
            const int pos = __popc(sm & lt);
            T.su[pos] = make_float4(uh, ul, 0.f, a2.w * a2.w);
            T.q0[pos] = a0;
            T.q1[pos] = a1;
            T.q2[pos] = a2;
            T.q3[pos] = a3;
            if (LM) T.q4[pos] = a4;
        }
        kahan_add(QA[0], QAc, pA[0]);
        kahan_add(QB[0], QBc, pB[0]);
        kahan_add(QC[0], QCc, pC[0]);
#pragma unroll
        for (int o = 1; o < 4; ++o) {
            QA[o] += pA[o];
            QB[o] += pB[o];
            QC[o] += pC[o];
        }
        __syncwarp();
        const int nf = __popc(fm), ns = __popc(sm), nx = __popc(xm), ne = __popc(em);
        {
            float ts = 0.f, td = 0.f;
            for (int kk = nf + (lane >> 3); kk < nf + nx; kk += 4) {
                const float4 f0 = T.fu[kk], f1 = T.fT[kk], f2 = T.fp[kk];
                const float d = (xn - f0.x) - f0.y;
                const float rho = rcp_fast(fmaf(d, d, f0.z));
                const float rho2 = rho * rho, drho2 = d * rho2;
                ts = fmaf(f0.w, rho, ts);
                fT_ = fmaf(f1.x, rho, fmaf(f1.y, rho2, fT_));
                fP = fmaf(f1.z, rho, fmaf(f1.w, rho2, fmaf(f2.x, drho2, fP)));
                fV = fmaf(f2.y, rho, fmaf(f2.z, rho2, fmaf(f2.w, drho2, fV)));
                if (LM) {
                    const float4 l0 = T.fL0[kk], l1 = T.fL1[kk];
                    const float drho = d * rho;
                    td = fmaf(l0.x, drho, td);
                    fDT = fmaf(l0.y, drho, fmaf(l0.z, drho2, fDT));
                    fDP = fmaf(l0.w, drho, fmaf(l1.x, rho, fmaf(l1.y, rho2, fmaf(l1.z, drho2, fDP))));
                }
            }
            kahan_add(fS, fC, ts);
            if (LM) kahan_add(fD, fDC, td);
        }
        if (nf + ns + ne == 0) continue;  // warp-uniform: nothing per point in this tile
        float2 TS[kJgQ / 2], TD[kJgQ / 2];  // tile partials of the value sums (Kahan-added below)
#pragma unroll
        for (int h = 0; h < kJgQ / 2; ++h) TS[h] = TD[h] = make_float2(0.f, 0.f);
        for (int kk = 0; kk < nf; ++kk) {
            const float4 f0 = T.fu[kk], f1 = T.fT[kk], f2 = T.fp[kk];
            const float d0 = (pl0 - f0.x) - f0.y;
            const float2 d0s = make_float2(d0, d0), b2 = make_float2(f0.z, f0.z);
            float4 l0, l1;
            if (LM) {
                l0 = T.fL0[kk];
                l1 = T.fL1[kk];
            }
#pragma unroll
            for (int h = 0; h < kJgQ / 2; ++h) {
                const float2 dsw = __fadd2_rn(d0s, offs[h]);      // (d[q+1], d[q])
                const float2 dn = __fadd2_rn(d0s, offn[h]);       // (d[q], d[q+1])
                const float2 es = __ffma2_rn(dsw, dsw, b2);       // (e[q+1], e[q])
                const float R = rcp_fast(es.x * es.y);
                const float2 rho = __fmul2_rn(es, make_float2(R, R));  // (1/e[q], 1/e[q+1])
                const float2 rho2 = __fmul2_rn(rho, rho);
                const float2 drho2 = __fmul2_rn(dn, rho2);
                TS[h] = __ffma2_rn(make_float2(f0.w, f0.w), rho, TS[h]);
                ST[h] = __ffma2_rn(make_float2(f1.x, f1.x), rho, ST[h]);
                ST[h] = __ffma2_rn(make_float2(f1.y, f1.y), rho2, ST[h]);
                SP[h] = __ffma2_rn(make_float2(f1.z, f1.z), rho, SP[h]);
                SP[h] = __ffma2_rn(make_float2(f1.w, f1.w), rho2, SP[h]);
                SP[h] = __ffma2_rn(make_float2(f2.x, f2.x), drho2, SP[h]);
                SV[h] = __ffma2_rn(make_float2(f2.y, f2.y), rho, SV[h]);
                SV[h] = __ffma2_rn(make_float2(f2.z, f2.z), rho2, SV[h]);
                SV[h] = __ffma2_rn(make_float2(f2.w, f2.w), drho2, SV[h]);
                if (LM) {
                    const float2 drho = __fmul2_rn(dn, rho);
                    TD[h] = __ffma2_rn(make_float2(l0.x, l0.x), drho, TD[h]);
                    SDT[h] = __ffma2_rn(make_float2(l0.y, l0.y), drho, SDT[h]);
                    SDT[h] = __ffma2_rn(make_float2(l0.z, l0.z), drho2, SDT[h]);
                    SDP[h] = __ffma2_rn(make_float2(l0.w, l0.w), drho, SDP[h]);
                    SDP[h] = __ffma2_rn(make_float2(l1.x, l1.x), rho, SDP[h]);
                    SDP[h] = __ffma2_rn(make_float2(l1.y, l1.y), rho2, SDP[h]);
                    SDP[h] = __ffma2_rn(make_float2(l1.z, l1.z), drho2, SDP[h]);
                }
            }
        }
        // cutoff-edge lines: the far-wing coefficients and the per-point pedestals,
        // masked to the points inside the cutoff
        for (int e = 0; e < ne; ++e) {
            const int kk = 31 - e;
            const float4 f0 = T.fu[kk], f1 = T.fT[kk], f2 = T.fp[kk], P = T.q0[kk], c = T.q1[kk];
            float4 l0, l1;
            if (LM) {
                l0 = T.fL0[kk];
                l1 = T.fL1[kk];
            }
            const float d0 = (pl0 - f0.x) - f0.y;
#pragma unroll
            for (int q = 0; q < kJgQ; ++q) {
                const float d = d0 + 32.f * q, d2 = d * d;
                if (d2 > cut2) continue;
                const float rho = rcp_fast(d2 + f0.z), rho2 = rho * rho, drho2 = d * rho2;
                const float pf = fmaf(-d2, icut2, 2.f);
                const float vs = fmaf(f0.w, rho, -P.x * pf);
                const float vT = fmaf(f1.x, rho, fmaf(f1.y, rho2, -P.y * pf));
                const float vp = fmaf(f1.z, rho, fmaf(f1.w, rho2, fmaf(f2.x, drho2, -fmaf(c.x, d, P.z * pf))));
                const float vv = fmaf(f2.y, rho, fmaf(f2.z, rho2, fmaf(f2.w, drho2, -fmaf(c.y, d, P.w * pf))));
                const int h = q >> 1;
                float vD = 0.f, vDT = 0.f, vDP = 0.f;
                if (LM) {
                    const float drho = d * rho;
                    vD = l0.x * drho;
                    vDT = fmaf(l0.y, drho, l0.z * drho2);
                    vDP = fmaf(l0.w, drho, fmaf(l1.x, rho, fmaf(l1.y, rho2, l1.z * drho2)));
                }
                if (q & 1) {
                    TS[h].y += vs; ST[h].y += vT; SP[h].y += vp; SV[h].y += vv;
                    if (LM) { TD[h].y += vD; SDT[h].y += vDT; SDP[h].y += vDP; }
                } else {
                    TS[h].x += vs; ST[h].x += vT; SP[h].x += vp; SV[h].x += vv;
                    if (LM) { TD[h].x += vD; SDT[h].x += vDT; SDP[h].x += vDP; }
                }
            }
        }
        for (int kk = 0; kk < ns; ++kk) {
            const float4 u = T.su[kk];
            const float4 q0 = T.q0[kk], q1 = T.q1[kk], q2 = T.q2[kk], q3 = T.q3[kk];
            const float4 q4 = LM ? T.q4[kk] : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
            for (int q = 0; q < kJgQ; ++q) {
                const float d = ((pl0 + 32.f * q) - u.x) - u.y;
                const float d2 = d * d;
                if (d2 > cut2) continue;
                float s = 0.f, sT = 0.f, sp = 0.f, sv = 0.f, D = 0.f, DT = 0.f, Dp = 0.f;
                jg_pair<LM>(d, d2 <= u.w, q0, q1, q2, q3, q4, icut2, s, sT, sp, sv, D, DT, Dp);
                const int h = q >> 1;
                if (q & 1) {
                    TS[h].y += s; ST[h].y += sT; SP[h].y += sp; SV[h].y += sv;
                    if (LM) { TD[h].y += D; SDT[h].y += DT; SDP[h].y += Dp; }
                } else {
                    TS[h].x += s; ST[h].x += sT; SP[h].x += sp; SV[h].x += sv;
                    if (LM) { TD[h].x += D; SDT[h].x += DT; SDP[h].x += Dp; }
                }
            }
        }
        // the compensated tile sums
#pragma unroll
        for (int h = 0; h < kJgQ / 2; ++h) {
            kahan_add(S[h].x, C[h].x, TS[h].x);
            kahan_add(S[h].y, C[h].y, TS[h].y);
            if (LM) {
                kahan_add(SD[h].x, CD[h].x, TD[h].x);
                kahan_add(SD[h].y, CD[h].y, TD[h].y);
            }
        }
    }
    {  // pedestals of the fast and far lines
        float wA[4], wB[4], wC[4];
        wA[0] = warp_sum(QA[0] - QAc);
        wB[0] = warp_sum(QB[0] - QBc);
        wC[0] = warp_sum(QC[0] - QCc);
#pragma unroll
        for (int o = 1; o < 4; ++o) {
            wA[o] = warp_sum(QA[o]);
            wB[o] = warp_sum(QB[o]);
            wC[o] = warp_sum(QC[o]);
        }
#pragma unroll
        for (int h = 0; h < kJgQ / 2; ++h) {
            const float i0 = pl0 + 64.f * h, i1 = i0 + 32.f;
            kahan_add(S[h].x, C[h].x, fmaf(i0, fmaf(i0, wC[0], wB[0]), wA[0]));
            kahan_add(S[h].y, C[h].y, fmaf(i1, fmaf(i1, wC[0], wB[0]), wA[0]));
            ST[h].x += fmaf(i0, fmaf(i0, wC[1], wB[1]), wA[1]);
            ST[h].y += fmaf(i1, fmaf(i1, wC[1], wB[1]), wA[1]);
            SP[h].x += fmaf(i0, fmaf(i0, wC[2], wB[2]), wA[2]);
            SP[h].y += fmaf(i1, fmaf(i1, wC[2], wB[2]), wA[2]);
            SV[h].x += fmaf(i0, fmaf(i0, wC[3], wB[3]), wA[3]);
            SV[h].y += fmaf(i1, fmaf(i1, wC[3], wB[3]), wA[3]);
        }
    }
    {  // node totals (4 lanes per node), then the interpolants at this lane's points
        float v[7] = {fS, fT_, fP, fV, fD, fDT, fDP};
#pragma unroll
        for (int c = 0; c < 7; ++c) {
            if (!LM && c >= 4) continue;
            v[c] += __shfl_xor_sync(kFull, v[c], 8);
            v[c] += __shfl_xor_sync(kFull, v[c], 16);
            if (gfar) v[c] += gfar[c * kJgFarNodes + (lane & (kJgFarNodes - 1))];  // the strip far field
        }
        float it[7][kJgQ];
#pragma unroll
        for (int c = 0; c < 7; ++c)
#pragma unroll
            for (int q = 0; q < kJgQ; ++q) it[c][q] = 0.f;
#pragma unroll
        for (int kk = 0; kk < kJgFarNodes; ++kk) {
            float w[kJgQ];
#pragma unroll
            for (int q = 0; q < kJgQ; ++q) w[q] = FT.L[kk][32 * q + lane];
#pragma unroll
            for (int c = 0; c < 7; ++c) {
                if (!LM && c >= 4) continue;
                const float n = __shfl_sync(kFull, v[c], kk);
#pragma unroll
                for (int q = 0; q < kJgQ; ++q) it[c][q] = fmaf(n, w[q], it[c][q]);
            }
        }
#pragma unroll
        for (int h = 0; h < kJgQ / 2; ++h) {
            kahan_add(S[h].x, C[h].x, it[0][2 * h]);
            kahan_add(S[h].y, C[h].y, it[0][2 * h + 1]);
            ST[h].x += it[1][2 * h]; ST[h].y += it[1][2 * h + 1];
            SP[h].x += it[2][2 * h]; SP[h].y += it[2][2 * h + 1];
            SV[h].x += it[3][2 * h]; SV[h].y += it[3][2 * h + 1];
            if (LM) {
                kahan_add(SD[h].x, CD[h].x, it[4][2 * h]);
                kahan_add(SD[h].y, CD[h].y, it[4][2 * h + 1]);
                SDT[h].x += it[5][2 * h]; SDT[h].y += it[5][2 * h + 1];
                SDP[h].x += it[6][2 * h]; SDP[h].y += it[6][2 * h + 1];
            }
        }
    }
#pragma unroll
    for (int h = 0; h < kJgQ / 2; ++h) {
        sum[0][2 * h] = S[h].x; sum[0][2 * h + 1] = S[h].y;
        sum[1][2 * h] = ST[h].x; sum[1][2 * h + 1] = ST[h].y;
        sum[2][2 * h] = SP[h].x; sum[2][2 * h + 1] = SP[h].y;
        sum[3][2 * h] = SV[h].x; sum[3][2 * h + 1] = SV[h].y;
        dsum[0][2 * h] = SD[h].x; dsum[0][2 * h + 1] = SD[h].y;
        dsum[1][2 * h] = SDT[h].x; dsum[1][2 * h + 1] = SDT[h].y;
        dsum[2][2 * h] = SDP[h].x; dsum[2][2 * h + 1] = SDP[h].y;
    }
}

// Segment weights: out[o] += W[o][0] s + W[o][1] s_T + W[o][2] s_p + W[o][3] s_v
struct SegW {
    float w[kJgMaxOut][4];
};

// dynamic shared memory of jg_linesum_kernel<*, NOUT>: the warps' tiles and their
// per-point output accumulators
constexpr size_t jg_smem_bytes(int nout) {
    return sizeof(JgTile) * kJgWarps + sizeof(float) * kJgWarps * nout * kJgWarpPts + sizeof(JgFarTable);
}

template <bool ANY_LM, int NOUT>
__global__ void __launch_bounds__(kJgWarps * 32, 2) jg_linesum_kernel(
    const SegDev* __restrict__ segs, const int* __restrict__ seg_n, const SegW* __restrict__ wts,
    const int2* __restrict__ pl_segs, JgOut g, long long n_nu, float cut_g, float* __restrict__ out,
    const double* __restrict__ pert, long long pstride, const float* __restrict__ sfar,
    const int4* __restrict__ sranges, int n_strips) {
    extern __shared__ float4 jg_sh[];
    JgTile* tiles = (JgTile*)jg_sh;
    JgFarTable& ftab = *(JgFarTable*)((float*)(tiles + kJgWarps) + (size_t)kJgWarps * NOUT * kJgWarpPts);
    jg_far_table_init(ftab);
    __syncthreads();  // the only block-wide barrier: before any warp leaves
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float* acc = (float*)(tiles + kJgWarps) + (size_t)warp * NOUT * kJgWarpPts;  // [NOUT][128], warp-private
    const int pl = blockIdx.y;
    const long long wb = (long long)blockIdx.x * kJgStrip + (long long)warp * kJgWarpPts;
    if (wb >= n_nu) return;
    const float xn = (float)jg_far_node(lane & (kJgFarNodes - 1));
    for (int o = 0; o < NOUT; ++o)
#pragma unroll
        for (int q = 0; q < kJgQ; ++q) acc[o * kJgWarpPts + 32 * q + lane] = 0.f;
    const int2 rng = pl_segs[pl];
    for (int si = rng.x; si < rng.x + rng.y; ++si) {
        const SegDev sg = segs[si];
        float s[4][kJgQ], ds[3][kJgQ];
        const long long nl = seg_n[si];
        const bool lm = ANY_LM && (sg.flags & SEG_LM);
        int4 sx = make_int4(0, 0, 0, 0);  // no strip far field: the whole window
        const float* gf = nullptr;
        if (sfar) {
            const size_t cell = (size_t)si * n_strips + blockIdx.x;
            sx = sranges[cell];
            gf = sfar + cell * kJgStripWords + (size_t)warp * kJgStripOut * kJgFarNodes;
        }
        if (lm)
            jg_segment<true>(sg, nl, g, wb, cut_g, lane, tiles[warp], ftab, xn, s, ds, sx, gf);
        else
            jg_segment<false>(sg, nl, g, wb, cut_g, lane, tiles[warp], ftab, xn, s, ds, sx, gf);
        // clamps (voigt.jl:276, line_mixing.jl:1368, cross_section_jacobian.jl:107-113, :312-319)
        const SegW& W = wts[si];
        // relaxation-matrix line mixing: rows (perturbation, d/dT, d/dp) x column amount
        const double* prow = pert && (sg.flags & SEG_RELMAT) ? pert + (size_t)pl * 3 * pstride + wb + lane : nullptr;
#pragma unroll
        for (int q = 0; q < kJgQ; ++q) {
            float v = s[0][q], vT = s[1][q], vp = s[2][q], vv = s[3][q];
            if (!(v > 0.f)) v = vT = vp = vv = 0.f;
            if (lm) {
                v += ds[0][q];
                vT += ds[1][q];
                vp += ds[2][q];
                if (!(v > 0.f)) v = vT = vp = 0.f;
            }
            if (prow) {
                v += (float)prow[32 * q];
                vT += (float)prow[pstride + 32 * q];
                vp += (float)prow[2 * pstride + 32 * q];
                if (!(v > 0.f)) v = vT = vp = 0.f;
            }
            for (int o = 0; o < NOUT; ++o)
                acc[o * kJgWarpPts + 32 * q + lane] += W.w[o][0] * v + W.w[o][1] * vT + W.w[o][2] * vp + W.w[o][3] * vv;
        }
    }
    float* base = out + (size_t)pl * NOUT * n_nu;
    for (int o = 0; o < NOUT; ++o)
#pragma unroll
        for (int q = 0; q < kJgQ; ++q) {
            const long long i = wb + 32 * q + lane;
            if (i < n_nu) base[(size_t)o * n_nu + i] = acc[o * kJgWarpPts + 32 * q + lane];
        }
}

// ------------------------------------------------------------------ RTE Jacobian
struct JgLayer {       // per (profile, layer), beyond LayerRT
    double frac;       // _cg_mass_frac (T_ave weight on the upper level)
    double wM;         // log-p weight of p_mid on the upper level
    double dp;         // layer thickness, hPa
};
struct JgProfile {     // per profile
    int n_retr;
    int retr_h2o, retr_co2;  // retrieved index of H2O / CO2 whose continuum VMR derivative is used, or -1
    int include_T, include_tsfc, include_eps, log_vmr;
    int n_state;
};

__device__ __forceinline__ double dB_dT64(double nu, double T) {  // planck.jl:67-71
    const double x = 1.4387769 * nu / T, ex = exp(x);
    return 1.191042953e-5 * 1.4387769 * (nu * nu * nu * nu) * ex / ((T * T) * (ex - 1.0) * (ex - 1.0));
}
__device__ __forceinline__ double cim_corr_d(double s) {
    if (s < 0.06) return 1.0 / 6.0;
    const double w = exp(-s);
    return 2.0 / (s * s) - 2.0 * w / ((w - 1.0) * (w - 1.0));
}
__device__ __forceinline__ double lit_corr_d(double s) {
    if (s < 1e-4) return 0.5 - s * (2.0 / 3.0 - s * 0.375);
    const double e = exp(-s);
    return (e * (s + 1.0) - 1.0) / (s * s) + e;
}

// continuum optical depth of one layer at (vh, vc, Tm), continuum.jl:183-250 and
// the dz(Tm) of optical_depth.jl:123-130 (vmr_jacobian.jl:300-311)
template <bool CIA>
__device__ __forceinline__ double cont_tau(double nu, const LayerRT& r, double dp, const ContDev& c, double Cs,
                                          double Cf, double te, double Se, double td, double vh, double vc,
                                          double Tm, const CiaPoint& cp) {
    const double p = r.p_mid;
    const double dz = 8.314462 * Tm / (0.028964 * 9.80665) * dp / p * 100.0;
    const double rho = (p / 1013.0) * (296.0 / Tm);
    const double rad = radfn(nu, Tm);
    double t = 0.0;
    if (c.mask & 1) {
        const double n = vh * p * 100.0 / (1.380649e-23 * Tm) * 1e-6;
        const double ks = Cs * pow(296.0 / Tm, te) * vh * rho * rad * n;
        const double kf = Cf * (1.0 - vh) * rho * rad * n;
        t += (ks + kf) * dz;
    }
    if (c.mask & 2) {
        const double n = vc * p * 100.0 / (1.380649e-23 * Tm) * 1e-6;
        const double tc = td == 0.0 ? 1.0 : pow(Tm / 246.0, td);
        t += Se * tc * (1e-20 * n * rho) * rad * dz;
    }
    if (CIA) t += cia_tau(c, cp, nu, vh, vc, p, Tm, dz);
    return t;
}

// One thread per (profile, grid point): the monochromatic Jacobian columns
// D[x][nu] = dI/dx (FP32) for every state element, and I (FP64).
// schwarzschild_jacobian.jl:66-266 with the state chains of vmr_jacobian.jl:383-503.
// Transmittances come from the FP64 cumulative optical depth: the top-of-layer
// transmittance of layer m is exp(-(OD_total - OD_below_and_m)).
//
// MODE selects what the sweep leaves behind:
//   0  D (forward mode, the columns of the monochromatic Jacobian) and I;
//   1  I only (the derivative terms are not formed);
//   2  the adjoint: with Ibar[profile][nu] = the radiance cotangent on the grid (the ILS
//      and channel resampling transposed, applied to dy dBT/dR), each term D[x][nu] is
//      multiplied by Ibar[nu] as it is formed and summed over the grid on the device
//      (warp shuffles, then FP64 shared-memory and global atomics) into xbar[profile][x]
//      = sum_nu Ibar D[x] = (K^T dy)[x].  D is never stored.  Dynamic shared memory:
//      n_state doubles.
template <bool CIA = false, int MODE = 0>
__global__ void __launch_bounds__(128) jg_rte_kernel(
    const float* __restrict__ jl, int n_out, const LayerRT* __restrict__ lrt, const JgLayer* __restrict__ jlay,
    const ProfileRT* __restrict__ prt, const JgProfile* __restrict__ jprof, const double* __restrict__ vlev,
    int L, const double* __restrict__ grid, long long n_nu, int src, ContDev cont, double* __restrict__ I,
    float* __restrict__ D, const double* __restrict__ Ibar = nullptr, double* __restrict__ xbar = nullptr) {
    extern __shared__ double jg_xsh[];
    const long long i_raw = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int p = blockIdx.y;
    const bool valid = i_raw < n_nu;
    if (MODE != 2 && !valid) return;
    // the adjoint keeps every lane to the end (warp reductions); others are clamped
    const long long i = valid ? i_raw : n_nu - 1;
    if (MODE == 2) {
        for (int x = threadIdx.x; x < jprof[p].n_state; x += blockDim.x) jg_xsh[x] = 0.0;
        __syncthreads();
    }
    const double ib = MODE == 2 && valid ? Ibar[(size_t)p * n_nu + i] : 0.0;
    const double nu = grid[i];
    const ProfileRT pr = prt[p];
    const JgProfile jp = jprof[p];
    const LayerRT* lr = lrt + (size_t)p * L;
    const JgLayer* jy = jlay + (size_t)p * L;
    const float* out = jl + (size_t)p * L * n_out * n_nu;
    const double* vl = vlev + (size_t)p * 4 * (L + 1);  // level VMR of the retrieved species
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
    const double invmu = 1.0 / pr.mu, eps = pr.eps;
    auto layer_s = [&](int k) {
        double t = (double)out[((size_t)k * n_out) * n_nu + i];
        if (cont.mask) t += cont_tau<CIA>(nu, lr[k], jy[k].dp, cont, Cs, Cf, te, Se, td, lr[k].vmr_h2o, lr[k].vmr_co2, lr[k].T_mid, cp);
        return t * invmu;
    };
    auto emission_down = [&](int k, double s, double& em, double& dem) {  // schwarzschild_jacobian.jl:221-243
        const double w = exp(-s), u = 1.0 - w;
        if (src == 0) {
            const double Ba = planck64(nu, lr[k].T_ave), Bb = planck64(nu, lr[k].T_bot);
            const double f = cim_corr(s), fp = cim_corr_d(s), core = Ba + (Bb - Ba) * f;
            em = u * core;
            dem = w * core + u * (Bb - Ba) * fp;
        } else {
            const double Bb = planck64(nu, lr[k].T_bot), Bt = planck64(nu, lr[k].T_top);
            const double fl = lit_corr(s), flp = lit_corr_d(s);
            em = Bb * u + (Bt - Bb) * fl;
            dem = Bb * w + (Bt - Bb) * flp;
        }
    };
    // pass 1: total optical depth and the downwelling radiance at the surface
    double OD = 0.0, Id = 0.0, gk = 1.0;
    for (int k = 0; k < L; ++k) {
        const double s = layer_s(k);
        OD += s;
        if (eps < 1.0) {
            double em, dem;
            emission_down(k, s, em, dem);
            Id += gk * em;
            gk *= exp(-s);
        }
    }
    const double Tr0 = exp(-OD), refl = 1.0 - eps;
    const double Bs = planck64(nu, pr.T_sfc);
    double Iv = eps * Bs * Tr0, Ib = eps * Bs * Tr0;
    const double dIde = Bs * Tr0 - (eps < 1.0 ? Id * Tr0 : 0.0);
    const double dIdTs = eps * dB_dT64(nu, pr.T_sfc) * Tr0;
    // pass 2, surface to top
    const int nT = jp.include_T ? L + 1 : 0;
    double cum = 0.0, gdn = 1.0, Id_below = 0.0;
    double carryT = 0.0, carryV[4] = {0, 0, 0, 0};
    const size_t nn = (size_t)n_nu;
    float* Dp = MODE == 0 ? D + (size_t)p * jp.n_state * nn : nullptr;
    auto emit = [&](size_t x, double val) {  // D[x][nu] = val
        if (MODE == 0) {
            Dp[x * nn + i] = (float)val;
        } else if (MODE == 2) {
            double v = valid ? val * ib : 0.0;
#pragma unroll
            for (int d = 16; d; d >>= 1) v += __shfl_xor_sync(0xffffffffu, v, d);
            if ((threadIdx.x & 31) == 0) atomicAdd(&jg_xsh[x], v);
        }
    };
    constexpr bool DERIV = MODE != 1;
    for (int m = 0; m < L; ++m) {
        const LayerRT r = lr[m];
        const JgLayer jm = jy[m];
        const double s = layer_s(m);
        cum += s;
        const double Tt = exp(-(OD - cum));  // transmittance from the top of layer m to space
        const double w = exp(-s), u = 1.0 - w;
        double e, dea, dTl_lo, dTl_hi;
        if (src == 0) {
            const double Ba = planck64(nu, r.T_ave), Bt = planck64(nu, r.T_top);
            const double f = cim_corr(s), fp = cim_corr_d(s), core = Ba + (Bt - Ba) * f;
            e = u * core;
            dea = w * core + u * (Bt - Ba) * fp;
            const double cavg = Tt * u * (1.0 - f) * dB_dT64(nu, r.T_ave);
            dTl_lo = cavg * (1.0 - jm.frac);
            dTl_hi = cavg * jm.frac + Tt * u * f * dB_dT64(nu, r.T_top);
        } else {
            const double Bb = planck64(nu, r.T_bot), Bt = planck64(nu, r.T_top);
            const double fl = lit_corr(s), flp = lit_corr_d(s);
            e = Bt * u + (Bb - Bt) * fl;
            dea = Bt * w + (Bb - Bt) * flp;
            dTl_lo = Tt * fl * dB_dT64(nu, r.T_bot);
            dTl_hi = Tt * (u - fl) * dB_dT64(nu, r.T_top);
        }
        double dIdtau = invmu * (-Ib + Tt * dea);
        if (eps < 1.0) {  // reflected downwelling, schwarzschild_jacobian.jl:210-264
            double em, dem;
            emission_down(m, s, em, dem);
            const double above = Id - Id_below - gdn * em;  // emitted above layer m
            dIdtau += refl * invmu * Tr0 * (-above + gdn * dem - Id);
            if (src == 0) {
                const double f = cim_corr(s);
                const double cavg = refl * Tr0 * gdn * u * (1.0 - f) * dB_dT64(nu, r.T_ave);
                dTl_lo += cavg * (1.0 - jm.frac) + refl * Tr0 * gdn * u * f * dB_dT64(nu, r.T_bot);
                dTl_hi += cavg * jm.frac;
            } else {
                const double fl = lit_corr(s);
                dTl_lo += refl * Tr0 * gdn * (u - fl) * dB_dT64(nu, r.T_bot);
                dTl_hi += refl * Tr0 * gdn * fl * dB_dT64(nu, r.T_top);
            }
            Id_below += gdn * em;
            gdn *= w;
        }
        Iv += Tt * e;
        Ib += Tt * e;
        // continuum derivatives by central differences (vmr_jacobian.jl:322-344)
        const float* om = out + (size_t)m * n_out * nn;
        double cT = 0.0, cvh = 0.0, cvc = 0.0;
        if (DERIV && cont.mask) {
            const double vh = r.vmr_h2o, vc = r.vmr_co2, Tm = r.T_mid;
            if (jp.include_T)
                cT = (cont_tau<CIA>(nu, r, jm.dp, cont, Cs, Cf, te, Se, td, vh, vc, Tm + 0.05, cp) -
                      cont_tau<CIA>(nu, r, jm.dp, cont, Cs, Cf, te, Se, td, vh, vc, Tm - 0.05, cp)) / 0.1;
            if (jp.retr_h2o >= 0) {
                const double h = fmax(fabs(vh), 1e-30) * 1e-6;
                cvh = (cont_tau<CIA>(nu, r, jm.dp, cont, Cs, Cf, te, Se, td, vh + h, vc, Tm, cp) -
                       cont_tau<CIA>(nu, r, jm.dp, cont, Cs, Cf, te, Se, td, vh - h, vc, Tm, cp)) / (2 * h);
            }
            if (jp.retr_co2 >= 0) {
                const double h = fmax(fabs(vc), 1e-30) * 1e-6;
                cvc = (cont_tau<CIA>(nu, r, jm.dp, cont, Cs, Cf, te, Se, td, vh, vc + h, Tm, cp) -
                       cont_tau<CIA>(nu, r, jm.dp, cont, Cs, Cf, te, Se, td, vh, vc - h, Tm, cp)) / (2 * h);
            }
        }
        if (DERIV && jp.include_T) {
            const double tlo = (double)om[1 * nn + i] + cT * (1.0 - jm.wM);
            const double thi = (double)om[2 * nn + i] + cT * jm.wM;
            emit((size_t)m, carryT + dTl_lo + dIdtau * tlo);
            carryT = dTl_hi + dIdtau * thi;
        }
        for (int rr = 0; DERIV && rr < jp.n_retr; ++rr) {
            const double cv = rr == jp.retr_h2o ? cvh : (rr == jp.retr_co2 ? cvc : 0.0);
            const double vlo = (double)om[(size_t)(3 + 2 * rr) * nn + i] + cv * (1.0 - jm.wM);
            const double vhi = (double)om[(size_t)(4 + 2 * rr) * nn + i] + cv * jm.wM;
            const double sc = jp.log_vmr ? vl[rr * (L + 1) + m] : 1.0;
            emit((size_t)(nT + rr * (L + 1) + m), sc * (carryV[rr] + dIdtau * vlo));
            carryV[rr] = dIdtau * vhi;
        }
    }
    if (DERIV && jp.include_T) emit((size_t)L, carryT);
    for (int rr = 0; DERIV && rr < jp.n_retr; ++rr) {
        const double sc = jp.log_vmr ? vl[rr * (L + 1) + L] : 1.0;
        if (DERIV) emit((size_t)(nT + rr * (L + 1) + L), sc * carryV[rr]);
    }
    int col = nT + jp.n_retr * (L + 1);
    if (DERIV && jp.include_tsfc) emit((size_t)(col++), dIdTs);
    if (DERIV && jp.include_eps) emit((size_t)(col++), dIde);
    if (eps < 1.0) Iv += refl * Id * Tr0;
    if (MODE != 2 && valid) I[(size_t)p * nn + i] = Iv;
    if (MODE == 2) {
        __syncthreads();
        for (int x = threadIdx.x; x < jp.n_state; x += blockDim.x) atomicAdd(&xbar[(size_t)p * jp.n_state + x], jg_xsh[x]);
    }
}

// ------------------------------------------------------------------ channel tail
// K[x][c] = dBT/dR_c * resample(ILS(D[x]))_c, vmr_jacobian.jl:359-380.  One warp per
// (state element, channel); the ILS taps (kernf: the normalised FP64 taps rounded to
// FP32) run over lanes (FP32 products, FP32 sums).  A window that lies inside the grid,
// as it does for every channel away from the padded ends, needs no per-tap bounds test.
__global__ void __launch_bounds__(256) jg_channel_kernel(const float* __restrict__ D, long long n_nu, int n_state,
                                                         const float* __restrict__ kernf, long long n_taps,
                                                         double dnu_hi, GridDev g, GridDev ch, int with_ils,
                                                         const double* __restrict__ R, int observable,
                                                         float* __restrict__ K) {
    const long long wid = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const int x = blockIdx.y, p = blockIdx.z;
    if (wid >= ch.n) return;
    const double nu = ch.at(wid);
    const float* Dx = D + ((size_t)p * n_state + x) * n_nu;
    auto value = [&](long long i) -> double {
        if (!with_ils) return (double)Dx[i];
        const long long half = (n_taps - 1) / 2, j0 = i - half;
        const int nt = (int)n_taps;
        float acc = 0.f;
        if (j0 >= 0 && j0 + n_taps <= n_nu) {
            const float* Dw = Dx + j0;
#pragma unroll 4
            for (int k = lane; k < nt; k += 32) acc = fmaf(Dw[k], kernf[k], acc);
        } else {
            for (int k = lane; k < nt; k += 32) {
                const long long j = j0 + k;
                if (j >= 0 && j < n_nu) acc = fmaf(Dx[j], kernf[k], acc);
            }
        }
        for (int d = 16; d; d >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, d);
        return (double)acc * dnu_hi;
    };
    double v;
    const double g0 = g.at(0), gl = g.at(n_nu - 1);
    if (nu <= g0) v = value(0);
    else if (nu >= gl) v = value(n_nu - 1);
    else {
        long long i = (long long)floor((nu - g0) / dnu_hi);
        i = max(0LL, min(i, n_nu - 2));
        while (i > 0 && g.at(i) > nu) --i;
        while (i + 2 < n_nu && g.at(i + 1) <= nu) ++i;
        const double a = g.at(i), b = g.at(i + 1), w = (nu - a) / (b - a);
        const double r0 = value(i);
        v = w == 0.0 ? r0 : r0 * (1.0 - w) + value(i + 1) * w;
    }
    if (lane == 0) {
        double scale = 1.0;
        if (observable == 0) {  // vmr_jacobian.jl:120-125
            const double Rc = R[(size_t)p * ch.n + wid];
            if (Rc <= 0.0) scale = 0.0;
            else {
                const double A = 1.191042953e-5 * (nu * nu * nu), Lg = log1p(A / Rc);
                scale = 1.4387769 * nu * A / ((Lg * Lg) * Rc * (Rc + A));
            }
        }
        K[((size_t)p * n_state + x) * ch.n + wid] = (float)(v * scale);
    }
}

// ------------------------------------------------------------------ adjoint tail
// The transpose of the channel tail for the pullback: per (profile, channel) the
// cotangent of R, rbar = dy dBT/dR (vmr_jacobian.jl:120-125; dy itself for the radiance
// observable), split onto the two grid nodes the linear resampling reads
// (sounder.jl:372-377): a0 at node ci, a1 at node ci + 1.
struct ChanAdj {
    long long ci;
    double a0, a1;
};
__global__ void __launch_bounds__(256) vjp_channel_kernel(const double* __restrict__ R, const double* __restrict__ dy,
                                                          long long n_nu, double dnu_hi, GridDev g, GridDev ch,
                                                          int observable, ChanAdj* __restrict__ out) {
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int p = blockIdx.y;
    if (c >= ch.n) return;
    const double nu = ch.at(c);
    const size_t pc = (size_t)p * ch.n + c;
    double scale = 1.0;
    if (observable == 0) {
        const double Rc = R[pc];
        if (Rc <= 0.0) scale = 0.0;
        else {
            const double A = 1.191042953e-5 * (nu * nu * nu), Lg = log1p(A / Rc);
            scale = 1.4387769 * nu * A / ((Lg * Lg) * Rc * (Rc + A));
        }
    }
    const double rb = dy[pc] * scale;
    ChanAdj a{0, 0.0, 0.0};
    const double g0 = g.at(0), gl = g.at(n_nu - 1);
    if (nu <= g0) { a.ci = 0; a.a0 = rb; }
    else if (nu >= gl) { a.ci = n_nu - 1; a.a0 = rb; }
    else {  // the node search of ils_bt_kernel
        long long i = (long long)floor((nu - g0) / dnu_hi);
        i = max(0LL, min(i, n_nu - 2));
        while (i > 0 && g.at(i) > nu) --i;
        while (i + 2 < n_nu && g.at(i + 1) <= nu) ++i;
        const double lo = g.at(i), hi = g.at(i + 1), w = (nu - lo) / (hi - lo);
        a.ci = i;
        a.a0 = w == 0.0 ? rb : rb * (1.0 - w);
        a.a1 = w == 0.0 ? 0.0 : rb * w;
    }
    out[pc] = a;
}

// Ibar[profile][j] = sum over channels of a0 K(j - ci) + a1 K(j - ci - 1), with K(k) =
// dnu_hi kern[k + half] inside the taps (apply_ils, ils.jl:131-153, transposed; zero
// outside the grid as the forward convolution) or the unit impulse without the ILS.
// One thread per grid point; the channels reaching it are found by a binary search on
// their (ascending) nodes.
__global__ void __launch_bounds__(256) ils_adjoint_kernel(const ChanAdj* __restrict__ ca, long long n_ch,
                                                          const double* __restrict__ kern, long long n_taps,
                                                          double dnu_hi, int with_ils, long long n_nu,
                                                          double* __restrict__ Ibar) {
    const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int p = blockIdx.y;
    if (j >= n_nu) return;
    const ChanAdj* c = ca + (size_t)p * n_ch;
    const long long half = with_ils ? (n_taps - 1) / 2 : 0;
    long long lo = 0, hi = n_ch;  // first channel with ci >= j - half - 1
    while (lo < hi) {
        const long long mid = (lo + hi) >> 1;
        if (c[mid].ci < j - half - 1) lo = mid + 1; else hi = mid;
    }
    double acc = 0.0;
    for (long long k = lo; k < n_ch && c[k].ci <= j + half; ++k) {
        const ChanAdj a = c[k];
        const long long d0 = j - a.ci, d1 = d0 - 1;
        if (with_ils) {
            if (d0 >= -half && d0 <= half) acc = fma(a.a0, kern[d0 + half], acc);
            if (d1 >= -half && d1 <= half) acc = fma(a.a1, kern[d1 + half], acc);
        } else {
            if (d0 == 0) acc += a.a0;
            if (d1 == 0) acc += a.a1;
        }
    }
    Ibar[(size_t)p * n_nu + j] = with_ils ? acc * dnu_hi : acc;
}

}  // namespace irs
