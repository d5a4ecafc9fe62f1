// lineparams.cuh -- per-(profile, layer, species) line parameters, computed once
// into SoA buffers, with DPTMIN rejection and compaction.
//
// Restates, per line (FP64, as the reference):
//   pressure_shift                 src/HITRAN/broadening.jl:156-160
//   pressure_broadened_width       broadening.jl:40-53
//   temperature_scaled_intensity   broadening.jl:89-99, Q_ratio partition.jl:10-47
//   Doppler factor, y, Snorm, pedestal H(cutoff)   src/CrossSections/voigt.jl:402-454
//   DPTMIN peak test               voigt.jl:333-355
//   VP_Y dispersive weight         line_mixing.jl:1193-1220 with Y(T) = y0 (296/T)^0.75
//
// Two passes over (segment, chunk of kLpChunk lines): pass A decides keep/reject
// and counts per chunk; pass B recomputes the parameters of the kept lines and
// writes them compacted (order preserved), so the line sums only see kept lines.
#pragma once
#include "faddeeva.cuh"

namespace irs {

constexpr int kLpThreads = 256;
constexpr int kLpPerThread = 8;
// Both passes are latency-bound (FP64 line physics, scattered line loads): three
// 256-thread CTAs per SM (80 registers, a few spills) measured 13 % faster than the
// two that 96-128 registers allow, four (64 registers) slower again.
constexpr int kLpMinBlocks = 3;
constexpr int kLpChunk = kLpThreads * kLpPerThread;  // lines per CTA

struct ListDev {
    const double *nu, *S296, *E, *gair, *gself, *nair, *delta, *y0;
    const int* tips;
    long long n;
    int mol;
    int has_y0;
};
struct SegDev {
    double T, p_atm, vs, coef, margin_g;
    long long off;
    int list, flags;
};
struct TipsDev {
    const double* q;
    const int* tmin;
    const int* n;
    int stride;
};
struct LpConfig {
    double cutoff, x_far, dptmn;
    double grid0, dnu_g;  // grid start and spacing (mixed parameters are in grid units)
    long long n_nu;       // grid points (for the pair counts)
    double u_gran;        // granularity of the FP32 high part of the shifted centres (mixed)
    int method;           // 1 Weideman, 2 PseudoVoigt, 3 FullFaddeeva
};

__device__ __forceinline__ double tips_lookup(const TipsDev& t, int idx, double T) {
    const double* q = t.q + (size_t)idx * t.stride;
    const int n = t.n[idx];
    int lo = (int)floor(T) - t.tmin[idx] + 1;  // 1-based, partition.jl:10-18
    int hi = lo + 1;
    lo = min(max(lo, 1), n);
    hi = min(max(hi, 1), n);
    const double fr = T - floor(T);
    return q[lo - 1] * (1.0 - fr) + q[hi - 1] * fr;
}

__device__ __forceinline__ double mol_mass(int mol) {  // broadening.jl:131-148
    switch (mol) {
        case 1: return 18.010; case 2: return 44.010; case 3: return 47.998;
        case 4: return 44.013; case 5: return 28.010; case 6: return 16.043;
        case 7: return 31.999; case 8: return 34.015; case 9: return 64.065;
        case 10: return 36.461; case 11: return 17.031; default: return 30.0;
    }
}

struct LinePhys {
    double nu0s, S, gl, gd;
};

// The factors of line_phys that depend only on the segment's (T, p, vmr_self) and the
// molecule, computed once per thread instead of once per line.
struct SegPhys {
    double T, p, vs;
    double ln_tr;       // log(296/T)
    double e_self;      // (296/T)^n_self for H2O and CO2 (constant n_self), else 0
    double gd_scale;    // 3.58126e-7 sqrt(T/M): gamma_D = nu gd_scale
    double c2_T;        // c2 / T
    double dinv;        // 1/T - 1/296
    double d_self, n_self;
    int mol;
};
__device__ __forceinline__ SegPhys seg_phys(int mol, double T, double p, double vs) {
    SegPhys g;
    g.T = T; g.p = p; g.vs = vs; g.mol = mol;
    g.ln_tr = log(296.0 / T);  // (296/T)^n as exp(n ln(296/T)): one exp per exponent
    g.n_self = mol == 1 ? 0.95 : (mol == 2 ? 0.75 : 0.0);   // broadening.jl:17-20 (else n_air)
    g.d_self = mol == 1 ? 0.002 : (mol == 2 ? -0.003 : 0.0);  // :21-24
    g.e_self = (mol == 1 || mol == 2) ? exp(g.n_self * g.ln_tr) : 0.0;
    g.gd_scale = 3.58126e-7 * sqrt(T / mol_mass(mol));
    g.c2_T = 1.4387752 / T;
    g.dinv = 1.0 / T - 1.0 / 296.0;
    return g;
}

__device__ __forceinline__ LinePhys line_phys(const ListDev& L, long long j, const TipsDev& tp, const SegPhys& g) {
    const double nu = L.nu[j];
    const double n_air = L.nair[j];
    const double e_air = exp(n_air * g.ln_tr);
    const double e_self = (g.mol == 1 || g.mol == 2) ? g.e_self : e_air;
    LinePhys o;
    o.gl = e_air * L.gair[j] * (1.0 - g.vs) * g.p + e_self * L.gself[j] * g.vs * g.p;
    o.gd = nu * g.gd_scale;
    const int ti = L.tips[j];
    const double Qr = ti >= 0 ? tips_lookup(tp, ti, 296.0) / tips_lookup(tp, ti, g.T) : 296.0 / g.T;
    const double c2 = 1.4387752;
    const double stim = (1.0 - exp(-nu * g.c2_T)) / (1.0 - exp(-c2 * nu / 296.0));
    const double boltz = exp(-c2 * L.E[j] * g.dinv);
    o.S = L.S296[j] * Qr * boltz * stim;
    o.nu0s = nu + (L.delta[j] * (1.0 - g.vs) + g.d_self * g.vs) * g.p;
    return o;
}
__device__ __forceinline__ LinePhys line_phys(const ListDev& L, long long j, const TipsDev& tp,
                                              double T, double p, double vs) {
    return line_phys(L, j, tp, seg_phys(L.mol, T, p, vs));
}

// The DPTMIN decision of one line, peak coef > dptmn with peak = S f/sqrt(pi)
// erfcx(gamma_L f) (voigt.jl:340-349).  The peak is estimated in FP32 (relative error
// below 1e-5: the exponent arguments stay below 80 in magnitude, the factors are
// normal) and decides when it is more than 1e-4 away from the threshold; otherwise,
// or when an FP32 factor leaves its safe range, the FP64 evaluation decides.  The
// decision is therefore the FP64 one.
__device__ __forceinline__ bool dptmin_keep(const ListDev& L, long long j, const TipsDev& tp, const SegPhys& g,
                                            double coef, double dptmn) {
    const double nu = L.nu[j];
    const float ln_tr = (float)g.ln_tr;
    const float e_air = expf((float)L.nair[j] * ln_tr);
    const float e_self = (g.mol == 1 || g.mol == 2) ? (float)g.e_self : e_air;
    const float p = (float)g.p, vs = (float)g.vs;
    const float gl = e_air * (float)L.gair[j] * (1.f - vs) * p + e_self * (float)L.gself[j] * vs * p;
    const float gd = fmaxf((float)(nu * g.gd_scale), 1e-10f);
    const float f = 0.8325546f / gd;  // sqrt(ln 2) / gamma_D
    const int ti = L.tips[j];
    const double Qr = ti >= 0 ? tips_lookup(tp, ti, 296.0) / tips_lookup(tp, ti, g.T) : 296.0 / g.T;
    const float a_b = -1.4387752f * (float)L.E[j] * (float)g.dinv;
    const float a_s = -(float)nu * (float)g.c2_T, a_r = -1.4387752f * (float)nu * (1.0f / 296.0f);
    const float amp = (float)(L.S296[j] * coef * Qr);
    const float y = gl * f;
    const bool safe = fabsf(a_b) < 80.f && a_s > -80.f && a_r > -80.f && amp > 1e-30f && amp < 1e30f &&
                      gl > 1e-30f && y < 1e30f;
    if (safe) {
        const float stim = expm1f(a_s) / expm1f(a_r);
        const float peak = amp * expf(a_b) * stim * (f * 0.56418958f) * erfcxf(y);
        const float thr = (float)dptmn;
        if (peak > thr * 1.0001f) return true;
        if (peak < thr * 0.9999f) return false;
    }
    const LinePhys ph = line_phys(L, j, tp, g);
    const double gd64 = fmax(ph.gd, 1e-10);
    const double f64 = kSqrtLn2 / gd64;
    return (ph.S * f64 * kInvSqrtPi) * erfcx64(ph.gl * f64) * coef > dptmn;
}

// Pass A: keep flags and per-chunk kept counts.  grid = (chunks, segments)
__global__ void __launch_bounds__(kLpThreads, kLpMinBlocks) lp_keep_kernel(
    const SegDev* __restrict__ segs, const ListDev* __restrict__ lists, TipsDev tp, LpConfig cfg,
    unsigned char* __restrict__ keep, int* __restrict__ chunk_count, int n_chunks_max) {
    const SegDev sg = segs[blockIdx.y];
    const ListDev L = lists[sg.list];
    const long long base = (long long)blockIdx.x * kLpChunk;
    __shared__ int s_cnt;
    if (threadIdx.x == 0) s_cnt = 0;
    __syncthreads();
    if (base >= L.n) {
        if (threadIdx.x == 0) chunk_count[(size_t)blockIdx.y * n_chunks_max + blockIdx.x] = 0;
        return;
    }
    int cnt = 0;
    const SegPhys g = seg_phys(L.mol, sg.T, sg.p_atm, sg.vs);
    for (int r = 0; r < kLpPerThread; ++r) {
        const long long j = base + r * kLpThreads + threadIdx.x;
        if (j >= L.n) break;
        bool k = true;
        if (sg.flags & 1) k = dptmin_keep(L, j, tp, g, sg.coef, cfg.dptmn);  // DPTMIN, voigt.jl:340-349
        keep[sg.off + j] = k ? 1 : 0;
        cnt += k;
    }
    atomicAdd(&s_cnt, cnt);
    __syncthreads();
    if (threadIdx.x == 0) chunk_count[(size_t)blockIdx.y * n_chunks_max + blockIdx.x] = s_cnt;
}

struct LpOutF64 {
    double *nu0, *f, *y, *Sn, *Hc, *YSn;
};
struct LpOutMixed {
    double* V;   // unshifted centre, grid units (the sorted key of the window searches)
    float2* U;   // shifted centre, grid units, as hi + lo: hi = (float)U, lo = (float)(U - hi)
    float4 *p0, *p1;
    float4* p2;
};
// U as hi + lo with hi a multiple of the power of two g (LpConfig::u_gran, chosen so
// that |U| < 2^24 g over the grid and its cutoff margin): for an integer grid index w,
// hi - w is then a multiple of g below 2^24 g in magnitude, exact in FP32, so the
// kernels get U - w as (hi - w) + lo without FP64 arithmetic (|lo| <= g/2)
__device__ __forceinline__ float2 split_hi_lo(double u, double g, double inv_g) {
    const double h = rint(u * inv_g) * g;  // exact: g is a power of two
    return make_float2((float)h, (float)(u - h));
}

// Pass B: compacted parameters.  PREC 0 -> FP64 arrays, 1 -> mixed arrays.
template <int PREC>
__global__ void __launch_bounds__(kLpThreads, kLpMinBlocks) lp_write_kernel(
    const SegDev* __restrict__ segs, const ListDev* __restrict__ lists, TipsDev tp, LpConfig cfg,
    const unsigned char* __restrict__ keep, const int* __restrict__ chunk_count, int n_chunks_max,
    int* __restrict__ seg_count, LpOutF64 o64, LpOutMixed om, unsigned long long* __restrict__ pair_counts,
    unsigned* __restrict__ seg_core_reach) {
    const SegDev sg = segs[blockIdx.y];
    const ListDev L = lists[sg.list];
    const long long base = (long long)blockIdx.x * kLpChunk;
    if (base >= L.n) return;
    __shared__ int s_warp[kLpPerThread][kLpThreads / 32];  // kept lines per (round, warp)
    __shared__ long long s_off;
    __shared__ unsigned long long s_pairs[2];
    __shared__ unsigned s_reach;  // largest core reach of the chunk's lines (FP32 bits, >= 0)
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x < 32) {  // offset of this chunk = kept lines of the earlier chunks
        long long s = 0;
        for (int c = lane; c < (int)blockIdx.x; c += 32) s += chunk_count[(size_t)blockIdx.y * n_chunks_max + c];
        for (int d = 16; d; d >>= 1) s += __shfl_down_sync(0xffffffffu, s, d);
        if (lane == 0) {
            s_off = s;
            s_pairs[0] = s_pairs[1] = 0;
            s_reach = 0u;
            if (blockIdx.x == gridDim.x - 1 || base + kLpChunk >= L.n) {
                // last chunk of the segment publishes the segment's kept count
                const long long last = (L.n - 1) / kLpChunk;
                if ((long long)blockIdx.x == last)
                    seg_count[blockIdx.y] = (int)(s + chunk_count[(size_t)blockIdx.y * n_chunks_max + blockIdx.x]);
            }
        }
    }
    // the keep flags of every round first, so the rounds below need no block barrier
    unsigned bals[kLpPerThread];
#pragma unroll
    for (int r = 0; r < kLpPerThread; ++r) {
        const long long j = base + r * kLpThreads + threadIdx.x;
        bals[r] = __ballot_sync(0xffffffffu, j < L.n && keep[sg.off + j]);
        if (lane == 0) s_warp[r][warp] = __popc(bals[r]);
    }
    __syncthreads();
    long long run = s_off;
    unsigned long long pairs = 0, core = 0;
    float reach = 0.f;  // x_far / fx in grid units: the Faddeeva core's half-width
    const double isp = kInvSqrtPi;
    const SegPhys g = seg_phys(L.mol, sg.T, sg.p_atm, sg.vs);
    const double inv_dg = 1.0 / cfg.dnu_g, inv_gran = 1.0 / cfg.u_gran;  // u_gran: a power of two
#pragma unroll 1
    for (int r = 0; r < kLpPerThread; ++r) {
        const long long j = base + r * kLpThreads + threadIdx.x;
        const unsigned bal = bals[r];
        const bool k = (bal >> lane) & 1u;
        int before = 0, total = 0;
#pragma unroll
        for (int w = 0; w < kLpThreads / 32; ++w) {
            before += w < warp ? s_warp[r][w] : 0;
            total += s_warp[r][w];
        }
        const long long slot = sg.off + run + before + __popc(bal & ((1u << lane) - 1u));
        if (k) {
            const LinePhys ph = line_phys(L, j, tp, g);
            const double gd = fmax(ph.gd, 1e-10);
            const double f = kSqrtLn2 / gd;
            const double y = ph.gl * f;
            const double Sn = ph.S * f * isp;
            double YSn = 0.0;
            if ((sg.flags & 2) && L.has_y0) {  // line_mixing.jl:1193-1220
                const double Y = L.y0[j] * exp(0.75 * g.ln_tr);  // y0 (296/T)^0.75
                if (Y != 0.0 && ph.S > 0.0) YSn = Y * sg.p_atm * Sn;
            }
            const double c = cfg.cutoff;
            // pair counts inside the cutoff on the uniform grid (roofline work units)
            {
                const double last = (double)(cfg.n_nu - 1);
                const double u = (ph.nu0s - cfg.grid0) * inv_dg;
                const double lo = fmax(ceil(u - c * inv_dg), 0.0);
                const double hi = fmin(floor(u + c * inv_dg), last);
                if (hi >= lo) pairs += (unsigned long long)(hi - lo + 1);
                const double wc = fmin(cfg.x_far * gd * (1.0 / kSqrtLn2), c) * inv_dg;
                const double clo = fmax(ceil(u - wc), 0.0);
                const double chi = fmin(floor(u + wc), last);
                if (chi >= clo) core += (unsigned long long)(chi - clo + 1);
            }
            if (cfg.method == 2) {  // PseudoVoigt, voigt.jl:422-441
                const double fG = 2.0 * gd, fL = 2.0 * ph.gl;
                const double fV = pow(pow(fG, 5.0) + 2.69269 * pow(fG, 4.0) * fL + 2.42843 * pow(fG, 3.0) * (fL * fL) +
                                      4.47163 * (fG * fG) * pow(fL, 3.0) + 0.07842 * fG * pow(fL, 4.0) + pow(fL, 5.0), 0.2);
                const double rr = fL / fV;
                const double gV = 0.5 * fV;
                const double eta = 1.36603 * rr - 0.47719 * (rr * rr) + 0.11116 * (rr * rr * rr);
                const double cG = 0.46971863934982566;  // sqrt(log(2)/pi)
                const double Gc = cG / gV * exp(-0.69314718055994531 * (c * c) / (gV * gV));
                const double Lc = gV * 0.31830988618379067 / (c * c + gV * gV);
                const double basev = ph.S * (eta * Lc + (1.0 - eta) * Gc);
                if (PREC == 0) {
                    o64.nu0[slot] = ph.nu0s; o64.f[slot] = gV; o64.y[slot] = eta;
                    o64.Sn[slot] = ph.S; o64.Hc[slot] = basev; o64.YSn[slot] = YSn;
                } else {
                    const double dg = cfg.dnu_g, co = sg.coef;
                    const double gVg = gV / dg;
                    om.V[slot] = (L.nu[j] - cfg.grid0) * inv_dg;
                    om.U[slot] = split_hi_lo((ph.nu0s - cfg.grid0) * inv_dg, cfg.u_gran, inv_gran);
                    const double P = basev * co;
                    om.p0[slot] = make_float4((float)(gVg * gVg), (float)(ph.S * co * eta * gVg / (M_PI * dg)),
                                              (float)(P * (dg / c) * (dg / c)), (float)(-2.0 * P));
                    om.p1[slot] = make_float4((float)(1.0 / (gVg * gVg)),
                                              (float)(ph.S * co * (1.0 - eta) * cG / gV), 0.f, 0.f);
                    om.p2[slot] = make_float4(0.f, 0.f, 0.f, 0.f);
                }
            } else {
                const double xc = c * f;
                double Hc;
                if (fabs(xc) > cfg.x_far) Hc = y * isp / (xc * xc + y * y);
                else Hc = cfg.method == 1 ? weideman24_64(xc, y) : faddeeva64(xc, y).x;
                if (PREC == 0) {
                    o64.nu0[slot] = ph.nu0s; o64.f[slot] = f; o64.y[slot] = y;
                    o64.Sn[slot] = Sn; o64.Hc[slot] = Hc; o64.YSn[slot] = YSn;
                } else {
                    const double dg = cfg.dnu_g, co = sg.coef;
                    const double fx = f * dg;         // x per grid unit
                    const double ifx = gd * (1.0 / kSqrtLn2) * inv_dg;  // 1 / fx
                    const double An = Sn * co;        // tau per unit H
                    const double P = An * Hc;         // pedestal scale
                    const double Yw = YSn * co;
                    om.V[slot] = (L.nu[j] - cfg.grid0) * inv_dg;
                    om.U[slot] = split_hi_lo((ph.nu0s - cfg.grid0) * inv_dg, cfg.u_gran, inv_gran);
                    // b^2 floored at 1e-12 grid units^2 (gamma_L ~ 1e-9 cm^-1) so the far-wing
                    // denominators stay normal in FP32 even at p -> 0
                    const double b = y * ifx;         // gamma_L in grid units
                    const double b2 = fmax(b * b, 1e-12);
                    const double dfar = cfg.x_far * ifx;
                    reach = fmaxf(reach, (float)fmin(dfar, 1.0e30));
                    const double c1 = P * (dg / c) * (dg / c);
                    om.p0[slot] = make_float4((float)b2, (float)(An * b * isp * ifx), (float)c1, (float)(-2.0 * P));
                    om.p1[slot] = make_float4((float)fmin(dfar * dfar, 3.0e38), (float)An, (float)fx, (float)y);
                    om.p2[slot] = make_float4((float)(Yw * isp * ifx), (float)Yw, (float)fmin(dfar, 1.0e30), 0.f);
                }
            }
        }
        run += total;
    }
    for (int d = 16; d; d >>= 1) {
        pairs += __shfl_down_sync(0xffffffffu, pairs, d);
        core += __shfl_down_sync(0xffffffffu, core, d);
    }
    for (int d = 16; d; d >>= 1) reach = fmaxf(reach, __shfl_xor_sync(0xffffffffu, reach, d));
    if (lane == 0) {
        atomicAdd(&s_pairs[0], pairs);
        atomicAdd(&s_pairs[1], core);
        atomicMax(&s_reach, __float_as_uint(reach));  // non-negative floats order as their bits
    }
    __syncthreads();
    if (threadIdx.x == 0 && pair_counts) {
        atomicAdd(&pair_counts[0], s_pairs[0]);
        atomicAdd(&pair_counts[1], s_pairs[1]);
    }
    if (threadIdx.x == 0 && seg_core_reach) atomicMax(&seg_core_reach[blockIdx.y], s_reach);
}

}  // namespace irs
