// linesum.cuh -- the line-by-line sum: sigma(nu_i) = max(sum_j Sn_j [H(x, y) - ped_j(nu_i)], 0)
// over lines within the cutoff (src/CrossSections/voigt.jl:243-313), times the layer
// column coef and summed over species into the layer optical depth
// (src/Sensor/sounder.jl:283-307); with VP_Y line mixing the CO2 term is
// max(sigma_V + sum_j YSn_j Im w, 0) (line_mixing.jl:1166-1186, :1351-1369).
//
// Two kernels:
//  * linesum_f64_kernel -- the plain FP64 GPU kernel: one thread per grid point,
//    a binary search per point and species for the window on the shifted centres,
//    FP64 arithmetic and IEEE division, exactly the reference kernel's structure.
//  * linesum_mixed_kernel -- FP32 + Kahan: a CTA owns a 2048-point strip of one
//    (profile, layer); each warp owns 256 contiguous points (8 per lane,
//    interleaved so stores are 128-byte coalesced); line tiles of 256 lines are
//    staged in shared memory and read as warp broadcasts; the cutoff becomes a
//    warp-uniform skip on edge tiles only; the far wing costs one MUFU
//    reciprocal and five FMA-pipe ops per pair; per-tile partial sums are added
//    into a Kahan-compensated FP32 accumulator per point.
#pragma once
#include "faddeeva.cuh"
#include "lineparams.cuh"

namespace irs {

// voigt.jl:220-236, 1-based
__device__ __forceinline__ long long lower_bound1(const double* a, double v, long long n) {
    long long lo = 1, hi = n + 1;
    while (lo < hi) {
        const long long mid = (lo + hi) >> 1;
        if (a[mid - 1] < v) lo = mid + 1; else hi = mid;
    }
    return lo;
}
__device__ __forceinline__ long long upper_bound1(const double* a, double v, long long n) {
    long long lo = 0, hi = n;
    while (lo < hi) {
        const long long mid = (lo + hi + 1) >> 1;
        if (a[mid - 1] > v) hi = mid - 1; else lo = mid;
    }
    return lo;
}

// ------------------------------------------------------------------ FP64
template <int METHOD>
__global__ void __launch_bounds__(256) linesum_f64_kernel(
    const SegDev* __restrict__ segs, const int* __restrict__ seg_count, const int2* __restrict__ pl_segs,
    LpOutF64 lp, const double* __restrict__ grid, long long n_nu, double cutoff, double x_far,
    double* __restrict__ tau) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int pl = blockIdx.y;
    if (i >= n_nu) return;
    const double nu = grid[i];
    const int2 rng = pl_segs[pl];
    double tsum = 0.0;
    const double rc = 1.0 / cutoff;
    for (int s = rng.x; s < rng.x + rng.y; ++s) {
        const SegDev sg = segs[s];
        const long long cnt = seg_count[s];
        const double* nu0 = lp.nu0 + sg.off;
        const long long jlo = lower_bound1(nu0, nu - cutoff, cnt);
        const long long jhi = upper_bound1(nu0, nu + cutoff, cnt);
        double acc = 0.0, accD = 0.0;
        const bool lm = (sg.flags & 2) != 0;
        for (long long j = jlo; j <= jhi; ++j) {
            const long long q = sg.off + j - 1;
            const double d = nu - lp.nu0[q];
            if (METHOD == 2) {  // PseudoVoigt, voigt.jl:301-311 (f = gV, y = eta, Sn = S, Hc = base)
                const double gV = lp.f[q], eta = lp.y[q];
                const double G = 0.46971863934982566 / gV * exp(-0.69314718055994531 * d * d / (gV * gV));
                const double Lz = gV * 0.31830988618379067 / (d * d + gV * gV);
                const double zr = d * rc;
                acc += lp.Sn[q] * (eta * Lz + (1.0 - eta) * G) - (2.0 - zr * zr) * lp.Hc[q];
            } else {            // voigt.jl:264-275
                const double x = d * lp.f[q];
                const double y = lp.y[q];
                const double zr = d * rc;
                const double ped = (2.0 - zr * zr) * lp.Hc[q];
                const double H = (fabs(x) > x_far ? y * kInvSqrtPi / (x * x + y * y) : hcore64<METHOD>(x, y)) - ped;
                acc += lp.Sn[q] * H;
            }
            if (lm) {  // line_mixing.jl:1177-1184
                const double x = d * lp.f[q];
                const double y = lp.y[q];
                const double imw = fabs(x) > x_far ? x * kInvSqrtPi / (x * x + y * y) : faddeeva64(x, y).y;
                accD += lp.YSn[q] * imw;
            }
        }
        double sig = fmax(acc, 0.0);
        if (lm) sig = fmax(sig + accD, 0.0);
        tsum += sig * sg.coef;
    }
    tau[(size_t)pl * n_nu + i] = tsum;
}

// ----------------------------------------------------------------- mixed
constexpr int kMxThreads = 256;
constexpr int kMxQ = 8;                          // points per lane
constexpr int kMxWarpPts = 32 * kMxQ;            // 256 points per warp
constexpr int kMxStrip = kMxThreads * kMxQ;      // 2048 points per CTA
constexpr int kMxTile = 256;                     // lines per shared-memory tile

__device__ __forceinline__ long long lower_bound0(const double* a, double v, long long n) {
    long long lo = 0, hi = n;
    while (lo < hi) {
        const long long mid = (lo + hi) >> 1;
        if (a[mid] < v) lo = mid + 1; else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ void kahan_add(float& s, float& c, float v) {
    const float y = v - c;
    const float t = s + y;
    c = (t - s) - y;
    s = t;
}

// 1/x with the MUFU approximation (max 1 ulp); x > 0 and finite here
__device__ __forceinline__ float rcp_fast(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// One tile of lines against the warp's 8 x 32 points.  For each line the warp
// decides (uniformly, every lane reads the same line) whether it is
//   out   -- beyond the cutoff for all of the warp's points: skipped;
//   fast  -- inside the cutoff and in the Lorentz far wing (|x| > x_far) for all
//            points: branch-free, one reciprocal per two pairs, pedestal folded
//            as c1*(d^2 + b^2) + c0' with the constant c0' summed once per line;
//   slow  -- anything else (Faddeeva core, cutoff edge): per-pair tests.
// p0 = (b2, a, c1, c0'), p1 = (dfar2, An, fx, y), p2 = (g, Yw, dfar, -), all in
// grid units relative to the CTA strip; see lp_write_kernel.
template <int METHOD, bool LM>
__device__ __forceinline__ void mixed_tile(int nt, const float2* __restrict__ su, const float4* __restrict__ s0,
                                           const float4* __restrict__ s1, const float4* __restrict__ s2,
                                           const float* pt, float wc, float cut, float cut2, float* tacc,
                                           float* tdsp, float& csum) {
    constexpr float kHalf = 0.5f * kMxWarpPts + 0.5f;
    for (int k = 0; k < nt; ++k) {
        const float2 u = su[k];
        const float dist = fabsf(u.x - wc);
        if (dist > cut + kHalf) continue;
        const float4 a0 = s0[k];
        const float4 a2 = s2[k];
        if (dist + kHalf <= cut && dist > a2.z + kHalf) {
            csum += a0.w;
#pragma unroll
            for (int q = 0; q < kMxQ; q += 2) {
                const float d0 = (pt[q] - u.x) - u.y;
                const float d1 = (pt[q + 1] - u.x) - u.y;
                const float e0 = fmaf(d0, d0, a0.x);
                const float e1 = fmaf(d1, d1, a0.x);
                const float R = rcp_fast(e0 * e1);
                const float r0 = e1 * R, r1 = e0 * R;
                tacc[q] = fmaf(a0.y, r0, fmaf(a0.z, e0, tacc[q]));
                tacc[q + 1] = fmaf(a0.y, r1, fmaf(a0.z, e1, tacc[q + 1]));
                if (LM) {
                    tdsp[q] = fmaf(a2.x * d0, r0, tdsp[q]);
                    tdsp[q + 1] = fmaf(a2.x * d1, r1, tdsp[q + 1]);
                }
            }
        } else {
            const float4 a1 = s1[k];
#pragma unroll
            for (int q = 0; q < kMxQ; ++q) {
                const float d = (pt[q] - u.x) - u.y;
                const float d2 = d * d;
                if (d2 > cut2) continue;
                const float e = d2 + a0.x;
                const float ped = fmaf(a0.z, e, a0.w);
                float v, vd = 0.f;
                if (d2 <= a1.x) {  // |x| <= x_far: Faddeeva core
                    const float x = d * a1.z;
                    if (METHOD == 1) {
                        v = fmaf(a1.y, weideman24_32(x, a1.w), ped);
                    } else {
                        const float2 w = faddeeva32(x, a1.w);
                        v = fmaf(a1.y, w.x, ped);
                        vd = a2.y * w.y;
                    }
                } else {
                    const float r = __frcp_rn(e);
                    v = fmaf(a0.y, r, ped);
                    vd = a2.x * d * r;
                }
                tacc[q] += v;
                if (LM) tdsp[q] += vd;
            }
        }
    }
}

// PseudoVoigt (voigt.jl:281-313): no far-wing shortcut; p0 = (gV2, aPV, c1, c0),
// p1 = (kPV, gPV, -, -): value = aPV/(d^2 + gV2) + gPV 2^(-kPV d^2) + c1 d^2 + c0.
__device__ __forceinline__ void mixed_tile_pv(int nt, const float2* __restrict__ su, const float4* __restrict__ s0,
                                              const float4* __restrict__ s1, const float* pt, float wc, float cut,
                                              float cut2, float* tacc) {
    constexpr float kHalf = 0.5f * kMxWarpPts + 0.5f;
    for (int k = 0; k < nt; ++k) {
        const float2 u = su[k];
        const float dist = fabsf(u.x - wc);
        if (dist > cut + kHalf) continue;
        const float4 a0 = s0[k];
        const float4 a1 = s1[k];
        const bool inside = dist + kHalf <= cut;
#pragma unroll
        for (int q = 0; q < kMxQ; ++q) {
            const float d = (pt[q] - u.x) - u.y;
            const float d2 = d * d;
            if (!inside && d2 > cut2) continue;
            tacc[q] += fmaf(a0.y, __frcp_rn(d2 + a0.x), fmaf(a1.y, exp2f(-a1.x * d2), fmaf(a0.z, d2, a0.w)));
        }
    }
}

template <int METHOD>
__global__ void __launch_bounds__(kMxThreads) linesum_mixed_kernel(
    const SegDev* __restrict__ segs, const int* __restrict__ seg_count, const int2* __restrict__ pl_segs,
    LpOutMixed lp, long long n_nu, float cut_g, float* __restrict__ tau) {
    __shared__ float2 su[kMxTile];
    __shared__ float4 s0[kMxTile];
    __shared__ float4 s1[kMxTile];
    __shared__ float4 s2[kMxTile];
    __shared__ long long s_rng[2];
    const int pl = blockIdx.y;
    const long long strip0 = (long long)blockIdx.x * kMxStrip;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float pt[kMxQ];
#pragma unroll
    for (int q = 0; q < kMxQ; ++q) pt[q] = (float)(warp * kMxWarpPts + q * 32 + lane);
    const float wc = (float)(warp * kMxWarpPts) + 0.5f * (kMxWarpPts - 1);
    const float cut2 = cut_g * cut_g;
    float tsum[kMxQ];
#pragma unroll
    for (int q = 0; q < kMxQ; ++q) tsum[q] = 0.f;

    const int2 rng = pl_segs[pl];
    for (int s = rng.x; s < rng.x + rng.y; ++s) {
        const SegDev sg = segs[s];
        const long long cnt = seg_count[s];
        const bool lm = (sg.flags & 2) != 0;
        if (threadIdx.x == 0) {
            // lines whose shifted centre can be within the cutoff of the strip: search
            // the sorted unshifted centres, widened by the largest pressure shift
            const double* V = lp.V + sg.off;
            s_rng[0] = lower_bound0(V, (double)strip0 - cut_g - sg.margin_g, cnt);
            s_rng[1] = lower_bound0(V, (double)(strip0 + kMxStrip - 1) + cut_g + sg.margin_g + 1e-9, cnt);
        }
        __syncthreads();
        const long long jlo = s_rng[0], jhi = s_rng[1];
        __syncthreads();
        float sum[kMxQ], comp[kMxQ], sumD[kMxQ], compD[kMxQ];
#pragma unroll
        for (int q = 0; q < kMxQ; ++q) sum[q] = comp[q] = sumD[q] = compD[q] = 0.f;
        for (long long t0 = jlo; t0 < jhi; t0 += kMxTile) {
            const int nt = (int)min((long long)kMxTile, jhi - t0);
            if (threadIdx.x < nt) {
                const long long q = sg.off + t0 + threadIdx.x;
                const double u = lp.U[q] - (double)strip0;
                const float uh = (float)u;
                su[threadIdx.x] = make_float2(uh, (float)(u - (double)uh));
                s0[threadIdx.x] = lp.p0[q];
                s1[threadIdx.x] = lp.p1[q];
                s2[threadIdx.x] = lp.p2[q];
            }
            __syncthreads();
            float tacc[kMxQ], tdsp[kMxQ];
#pragma unroll
            for (int q = 0; q < kMxQ; ++q) tacc[q] = tdsp[q] = 0.f;
            float csum = 0.f;
            if (METHOD == 2)
                mixed_tile_pv(nt, su, s0, s1, pt, wc, cut_g, cut2, tacc);
            else if (lm)
                mixed_tile<METHOD, true>(nt, su, s0, s1, s2, pt, wc, cut_g, cut2, tacc, tdsp, csum);
            else
                mixed_tile<METHOD, false>(nt, su, s0, s1, s2, pt, wc, cut_g, cut2, tacc, tdsp, csum);
#pragma unroll
            for (int q = 0; q < kMxQ; ++q) {
                kahan_add(sum[q], comp[q], tacc[q] + csum);
                if (lm) kahan_add(sumD[q], compD[q], tdsp[q]);
            }
            __syncthreads();
        }
#pragma unroll
        for (int q = 0; q < kMxQ; ++q) {
            float sig = fmaxf(sum[q], 0.f);
            if (lm) sig = fmaxf(sig + sumD[q], 0.f);
            tsum[q] += sig;
        }
    }
    float* out = tau + (size_t)pl * n_nu;
#pragma unroll
    for (int q = 0; q < kMxQ; ++q) {
        const long long i = strip0 + warp * kMxWarpPts + q * 32 + lane;
        if (i < n_nu) out[i] = tsum[q];
    }
}

}  // namespace irs
