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
#include "irs_internal.h"
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
    double* __restrict__ tau, double* __restrict__ pert, long long pstride) {
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
        if (pert && (sg.flags & SEG_RELMAT)) {  // relmat line mixing: finished by relmat_finish_kernel
            pert[(size_t)pl * pstride + i] = sig;
            continue;
        }
        tsum += sig * sg.coef;
    }
    tau[(size_t)pl * n_nu + i] = tsum;
}

// ----------------------------------------------------------------- mixed
// Each warp owns 128 consecutive grid points (4 per lane, point = 32 q + lane)
// and walks its own window of lines in tiles of 32 staged in warp-private shared
// memory (no block-wide barriers).  The staging lane of each line precomputes,
// once per (warp, line): the FP32 position split u = uh + ul relative to the
// warp, the class of the line for this warp (outside the cutoff / fast / slow),
// and, for fast lines, the line's pedestal as a quadratic in the point index, so
// the 32 pedestals of a tile reduce to three numbers.
//   fast: inside the cutoff and in the Lorentz far wing (|x| > x_far) for all 128
//         points: d by one FADD from a per-line origin, one MUFU reciprocal per
//         two pairs, one FMA into the tile sum;
//   slow: Faddeeva core or cutoff edge: per-pair tests.
// Tile sums go into a Kahan-compensated FP32 accumulator per point.
constexpr int kMxWarps = 16;
constexpr int kMxThreads = 32 * kMxWarps;
constexpr int kMxQ = 4;                               // points per lane
constexpr int kMxWarpPts = 32 * kMxQ;                 // 128 points per warp
constexpr int kMxStrip = kMxWarps * kMxWarpPts;       // 2048 points per CTA
constexpr unsigned kFull = 0xffffffffu;

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

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int d = 16; d; d >>= 1) v += __shfl_xor_sync(kFull, v, d);
    return v;
}

// Inner points of a slow line: |x| + y < 15 (plus one point each side), where
// faddeeva32 takes its CF4 or Weideman branch.  They span a few points of one or two
// 32-point rows, so evaluating them inside the per-point loop leaves most lanes of
// those rows idle; instead each tile evaluates the inner points of all its slow lines
// lane-parallel into cw (up to kCoreBuf per tile; lines beyond it keep the per-point
// evaluation) and the per-point loop reads them back.
constexpr int kCoreBuf = 128;

struct WarpTile {
    float4 fu[32];  // fast lines: uh, ul, b2, a               (PV: uh, ul, -, class)
    float4 su[32];  // slow lines: uh, ul, b2, a               (PV: gV2, aPV, c1, c0)
    float4 sp[32];  // slow lines: c1, c0, dfar2, An           (PV: kPV, gPV, -, -)
    float4 sq[32];  // slow lines: fx, y, g, Yw
    float fg[32];   // fast lines: g (dispersive line mixing)
    float4 ff[32];  // far lines: uh, ul, b2, a
    float ffg[32];  // far lines: g
    float4 eu[32];  // cutoff-edge lines (far field only): uh, ul, b2, a
    float4 ep[32];  // cutoff-edge lines: c1, c0, g, -
    int4 sr[32];    // slow lines (FullFaddeeva): inner points [x, y] of the block, their offset z in cw
    float2 cw[kCoreBuf];  // w(x + i y) at the inner points of the tile's slow lines, line after line
    // mid lines (far field only) share su/sp/sq with the slow lines, from the top
    // down (position 31 - k): su = (uh, ul, b2, a), sp = (c1, c0, fx, y),
    // sq = (An, g, Yw, dfar2)
};


// Far field.  A fast line whose centre lies kFarDist or more points from the centre
// of a warp's 128-point block contributes a function of the point index that is
// analytic well beyond the block (its poles sit at complex distance >= kFarDist - 64
// from it), so its far-wing sum over all such lines is evaluated at the 8 Chebyshev
// nodes of the block and interpolated to the 128 points with the fixed Lagrange
// weights L_k(i): 8 pairs per line instead of 128.  The interpolation error of one
// line's term is at most 1.6e-7 of its largest value on the block (degree 7, nodes
// on [0, 127], distance 320 = 5 half-widths); pedestals stay exact (quadratic sums),
// as do the near lines, the Faddeeva cores and the cutoff edges.
constexpr float kFarDist = 2.5f * kMxWarpPts;
constexpr int kFarNodes = 8;
struct FarTable {
    float L[kFarNodes][kMxWarpPts];  // L_k(i), i = 0..127
};
__device__ __forceinline__ double far_node(int k) {
    constexpr double h = 0.5 * (kMxWarpPts - 1);
    return h + h * cos((2 * k + 1) * 3.14159265358979323846 / (2 * kFarNodes));
}
// the same nodes rounded to FP32, as literals for fully unrolled node loops
__device__ __forceinline__ float far_node_f(int k) {
    static_assert(kMxWarpPts == 128, "far_node_f holds the nodes of a 128-point block");
    return k == 0 ? 1.257798691e+02f : k == 1 ? 1.162983170e+02f : k == 2 ? 9.877870941e+01f
         : k == 3 ? 7.588823700e+01f : k == 4 ? 5.111176300e+01f : k == 5 ? 2.822129059e+01f
         : k == 6 ? 1.070167923e+01f : 1.220134735e+00f;
}
// whole block, before any early exit
__device__ __forceinline__ void far_table_init(FarTable& F) {
    for (int idx = threadIdx.x; idx < kFarNodes * kMxWarpPts; idx += blockDim.x) {
        const int k = idx / kMxWarpPts, i = idx % kMxWarpPts;
        double v = 1.0;
        for (int j = 0; j < kFarNodes; ++j)
            if (j != k) v *= ((double)i - far_node(j)) / (far_node(k) - far_node(j));
        F.L[k][i] = (float)v;
    }
}

// Strip far field.  A line whose shifted centre lies kCtaR or more points from the
// centre of a 2048-point strip (the 8 warps of a CTA), and whose cutoff covers the
// whole strip, is a function of the point index analytic well beyond the strip: its
// far wing is evaluated once per strip at kCtaNodes Chebyshev nodes (by
// strip_far_kernel, the 8 warps sharing the lines) instead of once per warp, and the
// degree-23 interpolant is taken to each warp's 8 nodes by the fixed matrix M, where
// it joins the warp's own far field.  Worst error of one line's term: 2.2e-9 of its
// largest value on the strip (poles at distance >= 1536 from its centre; 16 nodes at
// 2048, the earlier choice, gave 1.4e-8 and left a quarter more lines to every warp's
// window).  The
// pedestals of these lines are quadratics summed exactly as for the warp's far lines
// (compensated, then evaluated at the nodes, which interpolation reproduces).  The
// lines are those with unshifted centre V in [c - rout, c - rin) or [c + rin, c + rout),
// rin = max(kCtaR, core reach + 1025) + margin, rout = cut - 1024 - margin (margin >= the
// pressure shift + 2 points; core reach = the segment's largest x_far / fx, so no line
// of the ranges has its Faddeeva core on the strip): one index range each side, taken
// out of every warp's window.
constexpr int kCtaNodes = 24;
constexpr float kCtaR = 1536.f;
constexpr double kCtaCentre = 0.5 * (kMxStrip - 1);  // 1023.5
constexpr int kStripWords = kMxWarps * kFarNodes;    // per (segment, strip): the warps' node values
// the nodes relative to the strip centre, 1023.5 cos((2k+1) pi / 48), rounded to FP32
__device__ __forceinline__ float cta_node_f(int k) {
    const int a = k < 12 ? k : 23 - k;
    const float v = a == 0 ? 1.021308594e+03f : a == 1 ? 1.003833740e+03f : a == 2 ? 9.691829834e+02f
                  : a == 3 ? 9.179492798e+02f : a == 4 ? 8.510091553e+02f : a == 5 ? 7.695080566e+02f
                  : a == 6 ? 6.748404541e+02f : a == 7 ? 5.686261597e+02f : a == 8 ? 4.526824646e+02f
                  : a == 9 ? 3.289932861e+02f : a == 10 ? 1.996749420e+02f : 6.694010162e+01f;
    return k < 12 ? v : -v;
}

// First index i in [0, n) with a[i] >= v (n if none), found by the whole warp: each
// round probes 32 evenly spaced positions and keeps the interval between the last
// probe below v and the first one at or above it (32-ary search: 4 dependent loads
// for 66 k lines instead of 17).  All lanes return the same value.
__device__ __forceinline__ long long warp_lower_bound(const double* a, double v, long long n, int lane) {
    long long lo = 0, hi = n;  // the answer lies in [lo, hi]
    while (hi - lo > 32) {
        const long long step = (hi - lo + 31) / 32;
        const long long p = min(lo + (long long)(lane + 1) * step - 1, hi - 1);
        const unsigned below = __ballot_sync(kFull, a[p] < v);  // a prefix of the lanes
        const int c = __popc(below);
        const long long nlo = lo + (long long)c * step;
        hi = min(hi, lo + (long long)(c + 1) * step);
        lo = min(nlo, hi);
    }
    const long long p = lo + lane;
    const unsigned below = __ballot_sync(kFull, p < hi && a[p] < v);
    return lo + __popc(below);
}

// window [jlo, jhi) of the lines that can reach this warp's points [wb, wb + kMxWarpPts - 1]
__device__ __forceinline__ void warp_window(const LpOutMixed& lp, const SegDev& sg, long long cnt,
                                            long long wb, float cut, int lane, long long& jlo, long long& jhi) {
    const double* V = lp.V + sg.off;
    jlo = warp_lower_bound(V, (double)wb - cut - sg.margin_g, cnt, lane);
    jhi = warp_lower_bound(V, (double)(wb + kMxWarpPts - 1) + cut + sg.margin_g + 1e-9, cnt, lane);
}

// Fast line, two points q and q+1 with packed FP32x2 arithmetic.  The squared
// distances are formed in swapped order es = (e[q+1], e[q]) so one reciprocal of
// their product gives both reciprocals with a single packed multiply:
//   r = es * (1/(e[q] e[q+1])) = (1/e[q], 1/e[q+1]).
__device__ __forceinline__ void fast_pair(float2 d0s, float2 offs, float2 b2, float2 a, float2& acc) {
    const float2 dds = __fadd2_rn(d0s, offs);       // (d[q+1], d[q])
    const float2 es = __ffma2_rn(dds, dds, b2);     // (e[q+1], e[q])
    const float R = rcp_fast(es.x * es.y);
    const float2 r = __fmul2_rn(es, make_float2(R, R));
    acc = __ffma2_rn(a, r, acc);
}

// ------------------------------------------------------------ strip far field
// M[w][j][k] = L_k(node j of warp w) for the strip nodes k, at the FP32 nodes the
// kernel evaluates; one thread per entry, once per line sum
__global__ void strip_table_kernel(float* __restrict__ M) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kMxWarps * kFarNodes * kCtaNodes) return;
    const int w = i / (kFarNodes * kCtaNodes), j = (i / kCtaNodes) % kFarNodes, k = i % kCtaNodes;
    const double x = (double)kMxWarpPts * w + far_node(j) - kCtaCentre;
    const double xk = (double)cta_node_f(k);
    double v = 1.0;
    for (int l = 0; l < kCtaNodes; ++l)
        if (l != k) v *= (x - (double)cta_node_f(l)) / (xk - (double)cta_node_f(l));
    M[i] = (float)v;
}

constexpr int kStripSegs = 16;  // segments whose ranges are searched together
constexpr int kStripUnroll = 4;  // tiles in flight per warp
constexpr int kStripWarps = 8;   // warps of strip_far_kernel (each serves kMxWarps / 8 line-sum warps)
constexpr int kStripThreads = 32 * kStripWarps;

// One CTA per (strip, profile-layer).  The segments' index ranges are searched first,
// spread over the warps (kStripSegs segments at a time); then each warp walks every
// segment's lines without waiting for the others (tiles warp, warp + 8, ... of the two
// ranges, kStripUnroll tiles per round with their loads issued together; each line at
// the 16 nodes) and leaves its node and pedestal sums in the segment's slot; after one
// block barrier each warp combines the slots of every segment (the warps in a fixed
// order) and takes them through M to its own 8 nodes: far[(segment, strip)][warp][node],
// and ranges[(segment, strip)].  Segments with line mixing (when the line sum treats
// them so) are left out; strips without such lines get empty ranges and zero values.
template <bool ANY_LM>
__global__ void __launch_bounds__(kStripThreads, 3) strip_far_kernel(
    const SegDev* __restrict__ segs, const int* __restrict__ seg_count, const unsigned* __restrict__ core_reach,
    const int2* __restrict__ pl_segs, LpOutMixed lp, float cut_g, int n_strips, const float* __restrict__ M,
    float* __restrict__ far, int4* __restrict__ ranges, unsigned long long* __restrict__ evald, int pl0, int seg0) {
    __shared__ float slot[kStripSegs][kStripWarps][kCtaNodes + 4];  // node sums, pedestal A, B, C
    __shared__ int sj[kStripSegs][4];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int strip = blockIdx.x, pl = pl0 + (int)blockIdx.y;  // cells counted from segment seg0
    const long long cb = (long long)strip * kMxStrip;
    const double c = (double)cb + kCtaCentre;
    unsigned long long work = 0;
    const int2 rng = pl_segs[pl];
    for (int s0 = rng.x; s0 < rng.x + rng.y; s0 += kStripSegs) {  // block-uniform
        const int ns = min(kStripSegs, rng.x + rng.y - s0);
        for (int i = warp; i < 4 * ns; i += kStripWarps) {  // search i: bound i % 4 of segment i / 4
            const SegDev sg = segs[s0 + i / 4];
            // rin: the interpolation distance, and every line's Faddeeva core (|x| <= x_far)
            // off the strip
            const double reach = (double)__uint_as_float(core_reach[s0 + i / 4]);
            const double m = sg.margin_g, rin = fmax((double)kCtaR, reach + 0.5 * kMxStrip + 1.0) + m;
            const double rout = (double)cut_g - 0.5 * kMxStrip - m;
            int j = 0;
            if (rout > rin && !(ANY_LM && (sg.flags & 2))) {
                const int b = i % 4;
                const double v = b == 0 ? c - rout : b == 1 ? c - rin : b == 2 ? c + rin : c + rout;
                j = (int)warp_lower_bound(lp.V + sg.off, v, seg_count[s0 + i / 4], lane);
            }
            if (lane == 0) sj[i / 4][i % 4] = j;
        }
        __syncthreads();
        for (int si = 0; si < ns; ++si) {
            const long long off = segs[s0 + si].off;
            const int jA = sj[si][0], jB = sj[si][1], jC = sj[si][2], jD = sj[si][3];
            const int nL = jB - jA, n = nL + (jD - jC);
            float2 acc[kCtaNodes / 2];
#pragma unroll
            for (int h = 0; h < kCtaNodes / 2; ++h) acc[h] = make_float2(0.f, 0.f);
            float PA = 0.f, PAc = 0.f, PB = 0.f, PBc = 0.f, PC = 0.f, PCc = 0.f;
            for (int t0 = warp * 32; t0 < n; t0 += kStripUnroll * 32 * kStripWarps) {
                float2 uf[kStripUnroll];
                float4 a0[kStripUnroll];
#pragma unroll
                for (int u = 0; u < kStripUnroll; ++u) {  // the loads first
                    const int t = t0 + u * 32 * kStripWarps + lane;
                    if (t < n) {
                        const long long q = off + (t < nL ? jA + t : jC + (t - nL));
                        uf[u] = lp.U[q];
                        a0[u] = lp.p0[q];
                    }
                }
#pragma unroll
                for (int u = 0; u < kStripUnroll; ++u) {
                    const int t = t0 + u * 32 * kStripWarps + lane;
                    float pa = 0.f, pb = 0.f, pc = 0.f;
                    if (t < n) {
                        const float uc = (uf[u].x - (float)cb) - (float)kCtaCentre;  // exact: see split_hi_lo
                        const float ul = uf[u].y;
                        const float2 b2 = make_float2(a0[u].x, a0[u].x), aa = make_float2(a0[u].y, a0[u].y);
#pragma unroll
                        for (int k = 0; k < kCtaNodes; k += 2) {  // pairs of nodes, one reciprocal per pair
                            const float2 xs = make_float2(cta_node_f(k + 1), cta_node_f(k));  // swapped
                            const float2 ds = __fadd2_rn(__fadd2_rn(xs, make_float2(-uc, -uc)), make_float2(-ul, -ul));
                            const float2 es = __ffma2_rn(ds, ds, b2);                       // (e[k+1], e[k])
                            const float R = rcp_fast(es.x * es.y);
                            const float2 r = __fmul2_rn(es, make_float2(R, R));             // (1/e[k], 1/e[k+1])
                            acc[k / 2] = __ffma2_rn(aa, r, acc[k / 2]);
                        }
                        // c1 (x - u)^2 + c0 = c1 x^2 - 2 c1 u x + (c1 u^2 + c0), x from the centre
                        pa = a0[u].z;
                        pb = a0[u].z * uc;
                        pc = fmaf(pb, uc, a0[u].w);
                    }
                    kahan_add(PA, PAc, pa);
                    kahan_add(PB, PBc, pb);
                    kahan_add(PC, PCc, pc);
                }
                if (lane == 0) work += (unsigned long long)min(kStripUnroll * 32, n - t0) * kCtaNodes;
            }
            float* sl = slot[si][warp];
#pragma unroll
            for (int h = 0; h < kCtaNodes / 2; ++h) {
                const float x = warp_sum(acc[h].x), y = warp_sum(acc[h].y);
                if (lane == 0) {
                    sl[2 * h] = x;
                    sl[2 * h + 1] = y;
                }
            }
            const float A = warp_sum(PA - PAc), B = warp_sum(PB - PBc), Cc = warp_sum(PC - PCc);
            if (lane == 0) {
                sl[kCtaNodes] = A;
                sl[kCtaNodes + 1] = B;
                sl[kCtaNodes + 2] = Cc;
            }
        }
        __syncthreads();
        // per segment: the strip's node values (lane k < 16: node k, the warps in a fixed
        // order, plus the pedestal quadratic), then through M to the 8 nodes of the
        // line-sum warps this warp serves
        float xk = 0.f;
#pragma unroll
        for (int k = 0; k < kCtaNodes; ++k) xk = lane == k ? cta_node_f(k) : xk;
        for (int si = 0; si < ns; ++si) {
            float fc = 0.f, SA = 0.f, SB = 0.f, SC = 0.f;
#pragma unroll
            for (int w = 0; w < kStripWarps; ++w) {
                if (lane < kCtaNodes) fc += slot[si][w][lane];
                SA += slot[si][w][kCtaNodes];
                SB += slot[si][w][kCtaNodes + 1];
                SC += slot[si][w][kCtaNodes + 2];
            }
            fc += fmaf(xk, fmaf(xk, SA, -2.f * SB), SC);
            const size_t cell = (size_t)(s0 + si - seg0) * n_strips + strip;
            for (int mw = warp; mw < kMxWarps; mw += kStripWarps) {
                const float* Mw = M + ((size_t)mw * kFarNodes + (lane & (kFarNodes - 1))) * kCtaNodes;
                float g = 0.f;
#pragma unroll
                for (int k = 0; k < kCtaNodes; ++k) g = fmaf(__ldg(Mw + k), __shfl_sync(kFull, fc, k), g);
                if (lane < kFarNodes) far[cell * kStripWords + mw * kFarNodes + lane] = g;
            }
            if (threadIdx.x == 0) ranges[cell] = make_int4(sj[si][0], sj[si][1], sj[si][2], sj[si][3]);
        }
        if (s0 + kStripSegs < rng.x + rng.y) __syncthreads();  // slots and ranges reused by the next batch
    }
    if (evald && lane == 0 && work) atomicAdd(evald, work);
}

// The optical-depth row of a warp's 128 points.  Each segment's clamped sums are
// added to it in segment order (the first one stores), so no per-point total stays
// in registers from one segment to the next.
struct OutRow {
    float* p;    // tau at the warp's first point
    int n;       // the warp's points inside the grid
    bool wrote;  // a segment has stored
};
__device__ __forceinline__ void out_add(OutRow& o, int q, int lane, float sig) {
    const int i = 32 * q + lane;
    if (i < o.n) o.p[i] = o.wrote ? o.p[i] + sig : sig;
}

// the next tile start: past the end a of the first range to b, past c to d
__device__ __forceinline__ int skip_ranges(int t, int a, int b, int c, int d) {
    t = t == a ? b : t;
    return t == c ? d : t;
}

template <int METHOD, bool LM, bool FAR>
__device__ __forceinline__ void warp_segment(const SegDev& sg, long long cnt, const LpOutMixed& lp, long long wb,
                                             float cut, float cut2, int lane, WarpTile& T, const FarTable& FT,
                                             float xn, OutRow& orow, unsigned long long& work,
                                             double* __restrict__ prow, int4 sx, float gnode) {
    constexpr float kCentre = 0.5f * (kMxWarpPts - 1);
    constexpr float kHalf = 0.5f * kMxWarpPts + 0.5f;
    long long jlo, jhi;
    warp_window(lp, sg, cnt, wb, cut, lane, jlo, jhi);
    const float pl0 = (float)lane;
    // per-lane constant offsets of the point pairs, swapped: (32(q+1), 32q)
    float2 offs[kMxQ / 2];
#pragma unroll
    for (int h = 0; h < kMxQ / 2; ++h) offs[h] = make_float2(32.f * (2 * h + 1), 32.f * (2 * h));
    float sum[kMxQ], comp[kMxQ], sumD[kMxQ], compD[kMxQ];
#pragma unroll
    for (int q = 0; q < kMxQ; ++q) sum[q] = comp[q] = sumD[q] = compD[q] = 0.f;
    // with line mixing, far-field node sums of the staged far lines: lane l accumulates
    // node l % 8 over every fourth far line
    float farS = 0.f, farC = 0.f, farDS = 0.f, farDC = 0.f;
    // with the far field, each lane accumulates its own lines' pedestal quadratics
    // A p^2 - 2 B p + C and the warp reduces them once per segment, so tiles holding only
    // far lines need no per-point work.  B and C are compensated; A is a plain sum: with
    // c1 = P / cut^2 and c0 = -2 P, A p^2 is below p^2 / (2 cut^2) of C at the block's
    // points, so its rounding does not reach the result
    float PA = 0.f, PAc = 0.f, PB = 0.f, PBc = 0.f, PC = 0.f, PCc = 0.f;
    // without line mixing each lane evaluates its own far lines at the 8 nodes and
    // accumulates them here (reduced across the warp once)
    float2 fnode[kFarNodes / 2];  // nodes (2h, 2h + 1)
#pragma unroll
    for (int h = 0; h < kFarNodes / 2; ++h) fnode[h] = make_float2(0.f, 0.f);
    const unsigned lt = (1u << lane) - 1u;
    // the window without the strip far field's ranges [sx.x, sx.y) and [sx.z, sx.w):
    // [ilo, ra), [rb, rc) and [rd, ihi), walked in turn (indices within a segment fit
    // in int: seg_count is an int)
    const int ilo = (int)jlo, ihi = (int)jhi;
    const int ra = min(max(sx.x, ilo), ihi), rb = min(max(sx.y, ilo), ihi);
    const int rc = min(max(sx.z, ilo), ihi), rd = min(max(sx.w, ilo), ihi);
    int nt = 0;
    for (int t0 = skip_ranges(ilo, ra, rb, rc, rd); t0 < ihi; t0 = skip_ranges(t0 + nt, ra, rb, rc, rd)) {
        nt = min(32, (t0 < ra ? ra : t0 < rc ? rc : ihi) - t0);
        float pa = 0.f, pb = 0.f, pc = 0.f;  // this line's pedestal quadratic (fast and far lines)
        int cls = 0;
        float4 a0, a1, a2;
        float uh = 0.f, ul = 0.f;
        if (lane < nt) {
            const long long q = sg.off + t0 + lane;
            const float2 uf = lp.U[q];
            uh = uf.x - (float)wb;  // exact: see split_hi_lo
            ul = uf.y;
            a0 = lp.p0[q];
            a2 = lp.p2[q];
            const float dist = fabsf(uh - kCentre);
            if (dist > cut + kHalf) cls = 0;
            else if (FAR && dist + kHalf > cut && dist > a2.z + kHalf) {
                cls = 4;  // far wing at every point, the cutoff falls among the points
            } else if (dist + kHalf <= cut && dist > a2.z + kHalf) {
                cls = (FAR && dist >= kFarDist) ? 3 : 1;
                // sum over points p of c1 (p - u)^2 + c0 = p^2 c1 - 2 p c1 u + (c1 u^2 + c0)
                pa = a0.z;
                pb = a0.z * uh;
                pc = fmaf(pb, uh, a0.w);
            } else {
                cls = 2;
                a1 = lp.p1[q];
                // mid: inside the cutoff, and |x| + y >= 15 at every point (the continued
                // fraction of faddeeva32 or the far wing, no Weideman/CF4 region)
                if (FAR && METHOD == 3 && dist + kHalf <= cut && fmaxf(dist - kHalf, 0.f) * a1.z + a1.w >= 15.05f)
                    cls = 5;
            }
        }
        // without line mixing each lane evaluates its own far line at the 8 nodes (summed
        // across the warp once per segment); tiles holding only far lines and lines out
        // of reach then need nothing else
        if (FAR && !LM) {
            if (cls == 3) {  // nodes in pairs, packed: one reciprocal of the product per pair
                const float2 u2 = make_float2(uh, uh), l2 = make_float2(ul, ul);
                const float2 b2 = make_float2(a0.x, a0.x), aa = make_float2(a0.y, a0.y);
#pragma unroll
                for (int k = 0; k < kFarNodes; k += 2) {
                    const float2 xs = make_float2(far_node_f(k + 1), far_node_f(k));  // swapped
                    const float2 ds = __fadd2_rn(__fadd2_rn(xs, make_float2(-u2.x, -u2.y)),
                                                 make_float2(-l2.x, -l2.y));
                    const float2 es = __ffma2_rn(ds, ds, b2);                       // (e[k+1], e[k])
                    const float R = rcp_fast(es.x * es.y);
                    const float2 r = __fmul2_rn(es, make_float2(R, R));             // (1/e[k], 1/e[k+1])
                    fnode[k / 2] = __ffma2_rn(aa, r, fnode[k / 2]);
                }
            }
            const unsigned nfar = __popc(__ballot_sync(kFull, cls == 3));
            if (lane == 0) work += (unsigned long long)nfar * kFarNodes;
            if (__all_sync(kFull, cls == 3 || cls == 0)) {
                PA += pa;
                kahan_add(PB, PBc, pb);
                kahan_add(PC, PCc, pc);
                continue;
            }
        }
        // FullFaddeeva slow lines: the inner points of the block, [plo, plo + nin - 1],
        // and their offsets in cw by a warp scan; cfit = the points that fit (warp-uniform)
        int nin = 0, plo = 1, coff = 0, cfit = 0;
        const unsigned sm = __ballot_sync(kFull, cls == 2);
        if (METHOD == 3 && sm) {  // (warp-uniform)
            if (cls == 2 && a1.w < 15.f) {
                const float hw = (15.f - a1.w) / a1.z + 1.f;
                const float c = uh + ul;
                const float lo = fmaxf(c - hw, 0.f), hi = fminf(c + hw, (float)(kMxWarpPts - 1));
                if (lo <= hi) {
                    plo = (int)ceilf(lo);
                    nin = max((int)floorf(hi) - plo + 1, 0);
                }
            }
            int inc = nin;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const int t = __shfl_up_sync(kFull, inc, d);
                if (lane >= d) inc += t;
            }
            coff = inc - nin;
            const unsigned ov = __ballot_sync(kFull, inc > kCoreBuf && nin > 0);
            cfit = ov ? __shfl_sync(kFull, coff, __ffs(ov) - 1) : __shfl_sync(kFull, inc, 31);
            if (inc > kCoreBuf) nin = 0;  // beyond the buffer: evaluated per point
        }
        const unsigned fm = __ballot_sync(kFull, cls == 1);
        const unsigned xm = (FAR && LM) ? __ballot_sync(kFull, cls == 3) : 0u;  // staged far lines
        const unsigned em = FAR ? __ballot_sync(kFull, cls == 4) : 0u;
        const unsigned mm = FAR ? __ballot_sync(kFull, cls == 5) : 0u;
        __syncwarp();
        if (cls == 1) {
            const int pos = __popc(fm & lt);
            T.fu[pos] = make_float4(uh, ul, a0.x, a0.y);
            if (LM) T.fg[pos] = a2.x;
        } else if (FAR && LM && cls == 3) {
            const int pos = __popc(xm & lt);
            T.ff[pos] = make_float4(uh, ul, a0.x, a0.y);
            if (LM) T.ffg[pos] = a2.x;
        } else if (FAR && cls == 4) {
            const int pos = __popc(em & lt);
            T.eu[pos] = make_float4(uh, ul, a0.x, a0.y);
            T.ep[pos] = make_float4(a0.z, a0.w, a2.x, 0.f);
        } else if (FAR && cls == 5) {
            const int pos = 31 - __popc(mm & lt);
            T.su[pos] = make_float4(uh, ul, a0.x, a0.y);
            T.sp[pos] = make_float4(a0.z, a0.w, a1.z, a1.w);
            T.sq[pos] = make_float4(a1.y, a2.x, a2.y, a1.x);
        } else if (cls == 2) {
            const int pos = __popc(sm & lt);
            T.su[pos] = make_float4(uh, ul, a0.x, a0.y);
            T.sp[pos] = make_float4(a0.z, a0.w, a1.x, a1.y);
            T.sq[pos] = make_float4(a1.z, a1.w, a2.x, a2.y);
            if (METHOD == 3) T.sr[pos] = make_int4(plo, plo + nin - 1, coff, 0);
        }
        float A = 0.f, B = 0.f, Cc = 0.f;
        if (FAR) {
            PA += pa;
            kahan_add(PB, PBc, pb);
            kahan_add(PC, PCc, pc);
        } else {
            A = warp_sum(pa);
            B = warp_sum(pb);
            Cc = warp_sum(pc);
        }
        __syncwarp();
        const int nf = __popc(fm), ns = __popc(sm), ne = FAR ? __popc(em) : 0, nm = FAR ? __popc(mm) : 0;
        if (FAR) {
            const int nx = __popc(xm);
            if (lane == 0)
                work += (unsigned long long)(nf + ns + ne + nm) * kMxWarpPts + (unsigned long long)nx * kFarNodes;
            if (LM) {  // staged far lines: lane l takes node l % 8 of every fourth one
                float ft = 0.f, fd = 0.f;
                for (int k = lane >> 3; k < nx; k += 4) {
                    const float4 f = T.ff[k];
                    const float d = (xn - f.x) - f.y;
                    const float r = rcp_fast(fmaf(d, d, f.z));
                    ft = fmaf(f.w, r, ft);
                    fd = fmaf(T.ffg[k] * d, r, fd);
                }
                kahan_add(farS, farC, ft);
                kahan_add(farDS, farDC, fd);
            }
        } else if (lane == 0) {
            work += (unsigned long long)(nf + ns) * kMxWarpPts;
        }
        if (FAR && nf + ns + ne + nm == 0) continue;  // warp-uniform: nothing per point in this tile
        if (METHOD == 3 && cfit > 0) {  // the inner points, one per lane: the slow line owning
                                        // element e is the last one whose offset is <= e
            for (int e = lane; e < cfit; e += 32) {
                int lo = 0, hi = ns - 1;
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (T.sr[mid].z <= e) lo = mid;
                    else hi = mid - 1;
                }
                const int4 r = T.sr[lo];
                const float4 u = T.su[lo], w = T.sq[lo];
                const float d = ((float)(r.x + (e - r.z)) - u.x) - u.y;  // as in the per-point loop
                T.cw[e] = faddeeva32_inline(d * w.x, w.y);
            }
            __syncwarp();
        }
        float2 acc2[kMxQ / 2];
        float tdsp[kMxQ];
#pragma unroll
        for (int h = 0; h < kMxQ / 2; ++h) acc2[h] = make_float2(0.f, 0.f);
#pragma unroll
        for (int q = 0; q < kMxQ; ++q) tdsp[q] = 0.f;
        for (int k = 0; k < nf; ++k) {
            const float4 f = T.fu[k];
            const float d0 = (pl0 - f.x) - f.y;
            const float2 d0s = make_float2(d0, d0), b2 = make_float2(f.z, f.z), a = make_float2(f.w, f.w);
#pragma unroll
            for (int h = 0; h < kMxQ / 2; ++h) fast_pair(d0s, offs[h], b2, a, acc2[h]);
            if (LM) {
                const float g = T.fg[k];
#pragma unroll
                for (int q = 0; q < kMxQ; ++q) {
                    const float d = d0 + 32.f * q;
                    tdsp[q] = fmaf(g * d, rcp_fast(fmaf(d, d, f.z)), tdsp[q]);
                }
            }
        }
        // cutoff-edge lines: the far-wing value and the pedestal at every point, masked
        // to the points inside the cutoff (packed, branch-free)
        for (int k = 0; k < ne; ++k) {
            const float4 f = T.eu[k], e = T.ep[k];
            const float d0 = (pl0 - f.x) - f.y;
            const float2 d0s = make_float2(d0, d0), b2 = make_float2(f.z, f.z), a = make_float2(f.w, f.w);
            const float2 c1 = make_float2(e.x, e.x), c0 = make_float2(e.y, e.y);
#pragma unroll
            for (int h = 0; h < kMxQ / 2; ++h) {
                const float2 dsw = __fadd2_rn(d0s, offs[h]);            // (d[q+1], d[q])
                const float2 es = __ffma2_rn(dsw, dsw, b2);             // (e[q+1], e[q])
                const float R = rcp_fast(es.x * es.y);
                const float2 r = __fmul2_rn(es, make_float2(R, R));     // (1/e[q], 1/e[q+1])
                const float2 dn = make_float2(dsw.y, dsw.x);
                const float2 dn2 = __fmul2_rn(dn, dn);
                const float2 v = __ffma2_rn(a, r, __ffma2_rn(c1, dn2, c0));
                acc2[h].x += dn2.x <= cut2 ? v.x : 0.f;
                acc2[h].y += dn2.y <= cut2 ? v.y : 0.f;
                if (LM) {
                    tdsp[2 * h] += dn2.x <= cut2 ? e.z * dn.x * r.x : 0.f;
                    tdsp[2 * h + 1] += dn2.y <= cut2 ? e.z * dn.y * r.y : 0.f;
                }
            }
        }
        float tacc[kMxQ];
#pragma unroll
        for (int h = 0; h < kMxQ / 2; ++h) {
            tacc[2 * h] = acc2[h].x;
            tacc[2 * h + 1] = acc2[h].y;
        }
        // mid lines: the far wing where |x| > x_far, else the continued fraction; the
        // warp takes the continued fraction only for the 32-point rows that need it
        for (int k = 0; k < nm; ++k) {
            const float4 u = T.su[31 - k], pm = T.sp[31 - k], qm = T.sq[31 - k];
            const float y2 = pm.w * pm.w;
#pragma unroll
            for (int q = 0; q < kMxQ; ++q) {
                const float d = ((pl0 + 32.f * q) - u.x) - u.y;
                const float d2 = d * d;
                const float ped = fmaf(pm.x, d2, pm.y);
                const float r = rcp_fast(d2 + u.z);
                float v = fmaf(u.w, r, ped), vd = qm.y * d * r;
                const bool core = d2 <= qm.w;
                if (__any_sync(kFull, core)) {
                    const float2 w = faddeeva_cf2(d * pm.z, pm.w, y2);
                    if (core) {
                        v = fmaf(qm.x, w.x, ped);
                        vd = qm.z * w.y;
                    }
                }
                tacc[q] += v;
                if (LM) tdsp[q] += vd;
            }
        }
        for (int k = 0; k < ns; ++k) {
            const float4 u = T.su[k];
            const float4 p = T.sp[k];
            const float4 w = T.sq[k];
            int rlo = 1, rhi = 0, rb = 0;  // inner points held in cw: [rlo, rhi] at rb + point
            if (METHOD == 3) {
                const int4 r = T.sr[k];
                rlo = r.x;
                rhi = r.y;
                rb = r.z - r.x;
            }
            if (METHOD == 3) {
                // every row: the far wing; rows holding a core point (warp-uniform): the
                // two-level continued fraction (one reciprocal) at every lane, the inner
                // points from cw, and an inner point beyond cw through faddeeva32
                const float y2 = w.y * w.y;
#pragma unroll
                for (int q = 0; q < kMxQ; ++q) {
                    const float d = ((pl0 + 32.f * q) - u.x) - u.y;
                    const float d2 = d * d;
                    const float ped = fmaf(p.x, d2, p.y);
                    const float r = rcp_fast(d2 + u.z);
                    float v = fmaf(u.w, r, ped), vd = w.z * d * r;
                    const bool core = d2 <= p.z;  // |x| <= x_far
                    if (__any_sync(kFull, core)) {
                        const float x = d * w.x;
                        const int pt = lane + 32 * q;
                        float2 fw = faddeeva_cf2(x, w.y, y2);
                        if (pt >= rlo && pt <= rhi) fw = T.cw[rb + pt];
                        else if (core && fabsf(x) + w.y < 15.f) fw = faddeeva32(x, w.y);
                        if (core) {
                            v = fmaf(p.w, fw.x, ped);
                            vd = w.w * fw.y;
                        }
                    }
                    if (d2 > cut2) v = vd = 0.f;
                    tacc[q] += v;
                    if (LM) tdsp[q] += vd;
                }
                continue;
            }
#pragma unroll
            for (int q = 0; q < kMxQ; ++q) {
                const float d = ((pl0 + 32.f * q) - u.x) - u.y;
                const float d2 = d * d;
                if (d2 > cut2) continue;
                const float ped = fmaf(p.x, d2, p.y);
                float v, vd;
                if (d2 <= p.z) {  // |x| <= x_far: Faddeeva core (Weideman-24)
                    v = fmaf(p.w, weideman24_32(d * w.x, w.y), ped);
                    vd = 0.f;
                } else {
                    const float r = rcp_fast(d2 + u.z);
                    v = fmaf(u.w, r, ped);
                    vd = w.z * d * r;
                }
                tacc[q] += v;
                if (LM) tdsp[q] += vd;
            }
        }
#pragma unroll
        for (int q = 0; q < kMxQ; ++q) {
            const float pp = pl0 + 32.f * q;
            kahan_add(sum[q], comp[q], FAR ? tacc[q] : tacc[q] + fmaf(pp, fmaf(pp, A, -2.f * B), Cc));
            if (LM) kahan_add(sumD[q], compD[q], tdsp[q]);
        }
    }
    if (FAR) {  // node totals, then the interpolant at this lane's points
        if (LM) {  // 4 lanes per node
            farS += __shfl_xor_sync(kFull, farS, 8);
            farS += __shfl_xor_sync(kFull, farS, 16);
            farDS += __shfl_xor_sync(kFull, farDS, 8);
            farDS += __shfl_xor_sync(kFull, farDS, 16);
        }
        float Fn[kFarNodes], Dn[kFarNodes];
#pragma unroll
        for (int k = 0; k < kFarNodes; ++k) {
            Fn[k] = LM ? __shfl_sync(kFull, farS, k)
                       : warp_sum((k & 1) ? fnode[k / 2].y : fnode[k / 2].x) + __shfl_sync(kFull, gnode, k);
            Dn[k] = LM ? __shfl_sync(kFull, farDS, k) : 0.f;
        }
        const float A = warp_sum(PA - PAc), B = warp_sum(PB - PBc), Cc = warp_sum(PC - PCc);
#pragma unroll
        for (int q = 0; q < kMxQ; ++q) {
            const float pp = pl0 + 32.f * q;
            float v = fmaf(pp, fmaf(pp, A, -2.f * B), Cc), vd = 0.f;
#pragma unroll
            for (int k = 0; k < kFarNodes; ++k) {
                const float w = FT.L[k][32 * q + lane];
                v = fmaf(Fn[k], w, v);
                if (LM) vd = fmaf(Dn[k], w, vd);
            }
            kahan_add(sum[q], comp[q], v);
            if (LM) kahan_add(sumD[q], compD[q], vd);
        }
    }
    // relmat line mixing: this species' clamped sum goes to its own row, and
    // relmat_finish_kernel adds max(sum + d_sigma, 0) once the perturbation is known
    const bool rel = prow && (sg.flags & SEG_RELMAT);
#pragma unroll
    for (int q = 0; q < kMxQ; ++q) {
        float sig = fmaxf(sum[q], 0.f);
        if (LM) sig = fmaxf(sig + sumD[q], 0.f);
        if (rel) prow[wb + 32 * q + lane] = (double)sig;
        else out_add(orow, q, lane, sig);
    }
    if (!rel) orow.wrote = true;
}

// PseudoVoigt (voigt.jl:281-313): no far-wing shortcut; p0 = (gV2, aPV, c1, c0),
// p1 = (kPV, gPV, -, -): value = aPV/(d^2 + gV2) + gPV 2^(-kPV d^2) + c1 d^2 + c0.
__device__ __forceinline__ void warp_segment_pv(const SegDev& sg, long long cnt, const LpOutMixed& lp, long long wb,
                                                float cut, float cut2, int lane, WarpTile& T, OutRow& orow) {
    constexpr float kCentre = 0.5f * (kMxWarpPts - 1);
    constexpr float kHalf = 0.5f * kMxWarpPts + 0.5f;
    long long jlo, jhi;
    warp_window(lp, sg, cnt, wb, cut, lane, jlo, jhi);
    const float pl0 = (float)lane;
    float sum[kMxQ], comp[kMxQ];
#pragma unroll
    for (int q = 0; q < kMxQ; ++q) sum[q] = comp[q] = 0.f;
    for (long long t0 = jlo; t0 < jhi; t0 += 32) {
        const int nt = (int)min(32LL, jhi - t0);
        __syncwarp();
        if (lane < nt) {
            const long long q = sg.off + t0 + lane;
            const float2 uf = lp.U[q];
            const float uh = uf.x - (float)wb;  // exact: see split_hi_lo
            const float dist = fabsf(uh - kCentre);
            const float cls = dist > cut + kHalf ? 0.f : (dist + kHalf <= cut ? 1.f : 2.f);
            T.fu[lane] = make_float4(uh, uf.y, 0.f, cls);
            T.su[lane] = lp.p0[q];
            T.sp[lane] = lp.p1[q];
        }
        __syncwarp();
        float tacc[kMxQ];
#pragma unroll
        for (int q = 0; q < kMxQ; ++q) tacc[q] = 0.f;
        for (int k = 0; k < nt; ++k) {
            const float4 u = T.fu[k];
            if (u.w == 0.f) continue;
            const float4 a0 = T.su[k];
            const float4 a1 = T.sp[k];
#pragma unroll
            for (int q = 0; q < kMxQ; ++q) {
                const float d = ((pl0 + 32.f * q) - u.x) - u.y;
                const float d2 = d * d;
                if (u.w == 2.f && d2 > cut2) continue;
                tacc[q] += fmaf(a0.y, rcp_fast(d2 + a0.x), fmaf(a1.y, exp2f(-a1.x * d2), fmaf(a0.z, d2, a0.w)));
            }
        }
#pragma unroll
        for (int q = 0; q < kMxQ; ++q) kahan_add(sum[q], comp[q], tacc[q]);
    }
#pragma unroll
    for (int q = 0; q < kMxQ; ++q) out_add(orow, q, lane, fmaxf(sum[q], 0.f));
    orow.wrote = true;
}

// PERT: segments flagged SEG_RELMAT write their clamped sums to the rows
// pert[(profile, layer)][pstride] instead of the optical depth, for
// relmat_finish_kernel (a separate instantiation, so the kernels without it are
// unchanged).
// dynamic shared memory of linesum_mixed_kernel: the warps' tiles, then the far table
constexpr size_t kMxSmem = sizeof(WarpTile) * kMxWarps + sizeof(FarTable);

template <int METHOD, bool ANY_LM, bool FAR, bool PERT = false>
__global__ void __launch_bounds__(kMxThreads, ANY_LM ? 1 : 2) linesum_mixed_kernel(
    const SegDev* __restrict__ segs, const int* __restrict__ seg_count, const int2* __restrict__ pl_segs,
    LpOutMixed lp, long long n_nu, float cut_g, float* __restrict__ tau, unsigned long long* __restrict__ evald,
    double* __restrict__ pert, long long pstride, const float* __restrict__ sfar, const int4* __restrict__ sranges,
    int n_strips, int pl0, int seg0) {
    extern __shared__ __align__(16) unsigned char mx_smem[];
    WarpTile* tiles = reinterpret_cast<WarpTile*>(mx_smem);
    FarTable& ftab = *reinterpret_cast<FarTable*>(mx_smem + sizeof(WarpTile) * kMxWarps);
    if (FAR) {
        far_table_init(ftab);
        __syncthreads();
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int pl = pl0 + (int)blockIdx.y;  // the launch's profile-layers start at pl0, its strip cells at seg0
    const long long wb = (long long)blockIdx.x * kMxStrip + (long long)warp * kMxWarpPts;
    if (wb >= n_nu) return;  // no block-wide barriers below: whole warps may leave
    const float xn = FAR ? (float)far_node(lane & (kFarNodes - 1)) : 0.f;
    unsigned long long work = 0;
    const float cut2 = cut_g * cut_g;
    WarpTile& T = tiles[warp];
    OutRow orow{tau + (size_t)pl * n_nu + wb, (int)min((long long)kMxWarpPts, n_nu - wb), false};
    const int2 rng = pl_segs[pl];
    for (int s = rng.x; s < rng.x + rng.y; ++s) {
        const SegDev sg = segs[s];
        const long long cnt = seg_count[s];
        if (METHOD == 2)
            warp_segment_pv(sg, cnt, lp, wb, cut_g, cut2, lane, T, orow);
        else if (ANY_LM && (sg.flags & 2))
            warp_segment<METHOD, true, FAR>(sg, cnt, lp, wb, cut_g, cut2, lane, T, ftab, xn, orow, work, nullptr,
                                            make_int4(0, 0, 0, 0), 0.f);
        else {
            int4 sx = make_int4(0, 0, 0, 0);  // no strip far field: the whole window
            float gn = 0.f;
            if (FAR && sfar) {
                const size_t cell = (size_t)(s - seg0) * n_strips + blockIdx.x;
                sx = sranges[cell];
                gn = sfar[cell * kStripWords + warp * kFarNodes + (lane & (kFarNodes - 1))];
            }
            warp_segment<METHOD, false, FAR>(sg, cnt, lp, wb, cut_g, cut2, lane, T, ftab, xn, orow, work,
                                             PERT ? pert + (size_t)pl * pstride : nullptr, sx, gn);
        }
    }
    if (evald && lane == 0 && work) atomicAdd(evald, work);
    if (!orow.wrote) {  // no segment stored: zero optical depth
#pragma unroll
        for (int q = 0; q < kMxQ; ++q) out_add(orow, q, lane, 0.f);
    }
}

}  // namespace irs
