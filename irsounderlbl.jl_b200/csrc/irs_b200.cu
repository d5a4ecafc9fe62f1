// irs_b200.cu -- libirs_b200: context, uploads, stage orchestration and the C ABI
// declared in include/irs_b200.h.  One translation unit holds every kernel so the
// Faddeeva constants live in a single __constant__ block.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <numeric>
#include <vector>

#include "faddeeva.cuh"
#include "irs_internal.h"
#include "lineparams.cuh"
#include "linesum.cuh"
#include "rte_ils.cuh"
#include "jacobian.cuh"
#include "oe.cuh"
#include "lm_pert.cuh"
#include "operators.cuh"
#include <atomic>
#include <chrono>
#include <exception>
#include <mutex>
#include <thread>

namespace irs {
const char* last_error();

void* workspace(irs_ctx* ctx, const std::string& name, size_t bytes) {
    DevBuf& b = ctx->work[name];
    if (b.bytes >= bytes && b.p) return b.p;
    if (b.p) IRS_CUDA(cudaFree(b.p));
    b.p = nullptr;
    b.bytes = 0;
    const size_t want = std::max<size_t>(bytes, 256);
    if (cudaMalloc(&b.p, want) != cudaSuccess) {
        cudaGetLastError();
        throw Error{IRS_E_NOMEM, "device allocation of " + std::to_string(want) + " bytes failed (" + name + ")"};
    }
    b.bytes = want;
    return b.p;
}

template <typename T>
static T* upload(irs_ctx* ctx, const std::string& name, const std::vector<T>& v) {
    T* d = (T*)workspace(ctx, name, std::max<size_t>(v.size(), 1) * sizeof(T));
    if (!v.empty()) IRS_CUDA(cudaMemcpyAsync(d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, ctx->stream));
    ctx->n_h2d += (double)(v.size() * sizeof(T));
    return d;
}

void upload_tables(irs_ctx* ctx) {
    if (ctx->tips_dirty) {
        const auto& tp = ctx->tables.tips;
        int stride = 2;
        for (auto& e : tp) stride = std::max<int>(stride, (int)e.second.second.size());
        std::vector<double> q((size_t)std::max<size_t>(tp.size(), 1) * stride, 0.0);
        std::vector<int> tmin(std::max<size_t>(tp.size(), 1), 0), n(std::max<size_t>(tp.size(), 1), 0);
        ctx->tips_index.clear();
        int idx = 0;
        for (auto& e : tp) {
            ctx->tips_index[e.first] = idx;
            tmin[idx] = e.second.first;
            n[idx] = (int)e.second.second.size();
            std::copy(e.second.second.begin(), e.second.second.end(), q.begin() + (size_t)idx * stride);
            ++idx;
        }
        ctx->n_tips = idx;
        ctx->d_tips = upload(ctx, "tips_q", q);
        ctx->d_tips_tmin = upload(ctx, "tips_tmin", tmin);
        ctx->d_tips_n = upload(ctx, "tips_n", n);
        ctx->tips_stride = stride;
        ctx->tips_dirty = false;
    }
    if (ctx->cont_dirty) {
        const Tables& t = ctx->tables;
        std::vector<double> h;
        h.insert(h.end(), t.h2o_nu.begin(), t.h2o_nu.end());
        h.insert(h.end(), t.h2o_cs.begin(), t.h2o_cs.end());
        h.insert(h.end(), t.h2o_cf.begin(), t.h2o_cf.end());
        h.insert(h.end(), t.h2o_te.begin(), t.h2o_te.end());
        std::vector<double> c;
        c.insert(c.end(), t.co2_nu.begin(), t.co2_nu.end());
        c.insert(c.end(), t.co2_s.begin(), t.co2_s.end());
        c.insert(c.end(), t.co2_tdep.begin(), t.co2_tdep.end());
        ctx->d_h2o = upload(ctx, "ckd_h2o", h);
        ctx->d_co2 = upload(ctx, "ckd_co2", c);
        ctx->n_h2o = (int)t.h2o_nu.size();
        ctx->n_co2 = (int)t.co2_nu.size();
        // CIA blocks of the three tables in order: (T, nu_min, nu_max, first knot, count)
        std::vector<double> blk, knu, ksg;
        for (int q = 0; q < 3; ++q) {
            ctx->cia_b0[q] = (int)(blk.size() / 5);
            for (const Tables::CiaBlock& b : t.cia[q]) {
                blk.insert(blk.end(), {b.T, b.nu.front(), b.nu.back(), (double)knu.size(), (double)b.nu.size()});
                knu.insert(knu.end(), b.nu.begin(), b.nu.end());
                ksg.insert(ksg.end(), b.sg.begin(), b.sg.end());
            }
        }
        ctx->cia_b0[3] = (int)(blk.size() / 5);
        ctx->d_cia_blk = upload(ctx, "cia_blk", blk);
        ctx->d_cia_nu = upload(ctx, "cia_nu", knu);
        ctx->d_cia_sg = upload(ctx, "cia_sg", ksg);
        ctx->cont_dirty = false;
    }
}

// continua of the call: MT-CKD H2O/CO2 and the CIA pairs whose tables are loaded
// (a missing table contributes zeros, continuum.jl:190-194, 268-272)
static ContDev cont_dev(irs_ctx* ctx, const irs_fm_options& o) {
    ContDev cd;
    cd.h2o = ctx->d_h2o; cd.co2 = ctx->d_co2; cd.n_h2o = ctx->n_h2o; cd.n_co2 = ctx->n_co2;
    cd.mask = 0;
    cd.cia.blk = ctx->d_cia_blk; cd.cia.nu = ctx->d_cia_nu; cd.cia.sg = ctx->d_cia_sg;
    for (int q = 0; q < 4; ++q) cd.cia.b0[q] = ctx->cia_b0[q];
    if (o.apply_continuum)
        for (int q = 0; q < 3; ++q)
            if ((o.continua & (4 << q)) && ctx->cia_b0[q + 1] > ctx->cia_b0[q]) cd.mask |= 4 << q;
    return cd;
}

static TipsDev tips_dev(irs_ctx* ctx) {
    TipsDev t;
    t.q = ctx->d_tips;
    t.tmin = ctx->d_tips_tmin;
    t.n = ctx->d_tips_n;
    t.stride = ctx->tips_stride;
    return t;
}

static void check_launch(irs_ctx* ctx) {
    ctx->n_launch += 1;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) throw Error{IRS_E_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e)};
}

static void validate_options(const irs_fm_options& o) {
    IRS_REQUIRE(o.method >= 1 && o.method <= 3, "method must be 1 (Weideman), 2 (PseudoVoigt) or 3 (FullFaddeeva)");
    IRS_REQUIRE(o.precision == IRS_FP64 || o.precision == IRS_MIXED || o.precision == IRS_MIXED_DIRECT,
                "precision must be IRS_FP64, IRS_MIXED or IRS_MIXED_DIRECT");
    IRS_REQUIRE(o.cutoff > 0.0, "cutoff must be positive");
    IRS_REQUIRE(o.apodization >= 0 && o.apodization <= 3, "unknown apodization");
    IRS_REQUIRE(o.T_method == 0 || o.T_method == 1, "T_method must be :logp_at_pcg or :mass_weighted");
    IRS_REQUIRE(o.source_function == 0 || o.source_function == 1, "source_function must be :cim or :toon");
    IRS_REQUIRE(o.line_mixing >= IRS_LM_NONE && o.line_mixing <= IRS_LM_RELMAT_VPW,
                "line_mixing must be 0 (none), 1 (per-line Y), 2 (VPYLineMixing) or 3 (VPWLineMixing)");
    if (o.line_mixing == IRS_LM_PER_LINE_Y)
        IRS_REQUIRE(o.lm_cutoff == o.cutoff, "lm_cutoff must equal cutoff with per-line Y");
    if (o.line_mixing != IRS_LM_NONE) {
        IRS_REQUIRE(o.method == IRS_FULLFADDEEVA, "line mixing evaluates the Voigt part with FullFaddeeva");
        IRS_REQUIRE(o.lm_cutoff > 0.0, "lm_cutoff must be positive");
    }
}

// ------------------------------------------------------- the line-sum pipeline
struct Plan {
    std::vector<Segment> segs;
    std::vector<int2> pl_segs;  // per (profile, layer): first segment, count
    int n_prof = 0, L = 0;
    int64_t slots = 0;
    int64_t max_list = 0;
};

static std::vector<ListDev> list_descs(irs_ctx* ctx) {
    std::vector<ListDev> v;
    for (auto& l : ctx->lists) {
        ListDev d;
        d.nu = l.nu; d.S296 = l.S296; d.E = l.E; d.gair = l.gair; d.gself = l.gself;
        d.nair = l.nair; d.delta = l.delta; d.y0 = l.y0; d.tips = l.tips;
        d.n = l.n; d.mol = l.species; d.has_y0 = l.has_y0 ? 1 : 0;
        v.push_back(d);
    }
    return v;
}

// Runs the line-parameter passes and the line sum for the plan; returns the
// device tau buffer ([n_prof * L][n_nu], FP32 for mixed or FP64 for plain).
static void* run_linesum(irs_ctx* ctx, Plan& pl, const double* d_grid, int64_t n_nu, double grid0,
                         double dnu_g, const irs_fm_options& o, int ev_mid, double* d_pert = nullptr,
                         long long pstride = 0) {
    cudaStream_t st = ctx->stream;
    const int nseg = (int)pl.segs.size();
    std::vector<SegDev> sd(std::max(nseg, 1));
    int64_t off = 0;
    for (int s = 0; s < nseg; ++s) {
        Segment& g = pl.segs[s];
        g.out_off = off;
        off += ctx->lists[g.list].n;
        SegDev& d = sd[s];
        d.T = g.T; d.p_atm = g.p_atm; d.vs = g.vmr_self; d.coef = g.coef; d.margin_g = g.margin_g;
        d.off = g.out_off; d.list = g.list; d.flags = g.flags;
        pl.max_list = std::max<int64_t>(pl.max_list, ctx->lists[g.list].n);
    }
    pl.slots = off;
    SegDev* d_segs = upload(ctx, "segs", sd);
    std::vector<ListDev> ld = list_descs(ctx);
    ListDev* d_lists = upload(ctx, "list_descs", ld);
    int2* d_pl = upload(ctx, "pl_segs", pl.pl_segs);
    int* d_count = (int*)workspace(ctx, "seg_count", sizeof(int) * std::max(nseg, 1));
    IRS_CUDA(cudaMemsetAsync(d_count, 0, sizeof(int) * std::max(nseg, 1), st));
    unsigned long long* d_pairs = (unsigned long long*)workspace(ctx, "pair_counts", 24);
    IRS_CUDA(cudaMemsetAsync(d_pairs, 0, 24, st));

    const int mixed = o.precision != IRS_FP64;
    const size_t tau_elem = mixed ? sizeof(float) : sizeof(double);
    void* d_tau = workspace(ctx, "tau", (size_t)pl.n_prof * pl.L * n_nu * tau_elem);
    IRS_CUDA(cudaMemsetAsync(d_tau, 0, (size_t)pl.n_prof * pl.L * n_nu * tau_elem, st));
    if (nseg == 0 || pl.slots == 0) {
        IRS_CUDA(cudaEventRecord(ctx->ev[ev_mid], st));
        return d_tau;
    }
    const int n_chunks = (int)((pl.max_list + kLpChunk - 1) / kLpChunk);
    unsigned char* d_keep = (unsigned char*)workspace(ctx, "keep", (size_t)pl.slots);
    int* d_chunk = (int*)workspace(ctx, "chunk_count", sizeof(int) * (size_t)nseg * n_chunks);
    LpConfig cfg;
    cfg.cutoff = o.cutoff; cfg.x_far = o.x_far; cfg.dptmn = o.dptmn;
    cfg.grid0 = grid0; cfg.dnu_g = dnu_g; cfg.method = o.method; cfg.n_nu = n_nu;
    {  // shifted centres within the grid plus its cutoff margins: |U| < 2^24 u_gran
        const double reach = (double)n_nu + 2.0 * o.cutoff / dnu_g + 64.0;
        cfg.u_gran = 1.0 / 16.0;
        while (reach >= 16777216.0 * cfg.u_gran) cfg.u_gran *= 2.0;
    }
    const TipsDev tp = tips_dev(ctx);
    dim3 g1(n_chunks, nseg);
    lp_keep_kernel<<<g1, kLpThreads, 0, st>>>(d_segs, d_lists, tp, cfg, d_keep, d_chunk, n_chunks);
    check_launch(ctx);
    LpOutF64 o64{};
    LpOutMixed om{};
    const size_t S = (size_t)pl.slots;
    if (!mixed) {
        double* base = (double*)workspace(ctx, "lp64", S * 6 * sizeof(double));
        o64.nu0 = base; o64.f = base + S; o64.y = base + 2 * S; o64.Sn = base + 3 * S;
        o64.Hc = base + 4 * S; o64.YSn = base + 5 * S;
        lp_write_kernel<0><<<g1, kLpThreads, 0, st>>>(d_segs, d_lists, tp, cfg, d_keep, d_chunk, n_chunks,
                                                      d_count, o64, om, d_pairs, nullptr);
    }
    unsigned* d_reach = nullptr;  // per segment: the largest Faddeeva-core half-width, grid units
    if (mixed) {
        char* base = (char*)workspace(ctx, "lpmx", S * (8 + 8 + 16 + 16 + 16));
        om.V = (double*)base;
        om.U = (float2*)(base + S * 8);
        om.p0 = (float4*)(base + S * 16);
        om.p1 = (float4*)(base + S * 32);
        om.p2 = (float4*)(base + S * 48);
        d_reach = (unsigned*)workspace(ctx, "core_reach", sizeof(unsigned) * std::max(nseg, 1));
        IRS_CUDA(cudaMemsetAsync(d_reach, 0, sizeof(unsigned) * std::max(nseg, 1), st));
        lp_write_kernel<1><<<g1, kLpThreads, 0, st>>>(d_segs, d_lists, tp, cfg, d_keep, d_chunk, n_chunks,
                                                      d_count, o64, om, d_pairs, d_reach);
    }
    check_launch(ctx);
    IRS_CUDA(cudaEventRecord(ctx->ev[ev_mid], st));
    const int npl = pl.n_prof * pl.L;
    if (!mixed) {
        dim3 g2((unsigned)((n_nu + 255) / 256), npl);
        if (o.method == 1)
            linesum_f64_kernel<1><<<g2, 256, 0, st>>>(d_segs, d_count, d_pl, o64, d_grid, n_nu, o.cutoff, o.x_far, (double*)d_tau, d_pert, pstride);
        else if (o.method == 2)
            linesum_f64_kernel<2><<<g2, 256, 0, st>>>(d_segs, d_count, d_pl, o64, d_grid, n_nu, o.cutoff, o.x_far, (double*)d_tau, d_pert, pstride);
        else
            linesum_f64_kernel<3><<<g2, 256, 0, st>>>(d_segs, d_count, d_pl, o64, d_grid, n_nu, o.cutoff, o.x_far, (double*)d_tau, d_pert, pstride);
    } else {
        dim3 g2((unsigned)((n_nu + kMxStrip - 1) / kMxStrip), npl);
        const float cut_g = (float)(o.cutoff / dnu_g);
        unsigned long long* d_eval = d_pairs + 2;
        const bool far = o.precision == IRS_MIXED;
        const bool anylm = o.line_mixing == IRS_LM_PER_LINE_Y;
        // strip far field (pre-pass): 528 bytes per (segment, strip) in a buffer of at most
        // ctx->strip_buf_max; larger batches run in groups of profile-layers (their segments
        // are contiguous) whose cells fit it
        const int n_strips = (int)g2.x;
        const size_t cell_bytes = kStripWords * sizeof(float) + sizeof(int4);
        const bool strip = far && o.method == 3;
        float* d_M = nullptr;
        char* d_sbuf = nullptr;
        size_t max_cells = 0;
        if (strip) {
            max_cells = std::min((size_t)nseg * n_strips, ctx->strip_buf_max / cell_bytes);
            d_sbuf = (char*)workspace(ctx, "strip_far", max_cells * cell_bytes);
            constexpr int nM = kMxWarps * kFarNodes * kCtaNodes;
            d_M = (float*)workspace(ctx, "strip_M", nM * sizeof(float));
            strip_table_kernel<<<(nM + 255) / 256, 256, 0, st>>>(d_M);
            check_launch(ctx);
        }
        std::vector<int> first(npl + 1, 0);  // first segment of each profile-layer (emitted in order)
        for (int q = 0; q < npl; ++q) first[q + 1] = first[q] + pl.pl_segs[q].y;
        for (int pa = 0; pa < npl;) {
            // this launch: profile-layers [pa, pb) and their segments [s_a, first[pb])
            int pb = npl;
            const int s_a = first[pa];
            float* d_sfar = nullptr;
            int4* d_srng = nullptr;
            if (strip) {
                pb = pa;
                while (pb < npl && (size_t)(first[pb + 1] - s_a) * n_strips <= max_cells) ++pb;
                if (pb == pa) pb = pa + 1;  // one profile-layer beyond the buffer: no strip far field
                const size_t cells = (size_t)(first[pb] - s_a) * n_strips;
                if (cells <= max_cells) {
                    d_sfar = (float*)d_sbuf;
                    d_srng = (int4*)(d_sbuf + cells * kStripWords * sizeof(float));
                    dim3 g3(n_strips, pb - pa);
                    if (anylm) strip_far_kernel<true><<<g3, kStripThreads, 0, st>>>(d_segs, d_count, d_reach, d_pl, om, cut_g, n_strips, d_M, d_sfar, d_srng, d_eval, pa, s_a);
                    else strip_far_kernel<false><<<g3, kStripThreads, 0, st>>>(d_segs, d_count, d_reach, d_pl, om, cut_g, n_strips, d_M, d_sfar, d_srng, d_eval, pa, s_a);
                    check_launch(ctx);
                }
            }
            const dim3 g2c(g2.x, pb - pa);
#define IRS_MX(M, LMX, F, P) do { \
        IRS_CUDA(cudaFuncSetAttribute(linesum_mixed_kernel<M, LMX, F, P>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMxSmem)); \
        linesum_mixed_kernel<M, LMX, F, P><<<g2c, kMxThreads, kMxSmem, st>>>(d_segs, d_count, d_pl, om, n_nu, cut_g, (float*)d_tau, d_eval, d_pert, pstride, d_sfar, d_srng, n_strips, pa, s_a); \
    } while (0)
            if (o.method == 1) { if (far) IRS_MX(1, false, true, false); else IRS_MX(1, false, false, false); }
            else if (o.method == 2) IRS_MX(2, false, false, false);
            else if (o.line_mixing == IRS_LM_PER_LINE_Y) { if (far) IRS_MX(3, true, true, false); else IRS_MX(3, true, false, false); }
            else if (d_pert) { if (far) IRS_MX(3, false, true, true); else IRS_MX(3, false, false, true); }
            else { if (far) IRS_MX(3, false, true, false); else IRS_MX(3, false, false, false); }
            check_launch(ctx);
            pa = pb;
        }
#undef IRS_MX
    }
    check_launch(ctx);
    return d_tau;
}

__global__ void ils_float_kernel(const double* __restrict__ k, long long n, float* __restrict__ kf) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) kf[i] = (float)k[i];
}

static void ensure_ils(irs_ctx* ctx, double dnu, double opd, double fwhm, int apod) {
    const double key[4] = {dnu, opd, fwhm, (double)apod};
    if (std::memcmp(key, ctx->ils_key, sizeof key) == 0) return;
    const int64_t n_half = (int64_t)std::ceil(16.0 / dnu);
    const int64_t n = 2 * n_half + 1;
    double* k = (double*)workspace(ctx, "ils", n * sizeof(double));
    ils_taps_kernel<<<(unsigned)((n + 127) / 128), 128, 0, ctx->stream>>>(dnu, opd, fwhm, apod, n_half, k);
    check_launch(ctx);
    ils_normalise_kernel<<<1, 1024, 0, ctx->stream>>>(k, n, dnu);
    check_launch(ctx);
    // the same taps rounded to FP32 for the Jacobian's channel contraction (FP32 sums)
    float* kf = (float*)workspace(ctx, "ils_f", n * sizeof(float));
    ils_float_kernel<<<(unsigned)((n + 255) / 256), 256, 0, ctx->stream>>>(k, n, kf);
    check_launch(ctx);
    std::memcpy(ctx->ils_key, key, sizeof key);
    ctx->ils_n = n;
}

// Runs f(0..n-1) on the host's cores.
template <class F>
static void parallel_for(int n, F&& f) {
    const int nt = std::max(1, std::min<int>(n, (int)std::thread::hardware_concurrency()));
    if (nt <= 1) {
        for (int i = 0; i < n; ++i) f(i);
        return;
    }
    std::atomic<int> next(0);
    std::exception_ptr err;
    std::mutex mu;
    std::vector<std::thread> th;
    for (int t = 0; t < nt; ++t)
        th.emplace_back([&] {
            for (int i; (i = next++) < n;) {
                try {
                    f(i);
                } catch (...) {
                    std::lock_guard<std::mutex> g(mu);
                    if (!err) err = std::current_exception();
                }
            }
        });
    for (auto& t : th) t.join();
    if (err) std::rethrow_exception(err);
}

// Relaxation-matrix line mixing (line_mixing = 2, 3): the poles of the LM species'
// perturbation for every (profile, layer) where it is present, at that layer's
// Curtis-Godson T and p of the species (sounder.jl:283-305), built on the host cores.
// With jac, three pole sets per (profile, layer), amplitudes times the column amount:
// the perturbation and its central differences in T (h = 0.02 K) and p (h = 1e-4 p),
// the pairs of evaluations folded into one set with amplitudes +-1/(2h)
// (cross_section_jacobian.jl:252-319).
struct RelmatPlan {
    std::vector<LmPole> poles;
    std::vector<long long> off;  // per row (profile, layer[, variant]): poles[off[k], off[k+1])
    std::vector<int> seg_of;     // per (profile, layer): the LM species' segment, or -1
    uint32_t iso_mask = 0;
};
static_assert(sizeof(LmPole) == sizeof(LmPoleDev), "pole layouts differ");
constexpr long long kPertAlign = 8192;  // rows padded to whole line-sum strips of either kernel
static_assert(kPertAlign % kMxStrip == 0 && kPertAlign % kJgStrip == 0, "perturbation row padding");

// Flags the LM species' segments SEG_RELMAT; false when relmat line mixing is off.
static bool relmat_prepare(irs_ctx* ctx, Plan& pl, const irs_fm_options& o, RelmatPlan& rp) {
    if (o.line_mixing != IRS_LM_RELMAT_VPY && o.line_mixing != IRS_LM_RELMAT_VPW) return false;
    const RelmatHost& R = ctx->relmat;
    IRS_REQUIRE(R.species != 0, "line_mixing 2 and 3 need the relaxation-matrix data (irs_upload_relmat)");
    int li = -1;
    for (size_t i = 0; i < ctx->lists.size(); ++i)
        if (ctx->lists[i].species == R.species && ctx->lists[i].n > 0) li = (int)i;
    if (li < 0) return false;  // the LM species has no line list in this call
    rp.iso_mask = ctx->lists[li].iso_mask;
    rp.seg_of.assign((size_t)pl.n_prof * pl.L, -1);
    for (size_t i = 0; i < pl.segs.size(); ++i)
        if (pl.segs[i].list == li) {
            pl.segs[i].flags |= SEG_RELMAT;
            rp.seg_of[pl.segs[i].prof * pl.L + pl.segs[i].layer] = (int)i;
        }
    return true;
}

// The pole lists of every (profile, layer) that has a relmat segment.
static void relmat_build(irs_ctx* ctx, const Plan& pl, const irs_fm_options& o, RelmatPlan& rp, bool jac) {
    const RelmatHost& R = ctx->relmat;
    const uint32_t iso_mask = rp.iso_mask;
    const std::vector<int>& seg_of = rp.seg_of;
    const int npl = pl.n_prof * pl.L;
    const int nv = jac ? 3 : 1;
    std::vector<std::vector<LmPole>> per((size_t)npl * nv);
    parallel_for(npl * nv, [&](int k) {
        const int v = k % nv;
        if (seg_of[k / nv] < 0) return;
        const Segment& g = pl.segs[seg_of[k / nv]];
        const double T = g.T, p = g.p_atm;
        std::vector<LmPole>& out = per[k];
        if (!jac) {  // keep_threshold 1e-4 (line_mixing.jl:1123)
            lm_poles(R, ctx->tables, o.line_mixing, iso_mask, T, p, 1e-4, out);
            return;
        }
        auto add = [&](double Tv, double pv, double scale) {
            std::vector<LmPole> q;
            lm_poles(R, ctx->tables, o.line_mixing, iso_mask, Tv, pv, 1e-4, q);
            for (LmPole& e : q) { e.ar *= scale; e.ai *= scale; }
            out.insert(out.end(), q.begin(), q.end());
        };
        const double hT = 0.02, hp = std::max(p, 1e-6) * 1e-4;
        if (v == 0) add(T, p, g.coef);
        if (v == 1) { add(T + hT, p, g.coef / (2 * hT)); add(T - hT, p, -g.coef / (2 * hT)); }
        if (v == 2) { add(T, p + hp, g.coef / (2 * hp)); add(T, p - hp, -g.coef / (2 * hp)); }
        std::stable_sort(out.begin(), out.end(), [](const LmPole& a, const LmPole& c) { return a.c < c.c; });
    });
    const size_t rows = per.size();
    rp.off.assign(rows + 1, 0);
    for (size_t k = 0; k < rows; ++k) rp.off[k + 1] = rp.off[k] + (long long)per[k].size();
    rp.poles.resize(rp.off[rows]);
    for (size_t k = 0; k < rows; ++k) std::copy(per[k].begin(), per[k].end(), rp.poles.begin() + rp.off[k]);
}

static bool relmat_plan(irs_ctx* ctx, Plan& pl, const irs_fm_options& o, RelmatPlan& rp, bool jac) {
    if (!relmat_prepare(ctx, pl, o, rp)) return false;
    relmat_build(ctx, pl, o, rp, jac);
    return true;
}

// The perturbation rows [row][pstride] on the device grid.
static const double* relmat_launch(irs_ctx* ctx, const RelmatPlan& rp, const double* d_grid, int64_t n_nu,
                                   double cutoff, double x_far, long long& pstride) {
    const int npl = (int)rp.off.size() - 1;
    pstride = ((n_nu + kPertAlign - 1) / kPertAlign) * kPertAlign;
    const LmPoleDev* d_p = (const LmPoleDev*)upload(ctx, "lm_poles", rp.poles);
    const long long* d_off = upload(ctx, "lm_off", rp.off);
    double* d_out = (double*)workspace(ctx, "lm_pert", (size_t)npl * pstride * sizeof(double));
    dim3 g((unsigned)((pstride + 255) / 256), npl);
    lm_pert_kernel<<<g, 256, 0, ctx->stream>>>(d_p, d_off, d_grid, n_nu, pstride, cutoff, x_far, d_out);
    check_launch(ctx);
    return d_out;
}

static void forward_pass(irs_ctx* ctx, const irs_profile* profs, int n_prof, const irs_sounder& s,
                         const irs_fm_options& o, double* d_R, double* d_BT) {
    upload_tables(ctx);
    cudaStream_t st = ctx->stream;
    const InternalGrid ig = internal_grid(s, o);
    const GridSpec ch = make_grid(s.nu_min, s.nu_max, s.dnu);
    const int64_t n_nu = ig.g.n;
    const int L = profs[0].n_lev - 1;
    Plan pl;
    pl.n_prof = n_prof;
    pl.L = L;
    std::vector<int> list_sp;
    std::vector<double> list_shift;
    for (auto& l : ctx->lists) {  // empty lists produce no segments
        list_sp.push_back(l.n > 0 ? l.species : -1);
        list_shift.push_back(l.max_abs_shift);
    }
    std::vector<LayerRT> lrt;
    std::vector<ProfileRT> prt(n_prof);
    for (int p = 0; p < n_prof; ++p) {
        IRS_REQUIRE(profs[p].n_lev == L + 1, "all profiles of a batch must have the same number of levels");
        const size_t before = pl.segs.size();
        layer_setup(profs[p], p, o, list_sp, list_shift, ig.dnu_hi, pl.segs, lrt, prt[p]);
        (void)before;
    }
    // per (profile, layer) segment ranges (segments are emitted in p, layer order)
    pl.pl_segs.assign((size_t)n_prof * L, make_int2(0, 0));
    for (size_t i = 0; i < pl.segs.size(); ++i) {
        const int key = pl.segs[i].prof * L + pl.segs[i].layer;
        if (pl.pl_segs[key].y == 0) pl.pl_segs[key].x = (int)i;
        pl.pl_segs[key].y++;
    }
    {  // size every workspace up front so no (synchronising) reallocation falls inside a timed stage
        int64_t slots = 0, max_list = 0;
        for (auto& g : pl.segs) { slots += ctx->lists[g.list].n; max_list = std::max<int64_t>(max_list, ctx->lists[g.list].n); }
        const bool mixed = o.precision != IRS_FP64;
        const int nseg = std::max<int>((int)pl.segs.size(), 1);
        workspace(ctx, "tau", (size_t)n_prof * L * n_nu * (mixed ? sizeof(float) : sizeof(double)));
        workspace(ctx, "I", (size_t)n_prof * n_nu * sizeof(double));
        workspace(ctx, "grid", n_nu * sizeof(double));
        if (slots > 0) {
            workspace(ctx, mixed ? "lpmx" : "lp64", (size_t)slots * (mixed ? 64 : 48));
            workspace(ctx, "keep", (size_t)slots);
            workspace(ctx, "chunk_count", sizeof(int) * (size_t)nseg * ((max_list + kLpChunk - 1) / kLpChunk));
        }
        workspace(ctx, "seg_count", sizeof(int) * nseg);
        if (o.precision == IRS_MIXED && o.method == 3) {  // the strip far field's buffers
            const size_t n_strips = (size_t)((n_nu + kMxStrip - 1) / kMxStrip);
            const size_t cb = kStripWords * sizeof(float) + sizeof(int4);
            workspace(ctx, "strip_far", std::min((size_t)nseg * n_strips, ctx->strip_buf_max / cb) * cb);
            workspace(ctx, "strip_M", sizeof(float) * kMxWarps * kFarNodes * kCtaNodes);
        }
        if (mixed) workspace(ctx, "core_reach", sizeof(unsigned) * nseg);
        workspace(ctx, "lrt", std::max<size_t>(lrt.size(), 1) * sizeof(LayerRT));
        workspace(ctx, "prt", std::max<size_t>(prt.size(), 1) * sizeof(ProfileRT));
    }
    // relmat line mixing: the LM species' clamped sums go to their own rows while the
    // host builds the poles (overlapping the line sum); the finish kernel then adds
    // max(sum + d_sigma, 0) into the optical depths
    RelmatPlan rp;
    const bool relmat = relmat_prepare(ctx, pl, o, rp);
    ctx->lm_ev = relmat;
    ctx->lm_host_pass = 0;
    const long long pstride = ((n_nu + kPertAlign - 1) / kPertAlign) * kPertAlign;
    std::vector<double> coef_pl;
    if (relmat) {
        coef_pl.assign((size_t)n_prof * L, 0.0);
        for (size_t k = 0; k < rp.seg_of.size(); ++k)
            if (rp.seg_of[k] >= 0) coef_pl[k] = pl.segs[rp.seg_of[k]].coef;
        workspace(ctx, "lm_pert", (size_t)n_prof * L * pstride * sizeof(double));
        workspace(ctx, "lm_sv", (size_t)n_prof * L * pstride * sizeof(double));
        workspace(ctx, "lm_coef", coef_pl.size() * sizeof(double));
        workspace(ctx, "lm_off", ((size_t)n_prof * L + 1) * sizeof(long long));
    }
    IRS_CUDA(cudaEventRecord(ctx->ev[0], st));
    double* d_grid = (double*)workspace(ctx, "grid", n_nu * sizeof(double));
    grid_values_kernel<<<(unsigned)((n_nu + 255) / 256), 256, 0, st>>>(to_dev(ig.g), d_grid);
    check_launch(ctx);
    if (o.with_ils) ensure_ils(ctx, ig.dnu_hi, s.opd_max, s.fwhm_gauss, o.apodization);
    double* d_sv = relmat ? (double*)workspace(ctx, "lm_sv", (size_t)n_prof * L * pstride * sizeof(double)) : nullptr;
    void* d_tau = run_linesum(ctx, pl, d_grid, n_nu, ig.g.at(0), ig.dnu_hi, o, 1, d_sv, pstride);
    if (relmat) {
        const auto h0 = std::chrono::steady_clock::now();
        relmat_build(ctx, pl, o, rp, false);  // host cores, while the GPU runs the line sum
        ctx->lm_host_pass = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - h0).count();
        IRS_CUDA(cudaEventRecord(ctx->ev[7], st));
        long long ps = 0;
        const double* d_pert = relmat_launch(ctx, rp, d_grid, n_nu, o.lm_cutoff, o.x_far, ps);
        const double* d_coef = upload(ctx, "lm_coef", coef_pl);
        dim3 gf((unsigned)((n_nu + 255) / 256), n_prof * L);
        if (o.precision != IRS_FP64)
            relmat_finish_kernel<float><<<gf, 256, 0, st>>>((float*)d_tau, d_sv, d_pert, d_coef, n_nu, pstride);
        else
            relmat_finish_kernel<double><<<gf, 256, 0, st>>>((double*)d_tau, d_sv, d_pert, d_coef, n_nu, pstride);
        check_launch(ctx);
        IRS_CUDA(cudaEventRecord(ctx->ev[8], st));
    }
    IRS_CUDA(cudaEventRecord(ctx->ev[2], st));
    LayerRT* d_lrt = upload(ctx, "lrt", lrt);
    ProfileRT* d_prt = upload(ctx, "prt", prt);
    double* d_I = (double*)workspace(ctx, "I", (size_t)n_prof * n_nu * sizeof(double));
    ContDev cd = cont_dev(ctx, o);
    if (o.apply_continuum) {
        if ((o.continua & 1) && ctx->n_h2o > 1) cd.mask |= 1;
        if ((o.continua & 2) && ctx->n_co2 > 1) cd.mask |= 2;
    }
    dim3 g3((unsigned)((n_nu + 255) / 256), n_prof);
    if (o.precision != IRS_FP64) {
        const size_t sm = (size_t)L * sizeof(RteLayerF);
        IRS_REQUIRE(sm <= 200 * 1024, "too many layers for the RTE kernel (at most 4266)");
        if (cd.mask & kCiaMask) {
            if (sm > 48 * 1024)
                IRS_CUDA(cudaFuncSetAttribute(rte_mixed_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
            rte_mixed_kernel<true><<<g3, 256, sm, st>>>((const float*)d_tau, d_lrt, d_prt, L, d_grid, n_nu, o.source_function, cd, d_I);
        } else {
            if (sm > 48 * 1024)
                IRS_CUDA(cudaFuncSetAttribute(rte_mixed_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
            rte_mixed_kernel<false><<<g3, 256, sm, st>>>((const float*)d_tau, d_lrt, d_prt, L, d_grid, n_nu, o.source_function, cd, d_I);
        }
    } else
        if (cd.mask & kCiaMask)
            rte_kernel<double, true><<<g3, 256, 0, st>>>((const double*)d_tau, d_lrt, d_prt, L, d_grid, n_nu, o.source_function, cd, d_I);
        else
            rte_kernel<double><<<g3, 256, 0, st>>>((const double*)d_tau, d_lrt, d_prt, L, d_grid, n_nu, o.source_function, cd, d_I);
    check_launch(ctx);
    IRS_CUDA(cudaEventRecord(ctx->ev[3], st));
    const double* d_kern = o.with_ils ? (const double*)ctx->work["ils"].p : nullptr;
    dim3 g4((unsigned)((ch.n * 32 + 255) / 256), n_prof);
    ils_bt_kernel<<<g4, 256, 0, st>>>(d_I, n_nu, d_kern, o.with_ils ? ctx->ils_n : 0, ig.dnu_hi, to_dev(ig.g),
                                       to_dev(ch), o.with_ils, d_R, d_BT);
    check_launch(ctx);
    IRS_CUDA(cudaEventRecord(ctx->ev[4], st));
}

// ------------------------------------------------------------ Jacobian
static int profiles_per_pass(irs_ctx* ctx, int n_prof, int L, size_t per_prof);

static int64_t state_size(const irs_state_spec& sp, int n_lev) {
    return (sp.include_temperature ? n_lev : 0) + (int64_t)sp.n_retrieved * n_lev + (sp.include_tsfc ? 1 : 0) +
           (sp.include_emissivity ? 1 : 0);
}

// vmr_jacobian.jl:152-505 for profiles [0, n_prof): K_h [n_prof][n_state][n_ch], y_h [n_prof][n_ch]
// Outputs: host K_h/y_h (double), or with K_dev non-null the device K_dev (float
// [n_prof][n_state][n_ch]) and host y_h.
// With dx_h non-null it computes the pullback dx = K^T dy instead (dy_h [n_prof][n_ch]
// host, dx_h [n_prof][n_state] host): the derivative line sum as above, then I, R and
// BT, the radiance cotangent on the grid by the transposed ILS, and one adjoint RTE sweep
// that contracts each derivative term with it on the device; neither D nor K is formed.
static void jacobian_device(irs_ctx* ctx, const irs_profile* profs, int n_prof, const irs_sounder& s,
                            const irs_fm_options& o_in, const irs_state_spec& sp, double* K_h, double* y_h,
                            float* K_dev = nullptr, const double* dy_h = nullptr, double* dx_h = nullptr) {
    const bool adjoint = dx_h != nullptr;
    IRS_REQUIRE(n_prof >= 1 && profs, "need at least one profile");
    IRS_REQUIRE(sp.n_retrieved >= 0 && sp.n_retrieved <= 4 && (sp.n_retrieved == 0 || sp.retrieved),
                "at most 4 retrieved species");
    IRS_REQUIRE(sp.observable == 0 || sp.observable == 1, "observable must be :bt or :radiance");
    irs_fm_options o = o_in;
    o.dptmn = 0.0;               // frozen line set (vmr_jacobian.jl:188-201)
    o.precision = IRS_MIXED;
    validate_options(o);
    upload_tables(ctx);
    cudaStream_t st = ctx->stream;
    const InternalGrid ig = internal_grid(s, o);
    const GridSpec ch = make_grid(s.nu_min, s.nu_max, s.dnu);
    const int64_t n_nu = ig.g.n, n_ch = ch.n;
    const int L = profs[0].n_lev - 1;
    const int64_t n_state = state_size(sp, L + 1);
    const int n_out = 3 + 2 * sp.n_retrieved;
    for (int r = 0; r < sp.n_retrieved; ++r)
        for (int p = 0; p < n_prof; ++p) {
            bool found = false;
            for (int q = 0; q < profs[p].n_species; ++q) found |= profs[p].species[q] == sp.retrieved[r];
            IRS_REQUIRE(found, "profile is missing a retrieved species");
        }
    std::vector<int> list_sp;
    std::vector<double> list_shift;
    std::vector<bool> has_list(64, false);
    for (auto& l : ctx->lists) {
        list_sp.push_back(l.n > 0 ? l.species : -1);
        list_shift.push_back(l.max_abs_shift);
        if (l.n > 0 && l.species >= 0 && l.species < 64) has_list[l.species] = true;
    }
    if (o.with_ils) ensure_ils(ctx, ig.dnu_hi, s.opd_max, s.fwhm_gauss, o.apodization);
    double* d_grid = (double*)workspace(ctx, "grid", n_nu * sizeof(double));
    grid_values_kernel<<<(unsigned)((n_nu + 255) / 256), 256, 0, st>>>(to_dev(ig.g), d_grid);
    check_launch(ctx);
    // profiles in chunks that fit the device
    int64_t max_list = 1;
    for (auto& l : ctx->lists) max_list = std::max<int64_t>(max_list, l.n);
    int64_t total_lines = 0;
    for (auto& l : ctx->lists) total_lines += l.n;
    const size_t per_prof = (size_t)L * total_lines * 96 + (size_t)n_out * L * n_nu * 4 + (size_t)n_state * n_nu * 4 +
                            (size_t)n_nu * 8 + (size_t)n_state * n_ch * 4;
    int chunk = profiles_per_pass(ctx, n_prof, L, per_prof);
    if (o.method == 3) {  // the strip far field's node values of a pass fit its buffer
        int n_lists = 0;
        for (auto& l : ctx->lists) n_lists += l.n > 0 ? 1 : 0;
        const size_t strip_prof = (size_t)L * std::max(n_lists, 1) * (size_t)((n_nu + kJgStrip - 1) / kJgStrip) *
                                  (kJgStripWords * sizeof(float) + sizeof(int4));
        chunk = std::max(1, std::min<int>(chunk, (int)std::min<size_t>(ctx->strip_buf_max / strip_prof, n_prof)));
    }
    std::vector<float> Kf;
    for (int p0 = 0; p0 < n_prof; p0 += chunk) {
        const int np = std::min(chunk, n_prof - p0);
        Plan pl;
        std::vector<LayerRT> lrt;
        std::vector<ProfileRT> prt(np);
        std::vector<JgLayer> jl;
        std::vector<JgProfile> jp(np);
        std::vector<double> vlev((size_t)np * 4 * (L + 1), 0.0);
        for (int p = 0; p < np; ++p) {
            const irs_profile& P = profs[p0 + p];
            IRS_REQUIRE(P.n_lev == L + 1, "all profiles of a batch must have the same number of levels");
            layer_setup(P, p, o, list_sp, list_shift, ig.dnu_hi, pl.segs, lrt, prt[p]);
            for (int k = 0; k < L; ++k) {
                JgLayer y;
                y.frac = cg_mass_frac(P.pressure[k], P.pressure[k + 1]);
                const double pm = 0.5 * (P.pressure[k] + P.pressure[k + 1]);
                y.wM = std::log(pm / P.pressure[k]) / std::log(P.pressure[k + 1] / P.pressure[k]);
                y.dp = std::fabs(P.pressure[k] - P.pressure[k + 1]);
                jl.push_back(y);
            }
            JgProfile& g = jp[p];
            g.n_retr = sp.n_retrieved;
            g.retr_h2o = g.retr_co2 = -1;
            for (int r = 0; r < sp.n_retrieved; ++r) {
                const int spc = sp.retrieved[r];
                const bool cont_vmr = o.apply_continuum && sp.vmr_coupling && spc < 64 && has_list[spc];
                if (spc == 1 && cont_vmr) g.retr_h2o = r;
                if (spc == 2 && cont_vmr) g.retr_co2 = r;
                for (int q = 0; q < P.n_species; ++q)
                    if (P.species[q] == spc)
                        for (int j = 0; j <= L; ++j) vlev[((size_t)p * 4 + r) * (L + 1) + j] = P.vmr[(size_t)q * P.n_lev + j];
            }
            g.include_T = sp.include_temperature;
            g.include_tsfc = sp.include_tsfc;
            g.include_eps = sp.include_emissivity;
            g.log_vmr = sp.log_vmr;
            g.n_state = (int)n_state;
        }
        pl.n_prof = np;
        pl.L = L;
        RelmatPlan rp;  // sets SEG_RELMAT on the LM species' segments
        const bool relmat = relmat_plan(ctx, pl, o, rp, true);
        pl.pl_segs.assign((size_t)np * L, make_int2(0, 0));
        std::vector<SegDev> sd(std::max<size_t>(pl.segs.size(), 1));
        std::vector<SegW> sw(std::max<size_t>(pl.segs.size(), 1));
        std::vector<int> sn(std::max<size_t>(pl.segs.size(), 1), 0);
        int64_t off = 0;
        for (size_t i = 0; i < pl.segs.size(); ++i) {
            Segment& g = pl.segs[i];
            const int key = g.prof * L + g.layer;
            if (pl.pl_segs[key].y == 0) pl.pl_segs[key].x = (int)i;
            pl.pl_segs[key].y++;
            g.out_off = off;
            sn[i] = (int)ctx->lists[g.list].n;
            off += sn[i];
            SegDev& d = sd[i];
            d.T = g.T; d.p_atm = g.p_atm; d.vs = g.vmr_self; d.coef = g.coef; d.margin_g = g.margin_g;
            d.off = g.out_off; d.list = g.list; d.flags = g.flags;
            std::memset(&sw[i], 0, sizeof(SegW));
            jacobian_weights(profs[p0 + g.prof], o, ctx->lists[g.list].species, g.layer, sp, sw[i].w);
        }
        const int nseg = (int)pl.segs.size();
        const size_t S = (size_t)std::max<int64_t>(off, 1);
        char* base = (char*)workspace(ctx, "jg_params", S * 96);
        JgOut go;
        go.V = (double*)base; go.U = (double*)(base + S * 8);
        go.q0 = (float4*)(base + S * 16); go.q1 = (float4*)(base + S * 32); go.q2 = (float4*)(base + S * 48);
        go.q3 = (float4*)(base + S * 64); go.q4 = (float4*)(base + S * 80);
        float* d_out = (float*)workspace(ctx, "jg_out", (size_t)np * L * n_out * n_nu * sizeof(float));
        float* d_D = adjoint ? nullptr : (float*)workspace(ctx, "jg_D", (size_t)np * n_state * n_nu * sizeof(float));
        double* d_I = (double*)workspace(ctx, "I", (size_t)np * n_nu * sizeof(double));
        double* d_RB = (double*)workspace(ctx, "jg_RB", (size_t)2 * np * n_ch * sizeof(double));
        float* d_K = adjoint ? nullptr
                     : K_dev ? K_dev + (size_t)p0 * n_state * n_ch
                             : (float*)workspace(ctx, "jg_K", (size_t)np * n_state * n_ch * sizeof(float));
        SegDev* d_segs = upload(ctx, "segs", sd);
        SegW* d_sw = upload(ctx, "jg_w", sw);
        int* d_sn = upload(ctx, "jg_n", sn);
        std::vector<ListDev> ld = list_descs(ctx);
        ListDev* d_lists = upload(ctx, "list_descs", ld);
        int2* d_pl = upload(ctx, "pl_segs", pl.pl_segs);
        LayerRT* d_lrt = upload(ctx, "lrt", lrt);
        ProfileRT* d_prt = upload(ctx, "prt", prt);
        JgLayer* d_jl = upload(ctx, "jg_layer", jl);
        JgProfile* d_jp = upload(ctx, "jg_prof", jp);
        double* d_vlev = upload(ctx, "jg_vlev", vlev);
        IRS_CUDA(cudaMemsetAsync(d_out, 0, (size_t)np * L * n_out * n_nu * sizeof(float), st));
        long long pstride = 0;
        const double* d_pert = relmat ? relmat_launch(ctx, rp, d_grid, n_nu, o.lm_cutoff, o.x_far, pstride) : nullptr;
        if (nseg > 0) {
            LpConfig cfg;
            cfg.cutoff = o.cutoff; cfg.x_far = o.x_far; cfg.dptmn = 0.0; cfg.grid0 = ig.g.at(0); cfg.u_gran = 1.0 / 16.0;
            cfg.dnu_g = ig.dnu_hi; cfg.method = o.method; cfg.n_nu = n_nu;
            unsigned* d_reach = (unsigned*)workspace(ctx, "jg_reach", sizeof(unsigned) * nseg);
            IRS_CUDA(cudaMemsetAsync(d_reach, 0, sizeof(unsigned) * nseg, st));
            jg_params_kernel<<<dim3((unsigned)((max_list + 255) / 256), nseg), 256, 0, st>>>(d_segs, d_lists, tips_dev(ctx), cfg, go, d_reach);
            check_launch(ctx);
            const dim3 g2((unsigned)((n_nu + kJgStrip - 1) / kJgStrip), np * L);
            const float cut_g = (float)(o.cutoff / ig.dnu_hi);
            const bool lm = o.line_mixing == 1;
            // strip far field (pre-pass): 1808 bytes per (segment, strip); the profile passes
            // are sized so a pass fits ctx->strip_buf_max (a single profile beyond it runs without)
            float* d_sfar = nullptr;
            int4* d_srng = nullptr;
            const int n_strips = (int)g2.x;
            const size_t cells = (size_t)nseg * n_strips;
            if (o.method == 3 && cells * (kJgStripWords * sizeof(float) + sizeof(int4)) <= ctx->strip_buf_max) {
                char* b = (char*)workspace(ctx, "jg_strip", cells * (kJgStripWords * sizeof(float) + sizeof(int4)));
                d_sfar = (float*)b;
                d_srng = (int4*)(b + cells * kJgStripWords * sizeof(float));
                constexpr int nM = kJgWarps * kJgFarNodes * kJgStripNodes;
                float* d_M = (float*)workspace(ctx, "jg_strip_M", nM * sizeof(float));
                jg_strip_table_kernel<<<(nM + 255) / 256, 256, 0, st>>>(d_M);
                check_launch(ctx);
                if (lm) jg_strip_kernel<true><<<g2, kJgWarps * 32, 0, st>>>(d_segs, d_sn, d_reach, d_pl, go, cut_g, n_strips, d_M, d_sfar, d_srng);
                else jg_strip_kernel<false><<<g2, kJgWarps * 32, 0, st>>>(d_segs, d_sn, d_reach, d_pl, go, cut_g, n_strips, d_M, d_sfar, d_srng);
                check_launch(ctx);
            }
#define IRS_JG(NO)                                                                                          \
    do {                                                                                                    \
        const size_t sm = jg_smem_bytes(NO);                                                                \
        IRS_CUDA(cudaFuncSetAttribute(jg_linesum_kernel<true, NO>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm)); \
        IRS_CUDA(cudaFuncSetAttribute(jg_linesum_kernel<false, NO>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm)); \
        if (lm) jg_linesum_kernel<true, NO><<<g2, kJgWarps * 32, sm, st>>>(d_segs, d_sn, d_sw, d_pl, go, n_nu, cut_g, d_out, d_pert, pstride, d_sfar, d_srng, n_strips); \
        else jg_linesum_kernel<false, NO><<<g2, kJgWarps * 32, sm, st>>>(d_segs, d_sn, d_sw, d_pl, go, n_nu, cut_g, d_out, d_pert, pstride, d_sfar, d_srng, n_strips); \
    } while (0)
            switch (n_out) {
                case 3: IRS_JG(3); break;
                case 5: IRS_JG(5); break;
                case 7: IRS_JG(7); break;
                case 9: IRS_JG(9); break;
                default: IRS_JG(11); break;
            }
#undef IRS_JG
            check_launch(ctx);
        }
        ContDev cd = cont_dev(ctx, o);
        if (o.apply_continuum) {
            if ((o.continua & 1) && ctx->n_h2o > 1) cd.mask |= 1;
            if ((o.continua & 2) && ctx->n_co2 > 1) cd.mask |= 2;
        }
        const dim3 gr((unsigned)((n_nu + 127) / 128), np);
        const bool cia = (cd.mask & kCiaMask) != 0;
        if (!adjoint) {
            if (cia)
                jg_rte_kernel<true><<<gr, 128, 0, st>>>(d_out, n_out, d_lrt, d_jl, d_prt, d_jp, d_vlev, L, d_grid, n_nu,
                                                        o.source_function, cd, d_I, d_D);
            else
                jg_rte_kernel<<<gr, 128, 0, st>>>(d_out, n_out, d_lrt, d_jl, d_prt, d_jp, d_vlev, L, d_grid, n_nu,
                                                  o.source_function, cd, d_I, d_D);
        } else if (cia) {
            jg_rte_kernel<true, 1><<<gr, 128, 0, st>>>(d_out, n_out, d_lrt, d_jl, d_prt, d_jp, d_vlev, L, d_grid, n_nu,
                                                       o.source_function, cd, d_I, nullptr);
        } else {
            jg_rte_kernel<false, 1><<<gr, 128, 0, st>>>(d_out, n_out, d_lrt, d_jl, d_prt, d_jp, d_vlev, L, d_grid,
                                                        n_nu, o.source_function, cd, d_I, nullptr);
        }
        check_launch(ctx);
        const double* d_kern = o.with_ils ? (const double*)ctx->work["ils"].p : nullptr;
        const int64_t n_taps = o.with_ils ? ctx->ils_n : 0;
        ils_bt_kernel<<<dim3((unsigned)((n_ch * 32 + 255) / 256), np), 256, 0, st>>>(
            d_I, n_nu, d_kern, n_taps, ig.dnu_hi, to_dev(ig.g), to_dev(ch), o.with_ils, d_RB, d_RB + (size_t)np * n_ch);
        check_launch(ctx);
        if (adjoint) {  // the pullback: radiance cotangent on the grid, then the adjoint sweep
            double* d_dy = (double*)workspace(ctx, "vjp_dy", (size_t)np * n_ch * sizeof(double));
            IRS_CUDA(cudaMemcpyAsync(d_dy, dy_h + (size_t)p0 * n_ch, (size_t)np * n_ch * sizeof(double),
                                     cudaMemcpyHostToDevice, st));
            ctx->n_h2d += (double)np * n_ch * sizeof(double);
            ChanAdj* d_ca = (ChanAdj*)workspace(ctx, "vjp_chan", (size_t)np * n_ch * sizeof(ChanAdj));
            vjp_channel_kernel<<<dim3((unsigned)((n_ch + 255) / 256), np), 256, 0, st>>>(
                d_RB, d_dy, n_nu, ig.dnu_hi, to_dev(ig.g), to_dev(ch), sp.observable, d_ca);
            check_launch(ctx);
            double* d_ib = (double*)workspace(ctx, "vjp_Ibar", (size_t)np * n_nu * sizeof(double));
            ils_adjoint_kernel<<<dim3((unsigned)((n_nu + 255) / 256), np), 256, 0, st>>>(
                d_ca, n_ch, d_kern, n_taps, ig.dnu_hi, o.with_ils, n_nu, d_ib);
            check_launch(ctx);
            double* d_xb = (double*)workspace(ctx, "vjp_xbar", (size_t)np * n_state * sizeof(double));
            IRS_CUDA(cudaMemsetAsync(d_xb, 0, (size_t)np * n_state * sizeof(double), st));
            const size_t xsm = (size_t)n_state * sizeof(double);
            if (cia)
                jg_rte_kernel<true, 2><<<gr, 128, xsm, st>>>(d_out, n_out, d_lrt, d_jl, d_prt, d_jp, d_vlev, L, d_grid,
                                                             n_nu, o.source_function, cd, d_I, nullptr, d_ib, d_xb);
            else
                jg_rte_kernel<false, 2><<<gr, 128, xsm, st>>>(d_out, n_out, d_lrt, d_jl, d_prt, d_jp, d_vlev, L, d_grid,
                                                              n_nu, o.source_function, cd, d_I, nullptr, d_ib, d_xb);
            check_launch(ctx);
            IRS_CUDA(cudaMemcpyAsync(dx_h + (size_t)p0 * n_state, d_xb, (size_t)np * n_state * sizeof(double),
                                     cudaMemcpyDeviceToHost, st));
            IRS_CUDA(cudaMemcpyAsync(y_h + (size_t)p0 * n_ch, d_RB + (sp.observable == 0 ? (size_t)np * n_ch : 0),
                                     (size_t)np * n_ch * sizeof(double), cudaMemcpyDeviceToHost, st));
            IRS_CUDA(cudaStreamSynchronize(st));
            continue;
        }
        jg_channel_kernel<<<dim3((unsigned)((n_ch * 32 + 255) / 256), (unsigned)n_state, np), 256, 0, st>>>(
            d_D, n_nu, (int)n_state, o.with_ils ? (const float*)ctx->work["ils_f"].p : nullptr, n_taps, ig.dnu_hi,
            to_dev(ig.g), to_dev(ch), o.with_ils, d_RB,
            sp.observable, d_K);
        check_launch(ctx);
        if (!K_dev) {
            Kf.resize((size_t)np * n_state * n_ch);
            IRS_CUDA(cudaMemcpyAsync(Kf.data(), d_K, Kf.size() * sizeof(float), cudaMemcpyDeviceToHost, st));
        }
        IRS_CUDA(cudaMemcpyAsync(y_h + (size_t)p0 * n_ch, d_RB + (sp.observable == 0 ? (size_t)np * n_ch : 0),
                                 (size_t)np * n_ch * sizeof(double), cudaMemcpyDeviceToHost, st));
        IRS_CUDA(cudaStreamSynchronize(st));
        if (!K_dev)
            for (size_t k = 0; k < Kf.size(); ++k) K_h[(size_t)p0 * n_state * n_ch + k] = (double)Kf[k];
    }
}

static void collect_times(irs_ctx* ctx) {
    float a = 0, b = 0, c = 0, d = 0;
    IRS_CUDA(cudaEventSynchronize(ctx->ev[4]));
    IRS_CUDA(cudaEventElapsedTime(&a, ctx->ev[0], ctx->ev[1]));
    IRS_CUDA(cudaEventElapsedTime(&b, ctx->ev[1], ctx->ev[2]));
    IRS_CUDA(cudaEventElapsedTime(&c, ctx->ev[2], ctx->ev[3]));
    IRS_CUDA(cudaEventElapsedTime(&d, ctx->ev[3], ctx->ev[4]));
    ctx->last.line_params_ms = a + ctx->prior.line_params_ms;
    ctx->last.line_sum_ms = b + ctx->prior.line_sum_ms;
    ctx->last.rte_ms = c + ctx->prior.rte_ms;
    ctx->last.ils_ms = d + ctx->prior.ils_ms;
    ctx->last.total_ms = a + b + c + d + ctx->prior.total_ms;
    unsigned long long pc[3] = {0, 0, 0};
    DevBuf& pb = ctx->work["pair_counts"];
    if (pb.p) IRS_CUDA(cudaMemcpy(pc, pb.p, 24, cudaMemcpyDeviceToHost));
    ctx->last.pairs = (double)pc[0] + ctx->prior.pairs;
    ctx->last.core_pairs = (double)pc[1] + ctx->prior.core_pairs;
    ctx->last.evaluated_pairs = (double)(pc[2] ? pc[2] : pc[0]) + ctx->prior.evaluated_pairs;
    ctx->last.h2d_bytes = ctx->n_h2d;
    ctx->last.d2h_bytes = ctx->n_d2h;
    ctx->last.launches = ctx->n_launch;
    float e = 0;
    if (ctx->lm_ev) IRS_CUDA(cudaEventElapsedTime(&e, ctx->ev[7], ctx->ev[8]));
    ctx->last.lm_device_ms = e + ctx->prior.lm_device_ms;
    ctx->last.lm_host_ms = ctx->lm_host_pass + ctx->prior.lm_host_ms;
}

// Device bytes the library may use: what is free plus its own workspaces (reused or
// grown in place).
static size_t device_budget(irs_ctx* ctx) {
    size_t free_b = 0, tot_b = 0;
    IRS_CUDA(cudaMemGetInfo(&free_b, &tot_b));
    size_t own = 0;
    for (auto& w : ctx->work) own += w.second.bytes;
    return free_b + own;
}

// Profiles per pass: bounded by device memory (60% of the budget) and by the grid
// limits of the per-segment and per-(profile, layer) launches (65535 in y).
static int profiles_per_pass(irs_ctx* ctx, int n_prof, int L, size_t per_prof) {
    int n_lists = 0;
    for (auto& l : ctx->lists) n_lists += l.n > 0 ? 1 : 0;
    const size_t by_mem = std::max<size_t>(1, device_budget(ctx) * 6 / 10 / std::max<size_t>(per_prof, 1));
    const size_t by_grid = std::max<size_t>(1, 65535 / (size_t)std::max(1, L * std::max(n_lists, 1)));
    return (int)std::min<size_t>((size_t)n_prof, std::min(by_mem, by_grid));
}

// forward_model for a batch: one pass when the batch fits, else sequential passes
// (each pass but the last is waited for so its stage times can be added up).
static void forward_device(irs_ctx* ctx, const irs_profile* profs, int n_prof, const irs_sounder& s,
                           const irs_fm_options& o, double* d_R, double* d_BT) {
    IRS_REQUIRE(n_prof >= 1 && profs, "need at least one profile");
    validate_options(o);
    ctx->n_h2d = ctx->n_d2h = ctx->n_launch = 0;
    ctx->lm_host_pass = 0;
    ctx->lm_ev = false;
    ctx->prior = irs_stage_times{};
    const InternalGrid ig = internal_grid(s, o);
    const GridSpec ch = make_grid(s.nu_min, s.nu_max, s.dnu);
    const int L = profs[0].n_lev - 1;
    IRS_REQUIRE(L >= 1, "a profile needs at least two levels");
    int64_t total_lines = 0;
    for (auto& l : ctx->lists) total_lines += l.n;
    const bool mixed = o.precision != IRS_FP64;
    const size_t per_prof = (size_t)L * total_lines * (mixed ? 65 : 49) + (size_t)L * ig.g.n * (mixed ? 4 : 8) +
                            (size_t)ig.g.n * 8;
    const int chunk = profiles_per_pass(ctx, n_prof, L, per_prof);
    for (int p0 = 0; p0 < n_prof; p0 += chunk) {
        const int np = std::min(chunk, n_prof - p0);
        forward_pass(ctx, profs + p0, np, s, o, d_R + (size_t)p0 * ch.n, d_BT + (size_t)p0 * ch.n);
        if (p0 + np < n_prof) {
            const double h2d = ctx->n_h2d, d2h = ctx->n_d2h, nl = ctx->n_launch;
            const irs_stage_times keep = ctx->prior;
            collect_times(ctx);
            ctx->prior = ctx->last;
            ctx->prior.line_params_ms += keep.line_params_ms;
            ctx->prior.line_sum_ms += keep.line_sum_ms;
            ctx->prior.rte_ms += keep.rte_ms;
            ctx->prior.ils_ms += keep.ils_ms;
            ctx->prior.total_ms += keep.total_ms;
            ctx->prior.pairs += keep.pairs;
            ctx->prior.core_pairs += keep.core_pairs;
            ctx->prior.evaluated_pairs += keep.evaluated_pairs;
            ctx->prior.lm_host_ms += keep.lm_host_ms;
            ctx->prior.lm_device_ms += keep.lm_device_ms;
            ctx->n_h2d = h2d, ctx->n_d2h = d2h, ctx->n_launch = nl;
        }
    }
}

// ------------------------------------------------------------ optimal estimation
// unpack_state (state_vector.jl:380-403) into an irs_profile whose arrays live in T / vmr
static void unpack_into(const irs_state_spec& sp, const double* x, const irs_profile& base, double eps_fixed,
                        std::vector<double>& T, std::vector<double>& vmr, irs_profile& out) {
    const int nl = base.n_lev;
    out = base;
    T.assign(base.temperature, base.temperature + nl);
    vmr.assign(base.vmr, base.vmr + (size_t)base.n_species * nl);
    int k = 0;
    if (sp.include_temperature) {
        for (int j = 0; j < nl; ++j) T[j] = x[k + j];
        k += nl;
    }
    for (int r = 0; r < sp.n_retrieved; ++r) {
        int q = -1;
        for (int i = 0; i < base.n_species; ++i)
            if (base.species[i] == sp.retrieved[r]) q = i;
        IRS_REQUIRE(q >= 0, "base profile is missing a retrieved species");
        for (int j = 0; j < nl; ++j) vmr[(size_t)q * nl + j] = sp.log_vmr ? std::exp(x[k + j]) : x[k + j];
        k += nl;
    }
    out.temperature = T.data();
    out.vmr = vmr.data();
    out.T_sfc = sp.include_tsfc ? x[k++] : T[0];
    out.eps_sfc = sp.include_emissivity ? x[k++] : eps_fixed;
}

// Profiles of the states x[list[i]] (arrays owned by the returned holder)
struct StateProfiles {
    std::vector<std::vector<double>> T, vmr;
    std::vector<irs_profile> prof;
};
static void build_profiles(const irs_state_spec& sp, const std::vector<int>& list, const double* x, int n,
                           const irs_profile* base, double eps_fixed, StateProfiles& h) {
    h.T.assign(list.size(), {});
    h.vmr.assign(list.size(), {});
    h.prof.assign(list.size(), irs_profile{});
    for (size_t i = 0; i < list.size(); ++i)
        unpack_into(sp, x + (size_t)list[i] * n, base[list[i]], eps_fixed, h.T[i], h.vmr[i], h.prof[i]);
}

static void launch_oe_normal(irs_ctx* ctx, const int* d_list, int n_list, int n, int n_ch, const float* K,
                             const double* w, const double* r, double* M, double* b) {
    const size_t smem = (size_t)(2 * kOeTile * n + kOeTile) * sizeof(double);
    static bool attr = false;
    if (!attr) {
        IRS_CUDA(cudaFuncSetAttribute(oe_normal_kernel<256>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
        IRS_CUDA(cudaFuncSetAttribute(oe_normal_kernel<512>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
        attr = true;
    }
    const int grid = std::min(n_list, 148 * 4);
    if (n * (n + 1) / 2 <= 256 * kOePairsPerThread)
        oe_normal_kernel<256><<<grid, 256, smem, ctx->stream>>>(d_list, n_list, n, n_ch, K, w, r, M, b);
    else
        oe_normal_kernel<512><<<grid, 512, smem, ctx->stream>>>(d_list, n_list, n, n_ch, K, w, r, M, b);
    check_launch(ctx);
}

static void launch_oe_solve(irs_ctx* ctx, const int* d_list, int n_list, int n, const double* M, const double* b,
                            const double* Sa_inv, const double* x, const double* xa, const double* gamma, double* dx,
                            double* d2, int* ok) {
    const size_t smem = ((size_t)n * n + 4 * (size_t)n) * sizeof(double);  // 210 KB at n = 160
    static bool attr = false;
    if (!attr) {
        IRS_CUDA(cudaFuncSetAttribute(oe_solve_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024));
        attr = true;
    }
    const int grid = std::min(n_list, 148);
    oe_solve_kernel<<<grid, kOeThreads, smem, ctx->stream>>>(d_list, n_list, n, M, b, Sa_inv, x, xa, gamma, dx, d2, ok);
    check_launch(ctx);
}

// optimal_estimation (optimal_estimation.jl:142-291) for a batch of scenes: every scene
// runs its own Levenberg-Marquardt (or Gauss-Newton) iteration; each LM stage (normal
// equations, damped solve, trial forward model, Jacobian at accepted states) is one
// batched call over the scenes still iterating.
// A banded Se per scene (lower band se_band[sc][i][k] = Se(i, i-k), k = 0..bw) on the
// channels with keep[i] != 0; null band: diagonal Se given as se_inv.
struct SeBand {
    const double* band = nullptr;
    int bw = 0;
    const uint8_t* keep = nullptr;
};

static void oe_batch(irs_ctx* ctx, const irs_profile* base, int n_scene, const irs_sounder& s,
                     const irs_fm_options& o_in, const irs_state_spec& sp, const double* y_obs, const double* se_inv,
                     const double* xa, const double* Sa_inv, const double* x0, const irs_oe_params& prm,
                     double* x_out, double* y_fit, double* M_out, int32_t* n_iter, int32_t* converged,
                     double* cost_out, const SeBand& seb = SeBand()) {
    IRS_REQUIRE(n_scene >= 1 && base, "need at least one scene");
    IRS_REQUIRE(prm.method == 0 || prm.method == 1, "method must be 0 (levenberg_marquardt) or 1 (gauss_newton)");
    IRS_REQUIRE(prm.max_iter >= 1 && prm.max_linesearch >= 1, "max_iter and max_linesearch must be positive");
    const int n = (int)state_size(sp, base[0].n_lev);
    IRS_REQUIRE(n >= 1 && n <= kOeMaxState, "the state vector must have 1 to 160 elements on this path");
    const int64_t n_ch = make_grid(s.nu_min, s.nu_max, s.dnu).n;
    irs_fm_options o = o_in;
    o.dptmn = 0.0;  // frozen line set for F as for K (optimal_estimation.jl:193-198)
    const cudaStream_t st = ctx->stream;
    const size_t S = (size_t)n_scene;
    // device state
    float* d_K = (float*)workspace(ctx, "oe_K", S * n * n_ch * sizeof(float));
    float* d_Kt = (float*)workspace(ctx, "oe_Ktmp", S * n * n_ch * sizeof(float));
    double* d_w = (double*)workspace(ctx, "oe_w", S * n_ch * sizeof(double));
    double* d_r = (double*)workspace(ctx, "oe_r", S * n_ch * sizeof(double));
    double* d_M = (double*)workspace(ctx, "oe_M", S * n * n * sizeof(double));
    double* d_b = (double*)workspace(ctx, "oe_b", S * n * sizeof(double));
    double* d_Sa = (double*)workspace(ctx, "oe_Sa", (size_t)n * n * sizeof(double));
    double* d_x = (double*)workspace(ctx, "oe_x", S * n * sizeof(double));
    double* d_xa = (double*)workspace(ctx, "oe_xa", S * n * sizeof(double));
    double* d_g = (double*)workspace(ctx, "oe_gamma", S * sizeof(double));
    double* d_dx = (double*)workspace(ctx, "oe_dx", S * n * sizeof(double));
    double* d_d2 = (double*)workspace(ctx, "oe_d2", S * sizeof(double));
    int* d_ok = (int*)workspace(ctx, "oe_ok", S * sizeof(int));
    int* d_list = (int*)workspace(ctx, "oe_list", S * sizeof(int));
    double* d_fm = (double*)workspace(ctx, "oe_fm", 2 * S * n_ch * sizeof(double));
    // banded Se: Cholesky factors on the kept channels; the retrieval then runs on
    // whitened residuals and Jacobians with unit weights (optimal_estimation.jl:166-176)
    const bool banded = seb.band != nullptr;
    std::vector<int> kidx;
    std::vector<double> Lb, w_unit;
    int* d_kidx = nullptr;
    double* d_Lb = nullptr;
    if (banded) {
        IRS_REQUIRE(seb.bw >= 0 && seb.bw <= kOeMaxBand, "the Se band half-width must be 0..32");
        for (int64_t i = 0; i < n_ch; ++i) if (seb.keep[i]) kidx.push_back((int)i);
        IRS_REQUIRE(!kidx.empty(), "channel_mask keeps no channel");
        const int nk = (int)kidx.size(), bw = seb.bw;
        Lb.assign(S * nk * (bw + 1), 0.0);
        for (size_t sc = 0; sc < S; ++sc) {  // banded Cholesky of Se[keep, keep]
            const double* B = seb.band + sc * n_ch * (bw + 1);
            double* L = Lb.data() + sc * nk * (bw + 1);
            for (int i = 0; i < nk; ++i) {
                for (int k = bw; k >= 0; --k) {
                    const int j = i - k;
                    if (j < 0) continue;
                    const int lag = kidx[i] - kidx[j];
                    double v = lag <= bw ? B[(size_t)kidx[i] * (bw + 1) + lag] : 0.0;
                    for (int m = 1; m <= bw && j - m >= 0; ++m)
                        if (k + m <= bw) v -= L[(size_t)i * (bw + 1) + k + m] * L[(size_t)j * (bw + 1) + m];
                    if (k == 0) {
                        IRS_REQUIRE(v > 0.0, "Se is not positive definite on the kept channels");
                        L[(size_t)i * (bw + 1)] = std::sqrt(v);
                    } else {
                        L[(size_t)i * (bw + 1) + k] = v / L[(size_t)j * (bw + 1)];
                    }
                }
            }
        }
        w_unit.assign(S * n_ch, 0.0);
        for (size_t sc = 0; sc < S; ++sc) for (int i : kidx) w_unit[sc * n_ch + i] = 1.0;
        se_inv = w_unit.data();
        d_kidx = upload(ctx, "oe_kidx", kidx);
        d_Lb = upload(ctx, "oe_Lband", Lb);
    }
    // residual y - F of one scene, whitened (L^-1 r on the kept channels) for a banded Se
    auto residual = [&](int sc, const double* Fs, double* r) {
        const double* ys = y_obs + (size_t)sc * n_ch;
        for (int64_t i = 0; i < n_ch; ++i) r[i] = ys[i] - Fs[i];
        if (!banded) return;
        const int nk = (int)kidx.size(), bw = seb.bw;
        const double* L = Lb.data() + (size_t)sc * nk * (bw + 1);
        std::vector<double> z(nk);
        for (int i = 0; i < nk; ++i) {
            double v = r[kidx[i]];
            for (int k = 1; k <= bw && k <= i; ++k) v -= L[(size_t)i * (bw + 1) + k] * z[i - k];
            z[i] = v / L[(size_t)i * (bw + 1)];
        }
        std::fill(r, r + n_ch, 0.0);
        for (int i = 0; i < nk; ++i) r[kidx[i]] = z[i];
    };
    IRS_CUDA(cudaMemcpyAsync(d_w, se_inv, S * n_ch * sizeof(double), cudaMemcpyHostToDevice, st));
    IRS_CUDA(cudaMemcpyAsync(d_Sa, Sa_inv, (size_t)n * n * sizeof(double), cudaMemcpyHostToDevice, st));
    IRS_CUDA(cudaMemcpyAsync(d_xa, xa, S * n * sizeof(double), cudaMemcpyHostToDevice, st));

    std::vector<double> x(x0, x0 + S * n), F(S * n_ch), J(S), gamma(S, prm.method == 1 ? 0.0 : prm.gamma0);
    std::vector<int32_t> iters(S, 0), conv(S, 0);
    std::vector<double> rbuf(n_ch);
    auto cost = [&](int sc, const double* Fs, const double* xs) {
        double c = 0.0;
        const double* ws = se_inv + (size_t)sc * n_ch;
        residual(sc, Fs, rbuf.data());
        for (int64_t i = 0; i < n_ch; ++i) c += rbuf[i] * ws[i] * rbuf[i];
        std::vector<double> d(n);
        for (int i = 0; i < n; ++i) d[i] = xs[i] - xa[(size_t)sc * n + i];
        for (int i = 0; i < n; ++i) {
            double v = 0.0;
            for (int j = 0; j < n; ++j) v += Sa_inv[(size_t)i * n + j] * d[j];
            c += d[i] * v;
        }
        return c;
    };
    // F and K at the states of `list` (K into the scene slots of d_K)
    auto jac = [&](const std::vector<int>& list) {
        if (list.empty()) return;
        StateProfiles h;
        build_profiles(sp, list, x.data(), n, base, prm.eps_fixed, h);
        std::vector<double> y((size_t)list.size() * n_ch);
        jacobian_device(ctx, h.prof.data(), (int)list.size(), s, o, sp, nullptr, y.data(), d_Kt);
        for (size_t i = 0; i < list.size(); ++i) {
            const int sc = list[i];
            if (sc != (int)i || d_Kt != d_K)
                IRS_CUDA(cudaMemcpyAsync(d_K + (size_t)sc * n * n_ch, d_Kt + i * n * n_ch, (size_t)n * n_ch * sizeof(float),
                                         cudaMemcpyDeviceToDevice, st));
            std::copy(y.begin() + i * n_ch, y.begin() + (i + 1) * n_ch, F.begin() + (size_t)sc * n_ch);
        }
        if (banded) {  // K <- L^-1 K for these scenes
            IRS_CUDA(cudaMemcpyAsync(d_list, list.data(), list.size() * sizeof(int), cudaMemcpyHostToDevice, st));
            const int nt = (int)list.size() * n;
            oe_whiten_kernel<<<(nt + 127) / 128, 128, 0, st>>>(d_list, (int)list.size(), n, (int)n_ch, d_K, d_kidx,
                                                               (int)kidx.size(), d_Lb, seb.bw);
            check_launch(ctx);
        }
    };
    auto upload_resid = [&](const std::vector<int>& list) {
        std::vector<double> r((size_t)n_ch);
        for (int sc : list) {
            residual(sc, F.data() + (size_t)sc * n_ch, r.data());
            IRS_CUDA(cudaMemcpyAsync(d_r + (size_t)sc * n_ch, r.data(), n_ch * sizeof(double), cudaMemcpyHostToDevice, st));
            IRS_CUDA(cudaStreamSynchronize(st));
        }
    };

    std::vector<int> all(S);
    std::iota(all.begin(), all.end(), 0);
    jac(all);
    for (int sc = 0; sc < n_scene; ++sc) J[sc] = cost(sc, F.data() + (size_t)sc * n_ch, x.data() + (size_t)sc * n);
    std::vector<int> active = all;
    while (!active.empty()) {
        for (int sc : active) iters[sc] += 1;
        upload_resid(active);
        IRS_CUDA(cudaMemcpyAsync(d_list, active.data(), active.size() * sizeof(int), cudaMemcpyHostToDevice, st));
        launch_oe_normal(ctx, d_list, (int)active.size(), n, (int)n_ch, d_K, d_w, d_r, d_M, d_b);
        std::vector<int> pending = active, accepted;
        std::vector<double> d2n(S, 0.0);
        for (int ls = 0; ls < prm.max_linesearch && !pending.empty(); ++ls) {
            IRS_CUDA(cudaMemcpyAsync(d_x, x.data(), S * n * sizeof(double), cudaMemcpyHostToDevice, st));
            IRS_CUDA(cudaMemcpyAsync(d_g, gamma.data(), S * sizeof(double), cudaMemcpyHostToDevice, st));
            IRS_CUDA(cudaMemcpyAsync(d_list, pending.data(), pending.size() * sizeof(int), cudaMemcpyHostToDevice, st));
            launch_oe_solve(ctx, d_list, (int)pending.size(), n, d_M, d_b, d_Sa, d_x, d_xa, d_g, d_dx, d_d2, d_ok);
            std::vector<double> dx(S * n), d2(S);
            std::vector<int> okv(S);
            IRS_CUDA(cudaMemcpyAsync(dx.data(), d_dx, S * n * sizeof(double), cudaMemcpyDeviceToHost, st));
            IRS_CUDA(cudaMemcpyAsync(d2.data(), d_d2, S * sizeof(double), cudaMemcpyDeviceToHost, st));
            IRS_CUDA(cudaMemcpyAsync(okv.data(), d_ok, S * sizeof(int), cudaMemcpyDeviceToHost, st));
            IRS_CUDA(cudaStreamSynchronize(st));
            std::vector<double> xt(S * n);
            std::vector<int> trial;
            for (int sc : pending) {
                if (!okv[sc]) continue;  // damped normal matrix not positive definite: no step
                for (int i = 0; i < n; ++i) xt[(size_t)sc * n + i] = x[(size_t)sc * n + i] + dx[(size_t)sc * n + i];
                trial.push_back(sc);
            }
            std::vector<double> Ft;
            if (!trial.empty()) {
                StateProfiles h;
                build_profiles(sp, trial, xt.data(), n, base, prm.eps_fixed, h);
                const size_t nt = trial.size();
                IRS_REQUIRE(2 * nt * n_ch <= 2 * S * n_ch, "trial batch");
                forward_device(ctx, h.prof.data(), (int)nt, s, o, d_fm, d_fm + nt * n_ch);
                Ft.resize(nt * n_ch);
                IRS_CUDA(cudaMemcpyAsync(Ft.data(), d_fm + (sp.observable == 0 ? nt * n_ch : 0), nt * n_ch * sizeof(double),
                                         cudaMemcpyDeviceToHost, st));
                IRS_CUDA(cudaStreamSynchronize(st));
            }
            std::vector<int> still;
            size_t ti = 0;
            for (int sc : pending) {
                if (!okv[sc]) {
                    if (prm.method == 0) { gamma[sc] *= prm.gamma_factor; still.push_back(sc); }
                    continue;
                }
                const double* Fs = Ft.data() + (ti++) * n_ch;
                const double Jt = cost(sc, Fs, xt.data() + (size_t)sc * n);
                if (Jt < J[sc]) {
                    d2n[sc] = d2[sc] / n;
                    std::copy(xt.begin() + (size_t)sc * n, xt.begin() + (size_t)(sc + 1) * n, x.begin() + (size_t)sc * n);
                    J[sc] = Jt;
                    if (prm.method == 0) gamma[sc] = std::max(gamma[sc] / prm.gamma_factor, prm.gamma_min);
                    accepted.push_back(sc);
                } else if (prm.method == 0) {
                    gamma[sc] *= prm.gamma_factor;
                    still.push_back(sc);
                }
            }
            pending.swap(still);
        }
        jac(accepted);  // F, K at the accepted states (optimal_estimation.jl:227-229)
        std::vector<int> next;
        for (int sc : accepted) {
            if (d2n[sc] < prm.conv_factor) conv[sc] = 1;
            else if (iters[sc] < prm.max_iter) next.push_back(sc);
        }
        active.swap(next);
    }
    // normal matrix at the solution for the diagnostics
    upload_resid(all);
    IRS_CUDA(cudaMemcpyAsync(d_list, all.data(), S * sizeof(int), cudaMemcpyHostToDevice, st));
    launch_oe_normal(ctx, d_list, n_scene, n, (int)n_ch, d_K, d_w, d_r, d_M, d_b);
    IRS_CUDA(cudaMemcpyAsync(M_out, d_M, S * n * n * sizeof(double), cudaMemcpyDeviceToHost, st));
    IRS_CUDA(cudaStreamSynchronize(st));
    std::copy(x.begin(), x.end(), x_out);
    std::copy(F.begin(), F.end(), y_fit);
    for (int sc = 0; sc < n_scene; ++sc) {
        n_iter[sc] = iters[sc];
        converged[sc] = conv[sc];
        cost_out[sc] = J[sc];
    }
}

}  // namespace irs

using namespace irs;

#define IRS_API_BEGIN try {
#define IRS_API_END                                  \
    return IRS_OK;                                   \
    }                                                \
    catch (const Error& e) {                         \
        set_error(e.msg);                            \
        return e.code;                               \
    }                                                \
    catch (const std::exception& e) {                \
        set_error(std::string("exception: ") + e.what()); \
        return IRS_E_STATE;                          \
    }

extern "C" {

int irs_abi_version(void) { return IRS_ABI_VERSION; }
const char* irs_last_error(void) { return irs::last_error(); }

int irs_create(int device, irs_ctx** out) {
    IRS_API_BEGIN
    IRS_REQUIRE(out, "out is NULL");
    *out = nullptr;
    int n = 0;
    IRS_CUDA(cudaGetDeviceCount(&n));
    IRS_REQUIRE(device >= 0 && device < n, "no such CUDA device");
    IRS_CUDA(cudaSetDevice(device));
    std::unique_ptr<irs_ctx> c(new irs_ctx);
    c->device = device;
    if (const char* e = std::getenv("IRS_STRIP_BUFFER_BYTES")) {
        const long long v = std::atoll(e);
        IRS_REQUIRE(v > 0, "IRS_STRIP_BUFFER_BYTES must be a positive byte count");
        c->strip_buf_max = (size_t)v;
    }
    IRS_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    for (auto& e : c->ev) IRS_CUDA(cudaEventCreate(&e));
    FaddeevaConsts fc;
    compute_faddeeva_consts(&fc);
    IRS_CUDA(cudaMemcpyToSymbol(c_fad, &fc, sizeof fc));
    *out = c.release();
    IRS_API_END
}

int irs_destroy(irs_ctx* ctx) {
    IRS_API_BEGIN
    if (!ctx) return IRS_OK;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    for (auto& l : ctx->lists) {
        cudaFree(l.nu);  // one allocation per list (see irs_upload_linelist)
    }
    for (auto& w : ctx->work) if (w.second.p) cudaFree(w.second.p);
    for (auto& e : ctx->ev) cudaEventDestroy(e);
    cudaStreamDestroy(ctx->stream);
    delete ctx;
    IRS_API_END
}

int irs_set_partition_table(irs_ctx* ctx, int mol, int iso, int t_min, int n, const double* q) {
    IRS_API_BEGIN
    IRS_REQUIRE(ctx && q && n >= 2, "invalid partition table");
    ctx->tables.tips[{mol, iso}] = {t_min, std::vector<double>(q, q + n)};
    ctx->tips_dirty = true;
    IRS_API_END
}

int irs_set_continuum_h2o(irs_ctx* ctx, int n, const double* nu, const double* cs, const double* cf,
                          const double* te) {
    IRS_API_BEGIN
    IRS_REQUIRE(ctx && n >= 2 && nu && cs && cf && te, "invalid H2O continuum table");
    for (int i = 1; i < n; ++i) IRS_REQUIRE(nu[i] > nu[i - 1], "continuum knots must increase");
    Tables& t = ctx->tables;
    t.h2o_nu.assign(nu, nu + n); t.h2o_cs.assign(cs, cs + n); t.h2o_cf.assign(cf, cf + n); t.h2o_te.assign(te, te + n);
    ctx->cont_dirty = true;
    IRS_API_END
}

int irs_set_continuum_co2(irs_ctx* ctx, int n, const double* nu, const double* s, const double* xf,
                          const double* td) {
    IRS_API_BEGIN
    IRS_REQUIRE(ctx && n >= 2 && nu && s && xf && td, "invalid CO2 continuum table");
    for (int i = 1; i < n; ++i) IRS_REQUIRE(nu[i] > nu[i - 1], "continuum knots must increase");
    Tables& t = ctx->tables;
    t.co2_nu.assign(nu, nu + n);
    t.co2_s.resize(n);
    for (int i = 0; i < n; ++i) t.co2_s[i] = s[i] * xf[i];  // continuum.jl:90
    t.co2_tdep.assign(td, td + n);
    ctx->cont_dirty = true;
    IRS_API_END
}

int irs_set_cia(irs_ctx* ctx, int pair, int n_blocks, const double* T, const int64_t* off, const double* nu,
                const double* sigma) {
    IRS_API_BEGIN
    IRS_REQUIRE(ctx && pair >= 1 && pair <= 3, "CIA pair must be 1 (CO2-CO2), 2 (N2-N2) or 3 (O2-O2)");
    IRS_REQUIRE(n_blocks >= 0 && (n_blocks == 0 || (T && off && nu && sigma)), "invalid CIA table");
    std::vector<Tables::CiaBlock> B;
    for (int b = 0; b < n_blocks; ++b) {
        IRS_REQUIRE(off[b + 1] >= off[b], "CIA block offsets must not decrease");
        if (off[b + 1] == off[b]) continue;
        Tables::CiaBlock c;
        c.T = T[b];
        c.nu.assign(nu + off[b], nu + off[b + 1]);
        c.sg.assign(sigma + off[b], sigma + off[b + 1]);
        for (size_t i = 1; i < c.nu.size(); ++i) IRS_REQUIRE(c.nu[i] > c.nu[i - 1], "CIA knots must increase");
        B.push_back(std::move(c));
    }
    ctx->tables.cia[pair - 1] = std::move(B);
    ctx->cont_dirty = true;
    IRS_API_END
}

int irs_upload_linelist(irs_ctx* ctx, int species, const irs_line* lines, int64_t n, const double* y0) {
    IRS_API_BEGIN
    IRS_REQUIRE(ctx && n >= 0 && (n == 0 || lines), "invalid line list");
    IRS_CUDA(cudaSetDevice(ctx->device));
    upload_tables(ctx);
    // HITRANLinelist sorts by wavenumber (linelist.jl:51-56); keep that order.
    std::vector<int64_t> ord(n);
    std::iota(ord.begin(), ord.end(), 0);
    std::stable_sort(ord.begin(), ord.end(), [&](int64_t a, int64_t b) { return lines[a].wavenumber < lines[b].wavenumber; });
    std::vector<double> h((size_t)n * 8);
    std::vector<int> tips(n);
    double max_shift = 0.0;
    uint32_t iso_mask = 0;
    const double d_self = species == 1 ? 0.002 : (species == 2 ? -0.003 : 0.0);
    for (int64_t k = 0; k < n; ++k) {
        const irs_line& l = lines[ord[k]];
        IRS_REQUIRE(l.mol_id == species, "line mol_id does not match the species of the list");
        h[0 * n + k] = l.wavenumber;
        h[1 * n + k] = l.intensity;
        h[2 * n + k] = l.lower_energy;
        h[3 * n + k] = (double)l.air_broad;
        h[4 * n + k] = (double)l.self_broad;
        h[5 * n + k] = (double)l.temp_depend;
        h[6 * n + k] = (double)l.pressure_shift;
        h[7 * n + k] = y0 ? y0[ord[k]] : 0.0;
        auto it = ctx->tips_index.find({(int)l.mol_id, (int)l.iso_id});
        tips[k] = it == ctx->tips_index.end() ? -1 : it->second;
        const int iso = l.iso_id == 0 ? 10 : (int)l.iso_id;
        if (iso >= 0 && iso < 32) iso_mask |= 1u << iso;
        max_shift = std::max(max_shift, std::fabs((double)l.pressure_shift) + std::fabs(d_self));
    }
    // replace an existing list of this species
    int slot = -1;
    for (size_t i = 0; i < ctx->lists.size(); ++i) if (ctx->lists[i].species == species) slot = (int)i;
    if (slot >= 0) {
        cudaFree(ctx->lists[slot].nu);
        ctx->lists.erase(ctx->lists.begin() + slot);
    }
    DevLineList d;
    d.species = species;
    d.n = n;
    d.has_y0 = y0 != nullptr;
    d.max_abs_shift = max_shift;
    d.iso_mask = iso_mask;
    const size_t bytes = (size_t)std::max<int64_t>(n, 1) * (8 * sizeof(double) + sizeof(int));
    char* base = nullptr;
    if (cudaMalloc((void**)&base, bytes) != cudaSuccess) {
        cudaGetLastError();
        throw Error{IRS_E_NOMEM, "device allocation for the line list failed"};
    }
    double* b = (double*)base;
    const size_t N = (size_t)std::max<int64_t>(n, 1);
    d.nu = b; d.S296 = b + N; d.E = b + 2 * N; d.gair = b + 3 * N; d.gself = b + 4 * N;
    d.nair = b + 5 * N; d.delta = b + 6 * N; d.y0 = b + 7 * N;
    d.tips = (int*)(b + 8 * N);
    if (n > 0) {
        for (int f = 0; f < 8; ++f)
            IRS_CUDA(cudaMemcpy(b + f * N, h.data() + (size_t)f * n, n * sizeof(double), cudaMemcpyHostToDevice));
        IRS_CUDA(cudaMemcpy(d.tips, tips.data(), n * sizeof(int), cudaMemcpyHostToDevice));
    }
    ctx->lists.push_back(d);
    std::sort(ctx->lists.begin(), ctx->lists.end(), [](const DevLineList& a, const DevLineList& b) { return a.species < b.species; });
    IRS_API_END
}

int irs_cross_sections(irs_ctx* ctx, int species, const double* grid, int64_t n_nu, double T, double p_atm,
                       double vmr_self, double cutoff, int method, double x_far, int precision, double* sigma) {
    IRS_API_BEGIN
    IRS_REQUIRE(ctx && grid && sigma && n_nu >= 1, "invalid arguments");
    IRS_REQUIRE(T > 0 && p_atm >= 0, "T must be positive and p_atm non-negative");
    IRS_CUDA(cudaSetDevice(ctx->device));
    int li = -1;
    for (size_t i = 0; i < ctx->lists.size(); ++i) if (ctx->lists[i].species == species) li = (int)i;
    IRS_REQUIRE(li >= 0, "no line list uploaded for this species");
    irs_fm_options o{};
    o.method = method; o.precision = precision; o.cutoff = cutoff; o.lm_cutoff = cutoff; o.x_far = x_far;
    o.dptmn = 0.0;
    validate_options(o);
    upload_tables(ctx);
    double dnu_g = n_nu > 1 ? (grid[n_nu - 1] - grid[0]) / double(n_nu - 1) : 1.0;
    if (precision != IRS_FP64) {
        IRS_REQUIRE(n_nu > 1 && dnu_g > 0, "the mixed kernel needs a uniform increasing grid");
        for (int64_t i = 0; i < n_nu; ++i)
            IRS_REQUIRE(std::fabs(grid[i] - (grid[0] + double(i) * dnu_g)) <= 1e-9 * std::max(1.0, std::fabs(grid[i])),
                        "the mixed kernel needs a uniform grid");
    }
    Plan pl;
    pl.n_prof = 1;
    pl.L = 1;
    Segment s{};
    s.T = T; s.p_atm = p_atm; s.vmr_self = vmr_self; s.coef = 1.0; s.list = li; s.flags = 0;
    s.margin_g = ctx->lists[li].max_abs_shift * p_atm / dnu_g + 2.0;
    pl.segs.push_back(s);
    pl.pl_segs.push_back(make_int2(0, 1));
    cudaStream_t st = ctx->stream;
    IRS_CUDA(cudaEventRecord(ctx->ev[0], st));
    double* d_grid = (double*)workspace(ctx, "grid", n_nu * sizeof(double));
    IRS_CUDA(cudaMemcpyAsync(d_grid, grid, n_nu * sizeof(double), cudaMemcpyHostToDevice, st));
    void* d_tau = run_linesum(ctx, pl, d_grid, n_nu, grid[0], dnu_g, o, 1);
    IRS_CUDA(cudaEventRecord(ctx->ev[2], st));
    if (precision != IRS_FP64) {
        std::vector<float> tmp(n_nu);
        IRS_CUDA(cudaMemcpyAsync(tmp.data(), d_tau, n_nu * sizeof(float), cudaMemcpyDeviceToHost, st));
        IRS_CUDA(cudaStreamSynchronize(st));
        for (int64_t i = 0; i < n_nu; ++i) sigma[i] = tmp[i];
    } else {
        IRS_CUDA(cudaMemcpyAsync(sigma, d_tau, n_nu * sizeof(double), cudaMemcpyDeviceToHost, st));
        IRS_CUDA(cudaStreamSynchronize(st));
    }
    IRS_API_END
}

int irs_forward_model_batch_device(irs_ctx* ctx, const irs_profile* profs, int n_prof, const irs_sounder* s,
                                   const irs_fm_options* o, double* d_R, double* d_BT, void* stream) {
    IRS_API_BEGIN
    IRS_REQUIRE(ctx && s && o && d_R && d_BT, "invalid arguments");
    IRS_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t user = (cudaStream_t)stream;
    if (user) {  // order our stream after the caller's work, and the caller's after ours
        IRS_CUDA(cudaEventRecord(ctx->ev[5], user));
        IRS_CUDA(cudaStreamWaitEvent(ctx->stream, ctx->ev[5], 0));
    }
    forward_device(ctx, profs, n_prof, *s, *o, d_R, d_BT);
    if (user) {
        IRS_CUDA(cudaEventRecord(ctx->ev[6], ctx->stream));
        IRS_CUDA(cudaStreamWaitEvent(user, ctx->ev[6], 0));
    }
    IRS_API_END
}

int irs_forward_model_batch(irs_ctx* ctx, const irs_profile* profs, int n_prof, const irs_sounder* s,
                            const irs_fm_options* o, double* R, double* BT) {
    IRS_API_BEGIN
    IRS_REQUIRE(ctx && s && o && R && BT, "invalid arguments");
    IRS_CUDA(cudaSetDevice(ctx->device));
    const GridSpec ch = make_grid(s->nu_min, s->nu_max, s->dnu);
    const size_t n = (size_t)n_prof * ch.n;
    double* d_out = (double*)workspace(ctx, "fm_out", 2 * n * sizeof(double));
    forward_device(ctx, profs, n_prof, *s, *o, d_out, d_out + n);
    IRS_CUDA(cudaMemcpyAsync(R, d_out, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    IRS_CUDA(cudaMemcpyAsync(BT, d_out + n, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    ctx->n_d2h += 2.0 * n * sizeof(double);
    IRS_CUDA(cudaStreamSynchronize(ctx->stream));
    collect_times(ctx);
    IRS_API_END
}

int irs_upload_relmat(irs_ctx* ctx, int species, const irs_relmat_band* bands, int n_bands,
                      const irs_wtfit_entry* wtfit, int64_t n_wtfit, double min_band_strength) {
    IRS_API_BEGIN
    IRS_REQUIRE(ctx && n_bands >= 0 && (n_bands == 0 || bands) && n_wtfit >= 0 && (n_wtfit == 0 || wtfit),
                "invalid relmat arguments");
    RelmatHost R;
    if (n_bands > 0) {
        IRS_REQUIRE(species > 0, "relmat species must be a HITRAN molecule id");
        R.species = species;
        R.min_band_strength = min_band_strength;
        for (int b = 0; b < n_bands; ++b) R.bands.push_back(make_band(bands[b], wtfit, n_wtfit));
    }
    ctx->relmat = std::move(R);
    IRS_API_END
}

int irs_vpw_band_xsec(irs_ctx* ctx, const double* grid, int64_t n_nu, const double* poles, const double* amps,
                      int64_t n_poles, double f, double cutoff, double x_far, double* sigma) {
    IRS_API_BEGIN
    IRS_REQUIRE(ctx && grid && sigma && n_nu >= 1 && n_poles >= 0 && (n_poles == 0 || (poles && amps)),
                "invalid arguments");
    IRS_REQUIRE(cutoff > 0.0, "cutoff must be positive");
    IRS_CUDA(cudaSetDevice(ctx->device));
    RelmatPlan rp;
    const double pre = f * kInvSqrtPi;
    for (int64_t k = 0; k < n_poles; ++k)  // compute_vpw_band_xsec, line_mixing.jl:972-1020
        rp.poles.push_back({poles[2 * k], f, poles[2 * k + 1] * f, amps[2 * k] * pre, amps[2 * k + 1] * pre, 0, 0});
    std::stable_sort(rp.poles.begin(), rp.poles.end(), [](const LmPole& a, const LmPole& b) { return a.c < b.c; });
    rp.off = {0, (long long)rp.poles.size()};
    double* d_grid = (double*)workspace(ctx, "lm_grid", n_nu * sizeof(double));
    IRS_CUDA(cudaMemcpyAsync(d_grid, grid, n_nu * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    long long ps = 0;
    const double* d_out = relmat_launch(ctx, rp, d_grid, n_nu, cutoff, x_far, ps);
    IRS_CUDA(cudaMemcpyAsync(sigma, d_out, n_nu * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    IRS_CUDA(cudaStreamSynchronize(ctx->stream));
    IRS_API_END
}

int irs_lm_perturbation(irs_ctx* ctx, int mode, const double* grid, int64_t n_nu, double T, double p_atm,
                        double cutoff, double x_far, double keep_threshold, uint32_t isotope_mask, double* dsigma) {
    IRS_API_BEGIN
    IRS_REQUIRE(ctx && grid && dsigma && n_nu >= 1, "invalid arguments");
    IRS_REQUIRE(mode == IRS_LM_RELMAT_VPY || mode == IRS_LM_RELMAT_VPW, "mode must be IRS_LM_RELMAT_VPY or _VPW");
    IRS_REQUIRE(T > 0.0 && p_atm >= 0.0 && cutoff > 0.0, "T must be positive, p_atm non-negative, cutoff positive");
    IRS_REQUIRE(ctx->relmat.species != 0, "no relaxation-matrix data uploaded (irs_upload_relmat)");
    IRS_CUDA(cudaSetDevice(ctx->device));
    RelmatPlan rp;
    lm_poles(ctx->relmat, ctx->tables, mode, isotope_mask, T, p_atm, keep_threshold, rp.poles);
    rp.off = {0, (long long)rp.poles.size()};
    double* d_grid = (double*)workspace(ctx, "lm_grid", n_nu * sizeof(double));
    IRS_CUDA(cudaMemcpyAsync(d_grid, grid, n_nu * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    long long ps = 0;
    const double* d_out = relmat_launch(ctx, rp, d_grid, n_nu, cutoff, x_far, ps);
    IRS_CUDA(cudaMemcpyAsync(dsigma, d_out, n_nu * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    IRS_CUDA(cudaStreamSynchronize(ctx->stream));
    IRS_API_END
}

int irs_synchronize(irs_ctx* ctx) {
    IRS_API_BEGIN
    IRS_REQUIRE(ctx, "ctx is NULL");
    IRS_CUDA(cudaSetDevice(ctx->device));
    IRS_CUDA(cudaStreamSynchronize(ctx->stream));
    collect_times(ctx);
    IRS_API_END
}

int irs_last_stage_times(irs_ctx* ctx, irs_stage_times* out) {
    IRS_API_BEGIN
    IRS_REQUIRE(ctx && out, "invalid arguments");
    *out = ctx->last;
    IRS_API_END
}

int irs_state_size(const irs_state_spec* spec, int n_lev, int64_t* n_state) {
    IRS_API_BEGIN
    IRS_REQUIRE(spec && n_state && n_lev >= 2, "invalid arguments");
    *n_state = state_size(*spec, n_lev);
    IRS_API_END
}

int irs_jacobian_batch(irs_ctx* ctx, const irs_profile* profs, int n_prof, const irs_sounder* s,
                       const irs_fm_options* o, const irs_state_spec* spec, double* K, double* y) {
    IRS_API_BEGIN
    IRS_REQUIRE(ctx && s && o && spec && K && y, "invalid arguments");
    IRS_CUDA(cudaSetDevice(ctx->device));
    jacobian_device(ctx, profs, n_prof, *s, *o, *spec, K, y);
    IRS_API_END
}

int irs_vjp_batch(irs_ctx* ctx, const irs_profile* profs, int n_prof, const irs_sounder* s,
                  const irs_fm_options* o, const irs_state_spec* spec, const double* dy, double* dx,
                  double* y) {
    IRS_API_BEGIN
    IRS_REQUIRE(ctx && s && o && spec && dy && dx && y && profs && n_prof >= 1, "invalid arguments");
    IRS_CUDA(cudaSetDevice(ctx->device));
    IRS_REQUIRE(state_size(*spec, profs[0].n_lev) * sizeof(double) <= 48 * 1024, "state vector too long for the adjoint");
    jacobian_device(ctx, profs, n_prof, *s, *o, *spec, nullptr, y, nullptr, dy, dx);
    IRS_API_END
}

int irs_oe_batch(irs_ctx* ctx, const irs_profile* base, int n_scene, const irs_sounder* s, const irs_fm_options* o,
                 const irs_state_spec* spec, const double* y_obs, const double* se_inv, const double* xa,
                 const double* Sa_inv, const double* x0, const irs_oe_params* prm, double* x_out, double* y_fit,
                 double* M_out, int32_t* n_iter, int32_t* converged, double* cost) {
    IRS_API_BEGIN
    IRS_REQUIRE(ctx && base && s && o && spec && y_obs && se_inv && xa && Sa_inv && x0 && prm && x_out && y_fit &&
                    M_out && n_iter && converged && cost,
                "invalid arguments");
    IRS_CUDA(cudaSetDevice(ctx->device));
    oe_batch(ctx, base, n_scene, *s, *o, *spec, y_obs, se_inv, xa, Sa_inv, x0, *prm, x_out, y_fit, M_out, n_iter,
             converged, cost);
    IRS_API_END
}

int irs_oe_batch_banded(irs_ctx* ctx, const irs_profile* base, int n_scene, const irs_sounder* s,
                        const irs_fm_options* o, const irs_state_spec* spec, const double* y_obs,
                        const double* se_band, int bw, const uint8_t* keep, const double* xa, const double* Sa_inv,
                        const double* x0, const irs_oe_params* prm, double* x_out, double* y_fit, double* M_out,
                        int32_t* n_iter, int32_t* converged, double* cost) {
    IRS_API_BEGIN
    IRS_REQUIRE(ctx && base && s && o && spec && y_obs && se_band && keep && xa && Sa_inv && x0 && prm && x_out &&
                    y_fit && M_out && n_iter && converged && cost,
                "invalid arguments");
    IRS_CUDA(cudaSetDevice(ctx->device));
    SeBand b;
    b.band = se_band;
    b.bw = bw;
    b.keep = keep;
    oe_batch(ctx, base, n_scene, *s, *o, *spec, y_obs, nullptr, xa, Sa_inv, x0, *prm, x_out, y_fit, M_out, n_iter,
             converged, cost, b);
    IRS_API_END
}

// ------------------------------------------------------------ operators
// device copies of caller arrays for the operator entry points (grown as needed)
static double* dev_copy(irs_ctx* ctx, const std::string& name, const double* h, int64_t n) {
    double* d = (double*)workspace(ctx, name, (size_t)std::max<int64_t>(n, 1) * sizeof(double));
    if (n > 0) IRS_CUDA(cudaMemcpyAsync(d, h, (size_t)n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    return d;
}
static void to_host(irs_ctx* ctx, double* h, const double* d, int64_t n) {
    if (n > 0) IRS_CUDA(cudaMemcpyAsync(h, d, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    IRS_CUDA(cudaStreamSynchronize(ctx->stream));
}

int irs_voigt_profile(irs_ctx* ctx, const double* nu, int64_t n, double nu0, double gamma_l, double gamma_d,
                      int method, double* out) {
    IRS_API_BEGIN
    IRS_REQUIRE(ctx && nu && out && n >= 0, "invalid arguments");
    IRS_REQUIRE(method >= 1 && method <= 3, "method must be 1 (Weideman), 2 (PseudoVoigt) or 3 (FullFaddeeva)");
    IRS_REQUIRE(gamma_d > 0.0 && gamma_l >= 0.0, "gamma_D must be positive and gamma_L non-negative");
    IRS_CUDA(cudaSetDevice(ctx->device));
    if (n == 0) return IRS_OK;
    double* d_in = dev_copy(ctx, "op_a", nu, n);
    double* d_out = (double*)workspace(ctx, "op_out", (size_t)n * sizeof(double));
    voigt_profile_kernel<<<(unsigned)((n + 255) / 256), 256, 0, ctx->stream>>>(d_in, n, nu0, gamma_l, gamma_d, method,
                                                                              d_out);
    check_launch(ctx);
    to_host(ctx, out, d_out, n);
    IRS_API_END
}

int irs_faddeeva(irs_ctx* ctx, const double* x, const double* y, int64_t n, double* re, double* im) {
    IRS_API_BEGIN
    IRS_REQUIRE(ctx && x && y && re && im && n >= 0, "invalid arguments");
    IRS_CUDA(cudaSetDevice(ctx->device));
    if (n == 0) return IRS_OK;
    for (int64_t i = 0; i < n; ++i) IRS_REQUIRE(y[i] >= 0.0, "w(x + iy) is evaluated for y >= 0");
    double* d_x = dev_copy(ctx, "op_a", x, n);
    double* d_y = dev_copy(ctx, "op_b", y, n);
    double* d_o = (double*)workspace(ctx, "op_out", 2 * (size_t)n * sizeof(double));
    faddeeva_kernel<<<(unsigned)((n + 255) / 256), 256, 0, ctx->stream>>>(d_x, d_y, n, d_o, d_o + n);
    check_launch(ctx);
    to_host(ctx, re, d_o, n);
    to_host(ctx, im, d_o + n, n);
    IRS_API_END
}

int irs_faddeeva32(irs_ctx* ctx, const double* x, const double* y, int64_t n, double* re, double* im) {
    IRS_API_BEGIN
    IRS_REQUIRE(ctx && x && y && re && im && n >= 0, "invalid arguments");
    IRS_CUDA(cudaSetDevice(ctx->device));
    if (n == 0) return IRS_OK;
    for (int64_t i = 0; i < n; ++i) IRS_REQUIRE(y[i] >= 0.0, "w(x + iy) is evaluated for y >= 0");
    double* d_x = dev_copy(ctx, "op_a", x, n);
    double* d_y = dev_copy(ctx, "op_b", y, n);
    double* d_o = (double*)workspace(ctx, "op_out", 2 * (size_t)n * sizeof(double));
    faddeeva32_kernel<<<(unsigned)((n + 255) / 256), 256, 0, ctx->stream>>>(d_x, d_y, n, d_o, d_o + n);
    check_launch(ctx);
    to_host(ctx, re, d_o, n);
    to_host(ctx, im, d_o + n, n);
    IRS_API_END
}

int irs_ils_kernel(irs_ctx* ctx, double dnu, double opd_max, double fwhm_gauss, int apodization, int64_t n_taps,
                   double* kern) {
    IRS_API_BEGIN
    IRS_REQUIRE(ctx && kern && dnu > 0.0 && opd_max > 0.0, "invalid arguments");
    IRS_REQUIRE(apodization >= 0 && apodization <= 3, "unknown apodization");
    const int64_t n_half = (int64_t)std::ceil(16.0 / dnu);
    IRS_REQUIRE(n_taps == 2 * n_half + 1, "n_taps must be 2 ceil(16/dnu) + 1");
    IRS_CUDA(cudaSetDevice(ctx->device));
    double* d_k = (double*)workspace(ctx, "op_out", (size_t)n_taps * sizeof(double));
    ils_taps_kernel<<<(unsigned)((n_taps + 127) / 128), 128, 0, ctx->stream>>>(dnu, opd_max, fwhm_gauss, apodization,
                                                                               n_half, d_k);
    check_launch(ctx);
    ils_normalise_kernel<<<1, 1024, 0, ctx->stream>>>(d_k, n_taps, dnu);
    check_launch(ctx);
    to_host(ctx, kern, d_k, n_taps);
    IRS_API_END
}

int irs_apply_ils(irs_ctx* ctx, const double* spectrum, int64_t n_nu, double dnu, const double* kern, int64_t n_taps,
                  double* out) {
    IRS_API_BEGIN
    IRS_REQUIRE(ctx && spectrum && kern && out && n_nu >= 0 && n_taps >= 1 && (n_taps % 2) == 1,
                "invalid arguments (the kernel needs an odd number of taps)");
    IRS_CUDA(cudaSetDevice(ctx->device));
    if (n_nu == 0) return IRS_OK;
    double* d_s = dev_copy(ctx, "op_a", spectrum, n_nu);
    double* d_k = dev_copy(ctx, "op_b", kern, n_taps);
    double* d_o = (double*)workspace(ctx, "op_out", (size_t)n_nu * sizeof(double));
    apply_ils_kernel<<<(unsigned)((n_nu + kIlsThreads - 1) / kIlsThreads), kIlsThreads, 0, ctx->stream>>>(
        d_s, n_nu, d_k, n_taps, dnu, d_o);
    check_launch(ctx);
    to_host(ctx, out, d_o, n_nu);
    IRS_API_END
}

int irs_schwarzschild_rte(irs_ctx* ctx, const double* grid, int64_t n_nu, int n_layers, const double* tau,
                          const double* T_lev, double T_sfc, double mu, double eps, int source_function,
                          const double* T_ave, double* I) {
    IRS_API_BEGIN
    IRS_REQUIRE(ctx && grid && tau && T_lev && I && n_nu >= 1 && n_layers >= 1, "invalid arguments");
    IRS_REQUIRE(mu > 0.0 && mu <= 1.0, "μ must be in (0, 1]");
    IRS_REQUIRE(source_function == 0 || source_function == 1, "source_function must be :toon or :cim");
    IRS_REQUIRE(source_function == 1 || T_ave, ":cim source_function requires T_ave");
    IRS_CUDA(cudaSetDevice(ctx->device));
    std::vector<LayerRT> lrt(n_layers);
    for (int k = 0; k < n_layers; ++k) {
        LayerRT& r = lrt[k];
        r = LayerRT{};
        r.T_bot = T_lev[k];
        r.T_top = T_lev[k + 1];
        r.T_ave = T_ave ? T_ave[k] : 0.5 * (T_lev[k] + T_lev[k + 1]);
    }
    std::vector<ProfileRT> prt(1);
    prt[0].T_sfc = T_sfc;
    prt[0].mu = mu;
    prt[0].eps = eps;
    double* d_grid = dev_copy(ctx, "op_a", grid, n_nu);
    double* d_tau = dev_copy(ctx, "op_b", tau, n_nu * n_layers);
    LayerRT* d_lrt = upload(ctx, "op_lrt", lrt);
    ProfileRT* d_prt = upload(ctx, "op_prt", prt);
    double* d_I = (double*)workspace(ctx, "op_out", (size_t)n_nu * sizeof(double));
    ContDev cd{};
    cd.mask = 0;
    rte_kernel<double><<<dim3((unsigned)((n_nu + 255) / 256), 1), 256, 0, ctx->stream>>>(
        d_tau, d_lrt, d_prt, n_layers, d_grid, n_nu, source_function, cd, d_I);
    check_launch(ctx);
    to_host(ctx, I, d_I, n_nu);
    IRS_API_END
}

int irs_grid_size(const irs_sounder* s, const irs_fm_options* o, int64_t* n_nu, int64_t* n_ch) {
    IRS_API_BEGIN
    IRS_REQUIRE(s && o && n_nu && n_ch, "invalid arguments");
    *n_nu = internal_grid(*s, *o).g.n;
    *n_ch = make_grid(s->nu_min, s->nu_max, s->dnu).n;
    IRS_API_END
}

}  // extern "C"
