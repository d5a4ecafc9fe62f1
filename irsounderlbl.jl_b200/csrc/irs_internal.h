// irs_internal.h -- shared declarations of libirs_b200 (not part of the C ABI).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <map>
#include <string>
#include <utility>
#include <vector>

#include "../../include/irs_b200.h"

namespace irs {

// ------------------------------------------------------------------ errors
void set_error(const std::string& msg);
struct Error {
    int code;
    std::string msg;
};
#define IRS_CUDA(call)                                                                 \
    do {                                                                               \
        cudaError_t e_ = (call);                                                       \
        if (e_ != cudaSuccess)                                                         \
            throw ::irs::Error{IRS_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)}; \
    } while (0)
#define IRS_REQUIRE(cond, msg)                                        \
    do {                                                              \
        if (!(cond)) throw ::irs::Error{IRS_E_ARG, std::string(msg)}; \
    } while (0)

// ------------------------------------------------------------------ grids
// Julia's float range a:s:b (src/Utils/wavenumber_grid.jl:23-26): start, step and
// stop are rationalised (n/den) when they have exact small-denominator forms and the
// elements are then (a_n + i s_n)/den, correctly rounded.
struct GridSpec {
    int64_t n = 0;
    int64_t den = 0;  // 0: literal start + i*step
    double a_n = 0, s_n = 0, start = 0, step = 0;
    double at(int64_t i) const { return den ? (a_n + double(i) * s_n) / double(den) : start + double(i) * step; }
};
GridSpec make_grid(double a, double b, double s);

// forward_model's internal monochromatic grid (src/Sensor/sounder.jl:155-161, 263-271)
struct InternalGrid {
    GridSpec g;
    double dnu_hi;
    int64_t hrf;
};
InternalGrid internal_grid(const irs_sounder& s, const irs_fm_options& o);

// ------------------------------------------------------------ atmosphere
// One (profile, layer, species) line-sum segment: Curtis-Godson state of the
// layer for that species (src/Sensor/sounder.jl:283-307).
struct Segment {
    double T;         // T_cg (K)
    double p_atm;     // p_cg / 1013.25
    double vmr_self;  // vmr_cg for H2O, else 0
    double coef;      // vmr_cg * dp * 2.1209e22 (molecules/cm^2)
    double margin_g;  // window margin (grid units) covering the pressure shifts
    int64_t out_off;  // first slot of this segment in the per-line parameter arrays
    int32_t list;     // line-list index in the context
    int32_t flags;    // SEG_DPTMIN | SEG_LM | SEG_RELMAT
    int32_t prof, layer;
};
// SEG_LM: per-line Y dispersive sum fused into the line sum; SEG_RELMAT: the
// relaxation-matrix perturbation of this (profile, layer) is added before the clamp.
enum { SEG_DPTMIN = 1, SEG_LM = 2, SEG_RELMAT = 4 };

// Per (profile, layer) inputs of the fused RTE/continuum kernel.
struct LayerRT {
    double T_ave;     // cg_temperature_mass (TBAR), layers.jl:93-106
    double T_top;     // T_levels[k+1]
    double T_bot;     // T_levels[k]
    double p_mid, T_mid, dz_cm;
    double vmr_h2o, vmr_co2;  // mid-layer (continua)
};
struct ProfileRT {
    double T_sfc, mu, eps;
};

// layers.jl:133-178 + sounder.jl:283-336 for one profile; appends to the vectors.
void layer_setup(const irs_profile& prof, int prof_index, const irs_fm_options& o,
                 const std::vector<int>& list_species, const std::vector<double>& list_max_shift,
                 double dnu_grid, std::vector<Segment>& segs, std::vector<LayerRT>& lrt,
                 ProfileRT& prt);

// Jacobian: schwarzschild_jacobian.jl:47-53 and the per-segment state-chain weights
double cg_mass_frac(double p1, double p2);
void jacobian_weights(const irs_profile& P, const irs_fm_options& o, int species, int layer,
                      const irs_state_spec& sp, float w[][4]);

// ------------------------------------------------------------ device data
struct DevLineList {
    int species = 0;
    int64_t n = 0;
    double max_abs_shift = 0;  // max |delta_air| + |delta_self| (cm^-1/atm)
    bool has_y0 = false;
    uint32_t iso_mask = 0;     // isotopologues present, iso 0 counted as 10 (line_mixing.jl:202-203)
    // SoA, sorted by wavenumber
    double *nu = nullptr, *S296 = nullptr, *E = nullptr, *gair = nullptr, *gself = nullptr,
           *nair = nullptr, *delta = nullptr, *y0 = nullptr;
    int* tips = nullptr;  // table index or -1
};

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
};

// Per-line parameter arrays for the line sum (one slot per (segment, line)).
struct LineParamsF64 {  // plain FP64 kernel; PseudoVoigt reuses f=gV, y=eta, Sn=S, Hc=base
    double *nu0, *f, *y, *Sn, *Hc, *YSn;
};
struct LineParamsMixed {  // FP32 kernel, grid units relative to the grid start
    double* V;            // unshifted centre (sorted key)
    double* U;            // shifted centre
    float4* p0;           // b2, a, c1, c0        (PV: gV2, aPV, c1, c0)
    float4* p1;           // dfar2, An, fx, y     (PV: kPV, gPV, -, -)
    float4* p2;           // g, Yw, dfar, - (dispersive line mixing, core reach)
};

struct Tables {
    std::map<std::pair<int, int>, std::pair<int, std::vector<double>>> tips;  // (tmin, q)
    double q_value(int mol, int iso, double T) const;  // partition.jl:8-24
    std::vector<double> h2o_nu, h2o_cs, h2o_cf, h2o_te;
    std::vector<double> co2_nu, co2_s, co2_tdep;  // S already multiplied by xfac
    // HITRAN CIA tables (CO2-CO2, N2-N2, O2-O2): per block T, knots, sigma
    struct CiaBlock {
        double T;
        std::vector<double> nu, sg;
    };
    std::vector<CiaBlock> cia[3];
};

// ---------------------------------------------- relaxation-matrix line mixing
// One band of HITRANRelmatData with its temperature-independent coupling pairs
// (BandCoupling, line_mixing.jl:65-70: CSR over the outer line i).
struct RelmatBandHost {
    std::vector<irs_relmat_line> lines;
    int li = 0, lf = 0, isot = 0, molecule = 2;
    bool whitelisted = false, has_wtfit = false;
    double nu_min = 0, nu_max = 0, eff_strength = 0;
    std::vector<int> row_ptr, col;
    std::vector<double> w0r, b0r;
};
struct RelmatHost {
    int species = 0;  // 0: no relmat uploaded
    double min_band_strength = 0;
    std::vector<RelmatBandHost> bands;
};
// A line-mixing pole: centre (cm^-1), Doppler factor f, y = Im(pole) f and the
// amplitudes (already times f/sqrt(pi)) of Re w and Im w; window 0 takes the pole
// where |nu - c| <= cutoff (VP_W), 1 where nu - cutoff <= c <= nu + cutoff (VP_Y).
struct LmPole {
    double c, f, y, ar, ai;
    int window, pad;
};
RelmatBandHost make_band(const irs_relmat_band& b, const irs_wtfit_entry* wt, int64_t n_wt);
// Poles of the whole LM perturbation at (T, p_atm), sorted by centre.
void lm_poles(const RelmatHost& R, const Tables& tabs, int mode, uint32_t iso_mask, double T,
              double p_atm, double keep_threshold, std::vector<LmPole>& out);

}  // namespace irs

struct irs_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[10] = {};
    irs::Tables tables;
    bool tips_dirty = true, cont_dirty = true;
    // device copies of tables
    double* d_tips = nullptr;  // [n_tab][331]
    int* d_tips_tmin = nullptr;
    int* d_tips_n = nullptr;
    int n_tips = 0;
    int tips_stride = 2;
    std::map<std::pair<int, int>, int> tips_index;
    double *d_h2o = nullptr, *d_co2 = nullptr;  // packed tables
    double *d_cia_blk = nullptr, *d_cia_nu = nullptr, *d_cia_sg = nullptr;
    int cia_b0[4] = {0, 0, 0, 0};
    int n_h2o = 0, n_co2 = 0;
    std::vector<irs::DevLineList> lists;
    irs::RelmatHost relmat;
    std::map<std::string, irs::DevBuf> work;  // named growable workspaces
    irs_stage_times last{};
    irs_stage_times prior{};  // stage times of the earlier passes of a multi-pass batch
    double n_h2d = 0, n_d2h = 0, n_launch = 0;  // counters of the current call
    double lm_host_pass = 0;  // host ms building relmat poles in the current pass
    bool lm_ev = false;       // ev[7], ev[8] bracket the relmat pole sums of the current pass
    // cached ILS kernel
    double ils_key[4] = {-1, -1, -1, -1};
    int64_t ils_n = 0;
    // bytes of the strip far field's node values per line-sum launch (larger batches run
    // in groups of profile-layers); IRS_STRIP_BUFFER_BYTES at context creation sets it
    size_t strip_buf_max = (size_t)2 << 30;
};

namespace irs {
void* workspace(irs_ctx* ctx, const std::string& name, size_t bytes);
void upload_tables(irs_ctx* ctx);
}
