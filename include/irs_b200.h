/*
 * irs_b200.h -- C ABI of libirs_b200.so, the B200 (sm_100a) line-by-line forward
 * path of IRSounderLBL.jl.
 *
 * Plain C types only (pointers, sizes, doubles), so the Julia package binds it
 * with `ccall` and Python with ctypes.  Every entry point returns an int status:
 * 0 on success, a negative IRS_E* code on failure; irs_last_error() then returns
 * a message for the calling thread (the Julia shim raises it as ErrorException,
 * which is how the reference reports errors).  All host buffers are owned by the
 * caller; the library never keeps a pointer to them after the call returns.
 *
 * Each declaration names the reference interface it replaces (paths are
 * relative to the IRSounderLBL.jl project root).
 */
#ifndef IRS_B200_H
#define IRS_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define IRS_ABI_VERSION 1

/* status codes */
#define IRS_OK            0
#define IRS_E_ARG        -1   /* invalid argument (sizes, enums, ranges)      */
#define IRS_E_CUDA       -2   /* CUDA runtime error                          */
#define IRS_E_STATE      -3   /* missing table / line list / context         */
#define IRS_E_NOMEM      -4   /* device allocation failed                    */

/* VoigtMethod, src/CrossSections/voigt.jl:32-36 */
#define IRS_WEIDEMAN      1
#define IRS_PSEUDOVOIGT   2
#define IRS_FULLFADDEEVA  3

/* arithmetic of the line sum */
#define IRS_FP64          0   /* FP64 everywhere: the plain GPU kernel                  */
#define IRS_MIXED         1   /* FP32 Faddeeva + Kahan-compensated FP32 line sum; the far
                                 wings of lines >= 640 grid points from a 256-point block
                                 are summed at 8 Chebyshev nodes and interpolated        */
#define IRS_MIXED_DIRECT  2   /* as IRS_MIXED with every (point, line) pair evaluated   */

/* HITRANLine, src/HITRAN/linelist.jl:20-31 (isbits, 56 bytes): a Julia
 * Vector{HITRANLine} is passed as pointer(ll.lines) without a copy. */
typedef struct {
    int8_t  mol_id;
    int8_t  iso_id;
    uint8_t _pad[6];
    double  wavenumber;
    double  intensity;
    double  a_coeff;
    float   air_broad;
    float   self_broad;
    double  lower_energy;
    float   temp_depend;
    float   pressure_shift;
} irs_line;

/* Sounder, src/Sensor/sounder.jl:33-40 */
typedef struct {
    double  nu_min, nu_max, dnu;
    int64_t n_channels;
    double  opd_max, fwhm_gauss;
} irs_sounder;

/* forward_model keyword arguments, src/Sensor/sounder.jl:233-252.
 * apodization: 0 :gaussian, 1/2/3 :norton_beer_weak/_medium/_strong (ils.jl:26-30)
 * T_method: 0 :logp_at_pcg, 1 :mass_weighted (layers.jl:133)
 * source_function: 0 :cim, 1 :toon (schwarzschild.jl:130)
 * line_mixing: 0 nothing, 1 VPYLineMixing with per-line Y(T) = y0 (296/T)^0.75
 *   (the y0 uploaded with the CO2 list; line_mixing.jl:1351-1369),
 *   2 VPYLineMixing(relmat) and 3 VPWLineMixing(relmat) on the relaxation-matrix
 *   data of irs_upload_relmat (line_mixing.jl:208-241, 1093-1154, 1303-1369)
 * continua: bit mask 1 :h2o, 2 :co2, 4 :co2_cia, 8 :n2, 16 :o2 (the CIA pairs use
 *   the tables of irs_set_cia and contribute zeros without them, as the reference)
 * method: VoigtMethod of the line sum (forward_model uses FullFaddeeva)
 * precision: IRS_FP64, IRS_MIXED or IRS_MIXED_DIRECT */
typedef struct {
    double  internal_dnu;      /* <= 0: use high_res_factor (or 4) */
    int32_t high_res_factor;   /* > 0 overrides internal_dnu       */
    int32_t apply_continuum;
    int32_t continua;
    int32_t with_ils;
    int32_t apodization;
    int32_t line_mixing;
    int32_t T_method;
    int32_t source_function;
    int32_t method;
    int32_t precision;
    double  cutoff, lm_cutoff, dptmn, x_far;
} irs_fm_options;

/* AtmosphericProfile (src/Atmosphere/profiles.jl:12-17) plus the per-scene
 * surface and geometry kwargs of forward_model: levels surface-first, hPa, K;
 * vmr is [n_species][n_lev] for the HITRAN molecule ids in species[]. */
typedef struct {
    int32_t       n_lev;
    int32_t       n_species;
    const double* pressure;
    const double* temperature;
    const int32_t* species;
    const double* vmr;
    double        T_sfc;       /* NaN: temperature[0] (sounder.jl:337) */
    double        mu;          /* ViewingGeometry.mu, geometry.jl:18-34 */
    double        eps_sfc;
} irs_profile;

/* per-stage device times of the last forward call, ms (CUDA events) */
typedef struct {
    double line_params_ms, line_sum_ms, rte_ms, ils_ms, total_ms;
    double pairs;              /* (grid point, line, layer) pairs inside the cutoff after DPTMIN */
    double core_pairs;         /* of which |x| <= x_far (Faddeeva evaluations) */
    double h2d_bytes;          /* host->device bytes copied by the call */
    double d2h_bytes;          /* device->host bytes copied by the call */
    double launches;           /* kernels launched by the call */
    double evaluated_pairs;    /* pair evaluations the line-sum kernel issued (IRS_MIXED:
                                  near lines x block points + far lines x nodes) */
    double lm_host_ms;         /* relaxation-matrix line mixing: host time building the poles
                                  (W(T), Y(T), eigenmodes; line_mixing 2 and 3) */
    double lm_device_ms;       /* its device pole sums (part of line_params_ms) */
} irs_stage_times;

typedef struct irs_ctx irs_ctx;

int         irs_abi_version(void);
const char* irs_last_error(void);

/* Context on one GPU: device buffers, streams, uploaded tables and line lists.
 * Not shared between host threads without external locking. */
int irs_create(int device, irs_ctx** out);
int irs_destroy(irs_ctx* ctx);

/* TIPS-2024 Q(T) table for (mol, iso) at 1 K from t_min
 * (replaces partition.jl:10-47 reading src/HITRAN/tips2024_data.jl). */
int irs_set_partition_table(irs_ctx* ctx, int mol, int iso, int t_min, int n, const double* q);

/* MT-CKD tables (replaces continuum.jl:49-99 reading data/mt_ckd_*). */
int irs_set_continuum_h2o(irs_ctx* ctx, int n, const double* nu, const double* cs,
                          const double* cf, const double* texp);
int irs_set_continuum_co2(irs_ctx* ctx, int n, const double* nu, const double* s,
                          const double* xfac, const double* tdep);

/* HITRAN CIA table of one pair (replaces continuum.jl:104-165 reading data/cia/*.cia):
 * pair 1 CO2-CO2, 2 N2-N2, 3 O2-O2; block b (file order) is at temperature T[b] with
 * knots nu/sigma[off[b] .. off[b+1]) in increasing nu (cm^-1; cm^5/molecule^2, clamped
 * at 0 as the reader does).  n_blocks = 0 removes the table; a missing table
 * contributes zeros, as in the reference. */
int irs_set_cia(irs_ctx* ctx, int pair, int n_blocks, const double* T, const int64_t* off,
                const double* nu, const double* sigma);

/* Upload the line list of one species (HITRANLinelist, linelist.jl:51-56; lines
 * sorted by wavenumber as HITRANLinelist guarantees -- unsorted input is sorted
 * here).  y0 (nullable) holds per-line first-order mixing coefficients used when
 * line_mixing = 1 (VPYLineMixing, line_mixing.jl:144-149). */
int irs_upload_linelist(irs_ctx* ctx, int species, const irs_line* lines, int64_t n,
                        const double* y0);

/* compute_voigt_cross_sections(ν_grid, linelist, T, p_atm; vmr_self, cutoff,
 * method, x_far) -- src/CrossSections/voigt.jl:375-462 -- for the uploaded list
 * of `species`, on the host grid[n_nu]; sigma[n_nu] (cm^2/molecule) is written. */
int irs_cross_sections(irs_ctx* ctx, int species, const double* grid, int64_t n_nu,
                       double T, double p_atm, double vmr_self, double cutoff, int method,
                       double x_far, int precision, double* sigma);

/* forward_model(prof, linelists; sounder, geom, T_sfc, ε_sfc, kwargs...) for a
 * batch of profiles -- src/Sensor/sounder.jl:233-360.  R and BT are host buffers
 * [n_prof][n_channels] (mW/m^2/sr/cm^-1 and K). */
int irs_forward_model_batch(irs_ctx* ctx, const irs_profile* profs, int n_prof,
                            const irs_sounder* s, const irs_fm_options* o,
                            double* R, double* BT);

/* Same as irs_forward_model_batch, but R and BT are DEVICE pointers and the call
 * returns once the work is enqueued.  The work runs on the context's stream,
 * ordered after the work already queued on `stream` (a cudaStream_t) and with
 * `stream` ordered after it.  With stream = NULL no ordering is set up: the
 * results are complete after irs_synchronize(ctx).  Used when results stay in HBM. */
int irs_forward_model_batch_device(irs_ctx* ctx, const irs_profile* profs, int n_prof,
                                   const irs_sounder* s, const irs_fm_options* o,
                                   double* R_dev, double* BT_dev, void* stream);

/* StateVectorSpec (src/Estimation/state_vector.jl:253-309) with full-profile VMR
 * blocks: state = [T (n_lev) if include_temperature][VMR or log VMR (n_lev) per
 * retrieved species, in order][T_sfc][eps].  observable: 0 :bt, 1 :radiance.
 * vmr_coupling as analytic_jacobian's keyword (vmr_jacobian.jl:152-172).
 * At most 4 retrieved species. */
typedef struct {
    int32_t        n_retrieved;
    const int32_t* retrieved;
    int32_t        include_temperature;
    int32_t        include_tsfc;
    int32_t        include_emissivity;
    int32_t        log_vmr;
    int32_t        vmr_coupling;
    int32_t        observable;
} irs_state_spec;

/* Length of the state vector for `spec` on n_lev levels. */
int irs_state_size(const irs_state_spec* spec, int n_lev, int64_t* n_state);

/* analytic_jacobian(prof, linelists, spec; sounder, geom, T_sfc, ε_sfc, observable,
 * kwargs...) -- src/Estimation/vmr_jacobian.jl:152-505 -- for a batch of profiles.
 * K is [n_prof][n_state][n_channels] (per profile the column-major Jacobian.K,
 * jacobian_fd.jl:43-50); y is [n_prof][n_channels], the observable at the
 * linearisation point.  The line set is frozen (no DPTMIN), as the reference does.
 * The line sum runs in FP32 with Kahan-compensated tile sums (o->precision is
 * ignored); transmittances and radiance derivatives are FP64. */
int irs_jacobian_batch(irs_ctx* ctx, const irs_profile* profs, int n_prof, const irs_sounder* s,
                       const irs_fm_options* o, const irs_state_spec* spec, double* K, double* y);

/* forward_model for one batch spread over n_ctx contexts (one per GPU; every context
 * must hold the same line lists and tables).  No counterpart in the reference, whose
 * profile loop is sequential (sounder.jl:283-307): the batch is split into contiguous
 * shards (irs_shard_range), each run by its own host thread through
 * irs_forward_model_batch on its context, and the shards' R and BT are written to the
 * caller's host buffers [n_prof][n_channels] at their offsets.  No collective.  A
 * context serves one host thread at a time, so each may appear once in ctxs. */
int irs_forward_model_batch_multi(irs_ctx* const* ctxs, int n_ctx, const irs_profile* profs, int n_prof,
                                  const irs_sounder* s, const irs_fm_options* o, double* R, double* BT);
/* The shard of n items that shard `shard` of n_shards takes: [*first, *first + *count),
 * contiguous and balanced (the first n % n_shards shards take one more).  Host only. */
int irs_shard_range(int64_t n, int n_shards, int shard, int64_t* first, int64_t* count);

/* Vector-Jacobian product dx = K^T dy for each profile (the pullback behind the
 * ChainRulesCore.rrule of forward_model): dy is [n_prof][n_channels], dx is
 * [n_prof][n_state]; y receives the observable.  Reverse mode on the device (the
 * reference forms K first, vmr_jacobian.jl:152-505): the derivative line sum, the
 * forward RTE, the radiance cotangent dy dBT/dR taken back through the channel
 * resampling and the ILS to the grid, and one adjoint RTE sweep
 * (schwarzschild_jacobian.jl:66-167 per grid point) that contracts every derivative term
 * with it; K is never formed.  At most 6144 state elements. */
int irs_vjp_batch(irs_ctx* ctx, const irs_profile* profs, int n_prof, const irs_sounder* s,
                  const irs_fm_options* o, const irs_state_spec* spec, const double* dy, double* dx,
                  double* y);

/* optimal_estimation keyword arguments (optimal_estimation.jl:142-156): method 0
 * :levenberg_marquardt, 1 :gauss_newton; eps_fixed = ε_fixed. */
typedef struct {
    int32_t max_iter, max_linesearch, method;
    double  gamma0, gamma_factor, gamma_min, conv_factor, eps_fixed;
} irs_oe_params;

/* optimal_estimation(y, spec, base_prof, linelists; xa, Sa, Se, x0, ...) --
 * src/Estimation/optimal_estimation.jl:142-291 -- for a batch of scenes with diagonal
 * Se (se_inv = 1/σ² per channel; 0 drops a channel, as channel_mask does).  Each scene
 * iterates on its own (LM damping, line search, convergence d²/n < conv_factor); every
 * stage is one batched GPU call over the scenes still iterating: FP64 normal equations
 * from the Jacobian, FP64 Cholesky solves, the forward model at trial states (dptmn = 0,
 * o->precision) and the analytic Jacobian at accepted states.
 * Arrays: base [n_scene]; y_obs, se_inv, y_fit [n_scene][n_channels]; xa, x0, x_out
 * [n_scene][n_state]; Sa_inv [n_state][n_state] (shared); M_out [n_scene][n_state]
 * [n_state] = K^T Se^-1 K at the solution; n_iter, converged, cost [n_scene].
 * At most 160 state elements. */
int irs_oe_batch(irs_ctx* ctx, const irs_profile* base, int n_scene, const irs_sounder* s,
                 const irs_fm_options* o, const irs_state_spec* spec, const double* y_obs,
                 const double* se_inv, const double* xa, const double* Sa_inv, const double* x0,
                 const irs_oe_params* prm, double* x_out, double* y_fit, double* M_out,
                 int32_t* n_iter, int32_t* converged, double* cost);

/* ------------------------------------------------------------------------------
 * Relaxation-matrix line mixing (src/CrossSections/line_mixing.jl).
 * ------------------------------------------------------------------------------ */
#define IRS_LM_NONE        0
#define IRS_LM_PER_LINE_Y  1   /* VP_Y with per-line y0 on the HITRAN list          */
#define IRS_LM_RELMAT_VPY  2   /* VPYLineMixing(relmat): first-order Y from W(T)    */
#define IRS_LM_RELMAT_VPW  3   /* VPWLineMixing(relmat): whitelisted bands by their
                                  eigenmodes, the other bands by VP_Y              */

/* RelmatLine (line_mixing.jl:35-47); Julia's isbits layout, 72 bytes, so a band's
 * Vector{RelmatLine} is passed as pointer(band.lines). */
typedef struct {
    int8_t  isot;
    double  nu;          /* line centre, cm^-1                 */
    int16_t ji;          /* initial J                          */
    int8_t  branch;      /* -1 P, 0 Q, +1 R                    */
    double  gv_air;      /* air HWHM at 296 K, cm^-1/atm       */
    float   n_air;
    float   shift;       /* pressure shift, cm^-1/atm          */
    double  e_lower;
    double  dipo0, popu_t0, dipo_t;
} irs_relmat_line;

/* RelmatBand (line_mixing.jl:72-82).  whitelisted: the band's name is in
 * VPWLineMixing.whitelist (default_vpw_whitelist, line_mixing.jl:813-849, is host
 * logic of the caller). */
typedef struct {
    const irs_relmat_line* lines;
    int64_t n_lines;
    double  nu_min, nu_max;
    int32_t li, lf, isot, molecule;
    int32_t whitelisted, _pad;
} irs_relmat_band;

/* One entry of a W0B0Table (line_mixing.jl:92-102, read by _load_wtfit :434-472):
 * the table of key (lli, llf) = (min(li,lf), max(li,lf)), branch pair sub = 3 t_i +
 * t_ip with t = 0 P, 1 Q, 2 R (pp, pq, ..., rr), J pair (ji, jip), W(T) = exp(w0r)
 * (T/T0)^b0r.  A later entry with the same key overwrites an earlier one. */
typedef struct {
    int32_t lli, llf, sub, ji, jip, _pad;
    double  w0r, b0r;
} irs_wtfit_entry;

/* HITRANRelmatData (line_mixing.jl:106-118) of `species` with the LM object's
 * min_band_strength: the context keeps a copy and builds each band's
 * temperature-independent coupling table (_build_coupling, :530-578) once.
 * n_bands = 0 removes it. */
int irs_upload_relmat(irs_ctx* ctx, int species, const irs_relmat_band* bands, int n_bands,
                      const irs_wtfit_entry* wtfit, int64_t n_wtfit, double min_band_strength);

/* Host-side building blocks (no device work; usable without a GPU).  q_ratio is
 * Q(296 K)/Q(T) of the band's isotopologue.  W is [n][n] row-major, W[i*n + j] the
 * reference's W[i, j]. */
int irs_relmat_w_matrix(const irs_relmat_band* band, const irs_wtfit_entry* wtfit, int64_t n_wtfit,
                        double T, double q_ratio, double* W, double* popu);      /* :607-700 */
int irs_relmat_y(const irs_relmat_band* band, const irs_wtfit_entry* wtfit, int64_t n_wtfit,
                 double T, double q_ratio, double* Y);                          /* :712-738 */
/* band_modes (:892-955): poles and amplitudes as interleaved (re, im) pairs
 * [2 n_lines]; n_kept of them are written. */
int irs_band_modes(const irs_relmat_band* band, const irs_wtfit_entry* wtfit, int64_t n_wtfit,
                   double T, double p_atm, double q_ratio, double keep_threshold,
                   double* poles, double* amps, double* f, int64_t* n_kept);

/* compute_vpw_band_xsec(ν_grid, modes; cutoff, x_far) (:972-1020) on the device:
 * grid[n_nu] sorted, poles/amps interleaved (re, im) [2 n_poles]. */
int irs_vpw_band_xsec(irs_ctx* ctx, const double* grid, int64_t n_nu, const double* poles,
                      const double* amps, int64_t n_poles, double f, double cutoff, double x_far,
                      double* sigma);

/* The line-mixing perturbation of the uploaded relmat at (T, p_atm) on grid[n_nu]:
 * mode IRS_LM_RELMAT_VPY is compute_lm_dispersive_correction (:1303-1337), mode
 * IRS_LM_RELMAT_VPW is _vpw_perturbation (:1120-1154).  isotope_mask: bit k keeps
 * isotopologue k (0 keeps all), the reference's `isotopes` filter. */
int irs_lm_perturbation(irs_ctx* ctx, int mode, const double* grid, int64_t n_nu, double T,
                        double p_atm, double cutoff, double x_far, double keep_threshold,
                        uint32_t isotope_mask, double* dsigma);

/* irs_oe_batch with a banded measurement covariance instead of a diagonal one: the
 * apodised Se of IASI L1C (apodized_measurement_covariance, covariance.jl:62-81) that
 * optimal_estimation takes as a matrix (optimal_estimation.jl:166-176).  se_band is
 * [n_scene][n_channels][bw+1] with se_band[s][i][k] = Se(i, i-k) (0 <= bw <= 32); keep
 * [n_channels] (1 keep, 0 drop, as channel_mask) restricts Se to Se[keep, keep].  The
 * library factors each scene's Se and retrieves on whitened residuals and Jacobians;
 * M_out is K^T Se^-1 K on the kept channels.  Other arguments as irs_oe_batch. */
int irs_oe_batch_banded(irs_ctx* ctx, const irs_profile* base, int n_scene, const irs_sounder* s,
                        const irs_fm_options* o, const irs_state_spec* spec, const double* y_obs,
                        const double* se_band, int bw, const uint8_t* keep, const double* xa,
                        const double* Sa_inv, const double* x0, const irs_oe_params* prm, double* x_out,
                        double* y_fit, double* M_out, int32_t* n_iter, int32_t* converged, double* cost);

/* ------------------------------------------------------------------------------
 * Array-level operators on the device, for callers that use them outside
 * forward_model.  Host arrays in and out, FP64.
 * ------------------------------------------------------------------------------ */
/* voigt_profile(ν, ν₀, γ_L, γ_D, method) over nu[n] (voigt.jl:177-200; method 1
 * Weideman, 2 PseudoVoigt, 3 FullFaddeeva), cm. */
int irs_voigt_profile(irs_ctx* ctx, const double* nu, int64_t n, double nu0, double gamma_l, double gamma_d,
                      int method, double* out);
/* w(x + iy) = erfcx(y - ix) for y >= 0 (faddeeva_voigt = Re w, voigt.jl:152-160). */
int irs_faddeeva(irs_ctx* ctx, const double* x, const double* y, int64_t n, double* re, double* im);
/* w(x + iy) by the FP32 evaluator of the mixed-precision line sums (no counterpart in
 * the reference, which evaluates FullFaddeeva in FP64 only): for checking its
 * accuracy against irs_faddeeva / erfcx.  Inputs are rounded to FP32. */
int irs_faddeeva32(irs_ctx* ctx, const double* x, const double* y, int64_t n, double* re, double* im);
/* ils_kernel(Δν, opd_max, fwhm; apodization) (ils.jl:80-115): the area-normalised taps
 * at k Δν, k = -n_half..n_half, n_taps = 2 ceil(16/Δν) + 1. */
int irs_ils_kernel(irs_ctx* ctx, double dnu, double opd_max, double fwhm_gauss, int apodization, int64_t n_taps,
                   double* kern);
/* apply_ils(ν_grid, spectrum, ils_δν, ils_kernel) (ils.jl:131-153): out[i] = Δν sum_k
 * spectrum[i + k - half] kern[k], zero outside the grid. */
int irs_apply_ils(irs_ctx* ctx, const double* spectrum, int64_t n_nu, double dnu, const double* kern,
                  int64_t n_taps, double* out);
/* schwarzschild_rte(ν_grid, τ_layers, T_levels, T_sfc; μ, ε_sfc, source_function,
 * T_ave) (schwarzschild.jl:130-274): tau is [n_layers][n_nu] (the Julia n_ν x n_layers
 * matrix in memory order), T_lev [n_layers + 1] surface first; source_function 0 :cim
 * (T_ave required), 1 :toon. */
int irs_schwarzschild_rte(irs_ctx* ctx, const double* grid, int64_t n_nu, int n_layers, const double* tau,
                          const double* T_lev, double T_sfc, double mu, double eps, int source_function,
                          const double* T_ave, double* I);

/* Wait for the context's work; fill per-stage times of the last forward call. */
int irs_synchronize(irs_ctx* ctx);
int irs_last_stage_times(irs_ctx* ctx, irs_stage_times* out);

/* No counterpart in the reference.  compute_voigt_cross_sections in FP64 for callers
 * that cannot allocate device memory (hosts whose allocator already owns the device,
 * such as a CUDA.jl memory pool, or hosts that forbid allocation after start-up):
 * it allocates nothing.  d_lines (56-byte records sorted by wavenumber), d_tips_q,
 * d_grid and d_sigma are device pointers owned by the caller; the work is queued on
 * `stream`.  d_tips_q holds n_tips TIPS tables packed one after another, each Q(T) at
 * tips_n temperatures 1 K apart from tips_t_min; tips_keys (host) gives the (mol, iso)
 * of table k at [2k], [2k + 1].  Each line takes the table of its own (mol, iso)
 * (Q_ratio, partition.jl:41-47) and Q proportional to T when none matches or d_tips_q
 * is NULL.  At most 131072 lines and 64 tables (IRS_E_ARG beyond).  Its per-line
 * scratch is one file-scope device array shared by all calls, so calls that overlap on
 * the GPU race; the first call in each CUDA context does a one-time set-up and should
 * come before any stream capture; after cudaDeviceReset reload the library. */
int irs_cross_sections_noalloc(const irs_line* d_lines, int64_t n_lines, const double* d_tips_q,
                               const int32_t* tips_keys, int n_tips, int tips_t_min, int tips_n,
                               const double* d_grid, int64_t n_nu, double T, double p_atm, double vmr_self,
                               double cutoff, int method, double x_far, double* d_sigma, void* stream);

/* ------------------------------------------------------------------------------
 * MLP surrogate of forward_model.  No counterpart in the reference: it maps a
 * profile plus scan angle (n_in floats) to channel brightness temperatures through
 * n_layers hidden GELU layers of n_hidden units, on the tcgen05 tensor cores (BF16
 * weights and activations, FP32 accumulation, FP32 master weights and Adam).  It is
 * trained on spectra of irs_forward_model_batch, and its callers fall back to that
 * path for inputs whose OOD score exceeds their threshold.  All X / Y / out buffers
 * are row-major [n][n_in] / [n][n_out] FP32; host pointers unless named _dev.
 * ------------------------------------------------------------------------------ */
typedef struct irs_surrogate irs_surrogate;

int irs_surrogate_create(irs_ctx* ctx, int n_in, int n_hidden, int n_layers, int n_out, uint64_t seed,
                         irs_surrogate** out);
int irs_surrogate_destroy(irs_surrogate* s);
/* parameters as one FP32 vector: per layer W [n_out_l][n_in_l] row-major, then b [n_out_l] */
int irs_surrogate_param_count(irs_surrogate* s, int64_t* n);
int irs_surrogate_get_params(irs_surrogate* s, float* params);
int irs_surrogate_set_params(irs_surrogate* s, const float* params);
/* input scaling x' = (x - x_mean) / x_sd, output y = y' y_sd + y_mean */
int irs_surrogate_set_scaling(irs_surrogate* s, const float* x_mean, const float* x_sd, const float* y_mean,
                              const float* y_sd);
/* OOD score of a sample = |W x'|^2 / n_in with W [n_in][n_in] the whitening matrix */
int irs_surrogate_set_whitening(irs_surrogate* s, const float* W);
/* epochs of Adam on 0.5 mean((y' - t')^2) over full mini-batches of a shuffled set, the
 * learning rate following a cosine schedule from lr down to lr / 100 */
int irs_surrogate_train(irs_surrogate* s, const float* X, const float* Y, int64_t n, int batch, int epochs,
                        float lr, uint64_t seed, double* loss_per_epoch);
/* loss and its gradient (same layout as the parameters) on one batch, no update */
int irs_surrogate_gradients(irs_surrogate* s, const float* X, const float* Y, int64_t n, float* grads,
                            double* loss);
/* Data-parallel training, split at the gradient so that it can be reduced across GPUs
 * between the halves.  irs_surrogate_grad_size: the length of the flat gradient (the
 * parameters in a padded device layout).  irs_surrogate_grad_device: the loss and
 * gradient of 0.5 mean((y' - t')^2) over rows idx_dev[0..n) (NULL: rows 0..n) of the
 * device arrays X_dev [rows][n_in], Y_dev [rows][n_out], written to g_dev (device, the
 * flat layout); loss (host, nullable) waits for the result.  irs_surrogate_apply_device:
 * one Adam step (as irs_surrogate_train's) from the gradient in g_dev with learning rate
 * lr.  Both are ordered after and before the work on `stream` (a cudaStream_t). */
int irs_surrogate_grad_size(irs_surrogate* s, int64_t* n);
int irs_surrogate_grad_device(irs_surrogate* s, const float* X_dev, const float* Y_dev, const int32_t* idx_dev,
                              int64_t n, float* g_dev, double* loss, void* stream);
int irs_surrogate_apply_device(irs_surrogate* s, const float* g_dev, float lr, void* stream);
/* predictions [n][n_out] and OOD scores [n] (ood nullable) */
int irs_surrogate_infer(irs_surrogate* s, const float* X, int64_t n, float* out, float* ood);
/* same with device buffers; ordered after and before the work on `stream` (a cudaStream_t) */
int irs_surrogate_infer_device(irs_surrogate* s, const float* X_dev, int64_t n, float* out_dev,
                               float* ood_dev, void* stream);
/* C [M][N] = A [M][K] B [N][K]^T with BF16 inputs (uint16 bit patterns), FP32 output */
int irs_gemm_bf16(irs_ctx* ctx, const uint16_t* A, const uint16_t* B, int M, int N, int K, float* C);

/* Number of internal grid points and channels forward_model uses for (s, o). */
int irs_grid_size(const irs_sounder* s, const irs_fm_options* o, int64_t* n_nu,
                  int64_t* n_channels);

#ifdef __cplusplus
}
#endif
#endif /* IRS_B200_H */
