/*
 * irs_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain C++ FP64 restatement of IRSounderLBL.jl's line-by-line forward path,
 * used as the parity oracle by tests/, by __graft_entry__.smoke() and by the CPU
 * baseline leg of bench.py.  Nothing in the product library links or calls it.
 *
 * Every function cites the reference file:line it follows (paths are relative to
 * the IRSounderLBL.jl project root).  The reference is Julia and cannot run in
 * this image, so parity of this restatement is pinned by:
 *   - the known-answer tests of test/runtests.jl (tests/test_oracle_pins.py);
 *   - scipy.special.wofz, which implements the same Faddeeva function that the
 *     reference reaches through SpecialFunctions.jl 2.7.2 -> OpenSpecFun_jll 0.5.6
 *     (tests/golden/make_golden.py writes the fixtures).
 */
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* HITRANLine, isbits layout of src/HITRAN/linelist.jl:20-31 (56 bytes). */
typedef struct {
    int8_t  mol_id;
    int8_t  iso_id;
    uint8_t _pad[6];
    double  wavenumber;      /* cm^-1 */
    double  intensity;       /* cm^-1/(molec cm^-2) at 296 K */
    double  a_coeff;         /* s^-1 (unused on this path) */
    float   air_broad;       /* cm^-1/atm */
    float   self_broad;      /* cm^-1/atm */
    double  lower_energy;    /* cm^-1 */
    float   temp_depend;     /* n_air */
    float   pressure_shift;  /* cm^-1/atm */
} orc_line;

/* Sounder, src/Sensor/sounder.jl:33-40. */
typedef struct {
    double nu_min, nu_max, dnu;
    int64_t n_channels;
    double opd_max, fwhm_gauss;
} orc_sounder;

/* forward_model keyword arguments, src/Sensor/sounder.jl:233-252.
 * Enumerations: apodization 0 gaussian, 1/2/3 Norton-Beer weak/medium/strong;
 * T_method 0 :logp_at_pcg, 1 :mass_weighted; source_function 0 :cim, 1 :toon;
 * line_mixing 0 none, 1 first-order VP_Y with per-line Y(T) = y0 (296/T)^0.75;
 * method 1 Weideman, 2 PseudoVoigt, 3 FullFaddeeva (forward_model always uses 3);
 * continua bit mask: 1 h2o, 2 co2, 4 co2_cia, 8 n2, 16 o2. */
typedef struct {
    double internal_dnu;      /* <= 0: use high_res_factor (or 4) */
    int32_t high_res_factor;  /* > 0 overrides internal_dnu */
    int32_t apply_continuum;
    int32_t continua;
    int32_t with_ils;
    int32_t apodization;
    int32_t line_mixing;
    int32_t T_method;
    int32_t source_function;
    int32_t method;
    int32_t _pad;
    double cutoff, lm_cutoff, dptmn, x_far;
    double mu, eps_sfc, T_sfc; /* T_sfc NaN -> temperature[1] */
} orc_fm_options;

/* tables (the reference loads these from data/ and src/HITRAN/tips2024_data.jl) */
void orc_clear_tables(void);
int  orc_set_tips(int mol, int iso, int tmin, int n, const double* q);
int  orc_set_ckd_h2o(int n, const double* nu, const double* cs, const double* cf, const double* texp);
int  orc_set_ckd_co2(int n, const double* nu, const double* s, const double* xfac, const double* tdep);

/* scalar physics */
void   orc_faddeeva(double x, double y, double* re, double* im);
double orc_weideman_voigt(double x, double y);
float  orc_weideman_voigt32(float x, float y);
double orc_pseudo_voigt_profile(double nu, double nu0, double gl, double gd);
/* voigt.jl:189-200 (normalised profile, cm) */
double orc_voigt_profile(double nu, double nu0, double gl, double gd, int method);
double orc_Q_ratio(int mol, int iso, double T);
double orc_partition_function(int mol, int iso, double T);
void   orc_line_params(const orc_line* l, double T, double p_atm, double vmr_self,
                       double* nu_shifted, double* S, double* gl, double* gd);
double orc_planck(double nu, double T);
double orc_bt(double nu, double R);
double orc_dB_dT(double nu, double T);
double orc_cim_correction(double s);
double orc_lit_correction(double s);
void   orc_layer_cg(double v1, double v2, double p1, double p2, double* vmr_cg, double* p_cg);
double orc_cg_temperature_mass(double T1, double T2, double p1, double p2);
double orc_scan_angle_to_local_zenith(double scan_deg);

/* operators */
int64_t orc_internal_grid(const orc_sounder* s, const orc_fm_options* o,
                          double* nu0, double* dnu_hi, int64_t* den);
void orc_grid_values(double nu_start, double dnu_hi, int64_t den, int64_t i0, int64_t n, double* out);
int orc_voigt_xsec(const orc_line* lines, int64_t n_lines, const double* grid, int64_t n_nu,
                   double T, double p_atm, double vmr_self, double cutoff, int method,
                   double x_far, double* sigma);
int64_t orc_reject_weak_lines(const orc_line* lines, int64_t n_lines, double T, double p_atm,
                              double coef, double vmr_self, double dptmn, uint8_t* keep);
int orc_lm_dispersive(const orc_line* lines, int64_t n_lines, const double* y0,
                      const double* grid, int64_t n_nu, double T, double p_atm,
                      double cutoff, double x_far, double* dsigma);
int orc_ils_kernel(double dnu, double opd_max, double fwhm, int apodization, int64_t n_taps,
                   double* kern);
int orc_rte(const double* grid, int64_t n_nu, int n_layers, const double* tau /* [layer][nu] */,
            const double* T_lev, double T_sfc, double mu, double eps, int source_function,
            const double* T_ave, double* I);

/* forward_model over channels [ch_begin, ch_end) (the whole sounder when ch_end <= 0).
 * prof_vmr is [n_prof_species][n_lev]; line lists are concatenated with offsets.
 * y0 (per line, may be NULL) carries the VP_Y first-order coefficients.
 * tau_out (may be NULL) receives the layer optical depths [layer][window nu]. */
int orc_forward_model(int n_lev, const double* p_lev, const double* T_lev,
                      int n_prof_species, const int* prof_species, const double* prof_vmr,
                      int n_lists, const int* list_species, const int64_t* list_offsets,
                      const orc_line* lines, const double* y0,
                      const orc_sounder* s, const orc_fm_options* o,
                      int64_t ch_begin, int64_t ch_end,
                      double* R_out, double* BT_out, double* tau_out, int64_t* n_nu_window);

/* Relaxation-matrix line mixing (line_mixing 2 VPYLineMixing, 3 VPWLineMixing,
 * line_mixing.jl:208-241): the perturbation of `species` at a layer's (T, p_atm) on the
 * window grid comes from `cb` (the numpy restatement in lm_oracle.py); the species'
 * cross section is then max(sigma_Voigt + dsigma, 0).  cb = NULL clears it. */
typedef int (*orc_lm_cb)(void* user, double T, double p_atm, const double* grid, int64_t n_nu,
                         double* dsigma);
int orc_set_lm_callback(int species, orc_lm_cb cb, void* user);

/* HITRAN CIA table of a pair (1 CO2-CO2, 2 N2-N2, 3 O2-O2; continuum.jl:104-160):
 * n_blocks blocks, block b at temperature T[b] with knots nu/sg[off[b] .. off[b+1])
 * in ascending nu, sigma already clamped at 0.  n_blocks = 0 removes it. */
int orc_set_cia(int pair, int n_blocks, const double* T, const int64_t* off, const double* nu,
                const double* sg);

int orc_num_threads(void);
const char* orc_last_error(void);

#ifdef __cplusplus
}
#endif
