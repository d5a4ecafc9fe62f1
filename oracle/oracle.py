"""ctypes wrapper of the FP64 oracle (liboracle.so) -- TEST INFRASTRUCTURE ONLY.

Imported by tests/, by ``__graft_entry__.smoke()`` and by the CPU-baseline leg of
``bench.py`` as the checker; the product library never calls it.  The C++ side
(``irs_oracle.cpp``) restates IRSounderLBL.jl's forward path with file:line
citations; this module only marshals numpy arrays and reads the bundled tables.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
DATA = HERE.parent / "irsounderlbl.jl_b200" / "data"

# HITRANLine isbits layout (src/HITRAN/linelist.jl:20-31), 56 bytes.
LINE_DTYPE = np.dtype({
    "names": ["mol_id", "iso_id", "wavenumber", "intensity", "a_coeff", "air_broad",
              "self_broad", "lower_energy", "temp_depend", "pressure_shift"],
    "formats": ["i1", "i1", "f8", "f8", "f8", "f4", "f4", "f8", "f4", "f4"],
    "offsets": [0, 1, 8, 16, 24, 32, 36, 40, 48, 52],
    "itemsize": 56,
})

APODIZATION = {"gaussian": 0, "norton_beer_weak": 1, "norton_beer_medium": 2,
               "norton_beer_strong": 3}
METHOD = {"Weideman": 1, "PseudoVoigt": 2, "FullFaddeeva": 3}
CONTINUA = {"h2o": 1, "co2": 2, "co2_cia": 4, "n2": 8, "o2": 16}


class Sounder(C.Structure):
    _fields_ = [("nu_min", C.c_double), ("nu_max", C.c_double), ("dnu", C.c_double),
                ("n_channels", C.c_int64), ("opd_max", C.c_double), ("fwhm_gauss", C.c_double)]


class FMOptions(C.Structure):
    _fields_ = [("internal_dnu", C.c_double), ("high_res_factor", C.c_int32),
                ("apply_continuum", C.c_int32), ("continua", C.c_int32),
                ("with_ils", C.c_int32), ("apodization", C.c_int32),
                ("line_mixing", C.c_int32), ("T_method", C.c_int32),
                ("source_function", C.c_int32), ("method", C.c_int32), ("_pad", C.c_int32),
                ("cutoff", C.c_double), ("lm_cutoff", C.c_double), ("dptmn", C.c_double),
                ("x_far", C.c_double), ("mu", C.c_double), ("eps_sfc", C.c_double),
                ("T_sfc", C.c_double)]


def fm_options(internal_dnu=0.001, high_res_factor=0, cutoff=25.0, lm_cutoff=None, dptmn=1e-6,
               apply_continuum=True, continua=("h2o", "co2", "co2_cia", "n2", "o2"),
               with_ils=True, apodization="gaussian", line_mixing=False,
               T_method="logp_at_pcg", source_function="cim", method="FullFaddeeva",
               x_far=122.0, mu=1.0, eps_sfc=1.0, T_sfc=None) -> FMOptions:
    """forward_model keyword arguments (src/Sensor/sounder.jl:233-252)."""
    o = FMOptions()
    o.internal_dnu = internal_dnu if internal_dnu is not None else -1.0
    o.high_res_factor = high_res_factor or 0
    o.apply_continuum = int(bool(apply_continuum))
    o.continua = sum(CONTINUA[c] for c in continua)
    o.with_ils = int(bool(with_ils))
    o.apodization = APODIZATION[apodization]
    o.line_mixing = int(line_mixing)  # 0 none, 1 per-line y0, 2 VP_Y relmat, 3 VP_W relmat
    o.T_method = {"logp_at_pcg": 0, "mass_weighted": 1}[T_method]
    o.source_function = {"cim": 0, "toon": 1}[source_function]
    o.method = METHOD[method]
    o.cutoff = cutoff
    o.lm_cutoff = cutoff if lm_cutoff is None else lm_cutoff
    o.dptmn = dptmn
    o.x_far = x_far
    o.mu = mu
    o.eps_sfc = eps_sfc
    o.T_sfc = float("nan") if T_sfc is None else T_sfc
    return o


def sounder(nu_min, nu_max, dnu, opd_max=None, fwhm_gauss=0.0, n_channels=None) -> Sounder:
    """Sounder(; ...) keyword constructor (src/Sensor/sounder.jl:49-56)."""
    s = Sounder()
    s.nu_min, s.nu_max, s.dnu = nu_min, nu_max, dnu
    s.opd_max = 1.0 / (2.0 * dnu) if opd_max is None else opd_max
    s.fwhm_gauss = fwhm_gauss
    s.n_channels = round((nu_max - nu_min) / dnu) + 1 if n_channels is None else n_channels
    return s


def read_tips(path=DATA / "tips2024_q.csv"):
    tables = {}
    for line in open(path):
        if line.startswith("#"):
            continue
        parts = line.strip().split(",")
        tables[(int(parts[0]), int(parts[1]))] = np.array([float(v) for v in parts[2:]])
    return 70, tables


def read_csv_cols(path):
    rows = [l.strip().split(",") for l in open(path).readlines()[1:] if l.strip()]
    return np.array(rows, dtype=np.float64).T.copy()


# int (*)(void* user, double T, double p_atm, const double* grid, int64_t n, double* dsigma)
LM_CALLBACK = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_double, C.c_double, C.POINTER(C.c_double), C.c_int64,
                          C.POINTER(C.c_double))


def _lines(a):
    a = np.ascontiguousarray(a, dtype=LINE_DTYPE)
    assert a.dtype.itemsize == 56, "HITRANLine records must be 56 bytes"
    return a


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Oracle:
    """FP64 restatement of the reference forward path (see irs_oracle.cpp)."""

    def __init__(self, lib_path: Path | None = None, load_tables: bool = True):
        lib_path = Path(lib_path or HERE / "liboracle.so")
        if not lib_path.exists():
            build()
        self.lib = C.CDLL(str(lib_path))
        L = self.lib
        d, i64, i32 = C.c_double, C.c_int64, C.c_int
        pd = C.POINTER(C.c_double)
        L.orc_faddeeva.argtypes = [d, d, pd, pd]
        for name in ("orc_weideman_voigt",):
            getattr(L, name).argtypes = [d, d]
            getattr(L, name).restype = d
        L.orc_weideman_voigt32.argtypes = [C.c_float, C.c_float]
        L.orc_weideman_voigt32.restype = C.c_float
        L.orc_voigt_profile.argtypes = [d, d, d, d, i32]
        L.orc_voigt_profile.restype = d
        L.orc_pseudo_voigt_profile.argtypes = [d, d, d, d]
        L.orc_pseudo_voigt_profile.restype = d
        for name in ("orc_Q_ratio", "orc_partition_function"):
            getattr(L, name).argtypes = [i32, i32, d]
            getattr(L, name).restype = d
        for name in ("orc_planck", "orc_bt", "orc_dB_dT"):
            getattr(L, name).argtypes = [d, d]
            getattr(L, name).restype = d
        for name in ("orc_cim_correction", "orc_lit_correction", "orc_scan_angle_to_local_zenith"):
            getattr(L, name).argtypes = [d]
            getattr(L, name).restype = d
        L.orc_cg_temperature_mass.argtypes = [d, d, d, d]
        L.orc_cg_temperature_mass.restype = d
        L.orc_layer_cg.argtypes = [d, d, d, d, pd, pd]
        L.orc_line_params.argtypes = [C.c_void_p, d, d, d, pd, pd, pd, pd]
        L.orc_set_tips.argtypes = [i32, i32, i32, i32, pd]
        L.orc_set_ckd_h2o.argtypes = [i32, pd, pd, pd, pd]
        L.orc_set_ckd_co2.argtypes = [i32, pd, pd, pd, pd]
        L.orc_voigt_xsec.argtypes = [C.c_void_p, i64, pd, i64, d, d, d, d, i32, d, pd]
        L.orc_reject_weak_lines.argtypes = [C.c_void_p, i64, d, d, d, d, d, C.c_void_p]
        L.orc_reject_weak_lines.restype = i64
        L.orc_lm_dispersive.argtypes = [C.c_void_p, i64, pd, pd, i64, d, d, d, d, pd]
        L.orc_ils_kernel.argtypes = [d, d, d, i32, i64, pd]
        L.orc_rte.argtypes = [pd, i64, i32, pd, pd, d, d, d, i32, pd, pd]
        L.orc_internal_grid.argtypes = [C.POINTER(Sounder), C.POINTER(FMOptions), pd, pd,
                                        C.POINTER(C.c_int64)]
        L.orc_internal_grid.restype = i64
        L.orc_grid_values.argtypes = [d, d, i64, i64, i64, pd]
        L.orc_forward_model.argtypes = [i32, pd, pd, i32, C.c_void_p, pd, i32, C.c_void_p,
                                        C.c_void_p, C.c_void_p, C.c_void_p,
                                        C.POINTER(Sounder), C.POINTER(FMOptions), i64, i64,
                                        pd, pd, C.c_void_p, C.POINTER(C.c_int64)]
        L.orc_analytic_jacobian.argtypes = [i32, pd, pd, i32, C.c_void_p, pd, i32, C.c_void_p,
                                            C.c_void_p, C.c_void_p, C.c_void_p,
                                            C.POINTER(Sounder), C.POINTER(FMOptions), i32, C.c_void_p,
                                            i32, i32, i32, i32, i32, i32, i64, i64, pd, pd]
        L.orc_set_lm_callback.argtypes = [i32, LM_CALLBACK, C.c_void_p]
        L.orc_set_cia.argtypes = [i32, i32, pd, C.c_void_p, pd, pd]
        L.orc_last_error.restype = C.c_char_p
        if load_tables:
            self.load_tables()

    def set_cia(self, pair, blocks):
        """CIA table of a pair (1 CO2-CO2, 2 N2-N2, 3 O2-O2): [(T, nu[], sigma[])], or None."""
        blocks = blocks or []
        T = np.array([b[0] for b in blocks], dtype=np.float64)
        off = np.zeros(len(blocks) + 1, dtype=np.int64)
        off[1:] = np.cumsum([len(b[1]) for b in blocks])
        nu = np.ascontiguousarray(np.concatenate([b[1] for b in blocks]) if blocks else np.zeros(1))
        sg = np.ascontiguousarray(np.concatenate([b[2] for b in blocks]) if blocks else np.zeros(1))
        self._check(self.lib.orc_set_cia(pair, len(blocks), _dp(T if len(T) else np.zeros(1)), off.ctypes.data,
                                         _dp(nu), _dp(sg)))

    # -- tables -------------------------------------------------------------
    def load_tables(self, h2o=True, co2=True):
        self.lib.orc_clear_tables()
        tmin, tips = read_tips()
        for (mol, iso), q in tips.items():
            q = np.ascontiguousarray(q)
            self.lib.orc_set_tips(mol, iso, tmin, len(q), _dp(q))
        if h2o:
            nu, cs, cf, te = read_csv_cols(DATA / "mt_ckd43_h2o_coeffs.csv")
            self.lib.orc_set_ckd_h2o(len(nu), _dp(nu), _dp(cs), _dp(cf), _dp(te))
        if co2:
            nu, s, xf, td = read_csv_cols(DATA / "mt_ckd_co2_coeffs.csv")
            self.lib.orc_set_ckd_co2(len(nu), _dp(nu), _dp(s), _dp(xf), _dp(td))

    def _check(self, rc):
        if rc != 0:
            raise RuntimeError(self.lib.orc_last_error().decode())

    # -- scalars ------------------------------------------------------------
    def faddeeva(self, x, y):
        x = np.atleast_1d(np.asarray(x, dtype=np.float64))
        y = np.broadcast_to(np.asarray(y, dtype=np.float64), x.shape)
        re, im = C.c_double(), C.c_double()
        out = np.empty(x.shape, dtype=np.complex128)
        for k, (a, b) in enumerate(zip(x.ravel(), y.ravel())):
            self.lib.orc_faddeeva(a, b, C.byref(re), C.byref(im))
            out.ravel()[k] = complex(re.value, im.value)
        return out

    def line_params(self, line, T, p_atm, vmr_self=0.0):
        rec = np.asarray(line, dtype=LINE_DTYPE).reshape(1).copy()
        o = [C.c_double() for _ in range(4)]
        self.lib.orc_line_params(rec.ctypes.data, T, p_atm, vmr_self, *[C.byref(v) for v in o])
        return tuple(v.value for v in o)

    # -- operators ------------------------------------------------------------
    def voigt_xsec(self, lines, grid, T, p_atm, vmr_self=0.0, cutoff=25.0, method="FullFaddeeva",
                   x_far=122.0):
        """compute_voigt_cross_sections (src/CrossSections/voigt.jl:375-462)."""
        lines = _lines(lines)
        grid = np.ascontiguousarray(grid, dtype=np.float64)
        out = np.empty(len(grid))
        self._check(self.lib.orc_voigt_xsec(lines.ctypes.data, len(lines), _dp(grid), len(grid),
                                            T, p_atm, vmr_self, cutoff, METHOD[method], x_far,
                                            _dp(out)))
        return out

    def reject_weak_lines(self, lines, T, p_atm, coef, vmr_self=0.0, dptmn=1e-6):
        lines = _lines(lines)
        keep = np.zeros(len(lines), dtype=np.uint8)
        self.lib.orc_reject_weak_lines(lines.ctypes.data, len(lines), T, p_atm, coef, vmr_self,
                                       dptmn, keep.ctypes.data)
        return keep.astype(bool)

    def lm_dispersive(self, lines, y0, grid, T, p_atm, cutoff=25.0, x_far=122.0):
        lines = _lines(lines)
        y0 = np.ascontiguousarray(y0, dtype=np.float64)
        grid = np.ascontiguousarray(grid, dtype=np.float64)
        out = np.empty(len(grid))
        self._check(self.lib.orc_lm_dispersive(lines.ctypes.data, len(lines), _dp(y0), _dp(grid),
                                               len(grid), T, p_atm, cutoff, x_far, _dp(out)))
        return out

    def ils_kernel(self, dnu, opd_max, fwhm, apodization="gaussian"):
        import math
        n_half = math.ceil(16.0 / dnu)
        out = np.empty(2 * n_half + 1)
        self._check(self.lib.orc_ils_kernel(dnu, opd_max, fwhm, APODIZATION[apodization],
                                            len(out), _dp(out)))
        return np.arange(-n_half, n_half + 1) * dnu, out

    def rte(self, grid, tau, T_lev, T_sfc, mu=1.0, eps=1.0, source_function="toon", T_ave=None):
        grid = np.ascontiguousarray(grid, dtype=np.float64)
        tau = np.ascontiguousarray(tau, dtype=np.float64)  # [layer][nu]
        T_lev = np.ascontiguousarray(T_lev, dtype=np.float64)
        src = {"cim": 0, "toon": 1}[source_function]
        ta = None if T_ave is None else np.ascontiguousarray(T_ave, dtype=np.float64)
        out = np.empty(len(grid))
        self._check(self.lib.orc_rte(_dp(grid), len(grid), tau.shape[0], _dp(tau), _dp(T_lev),
                                     T_sfc, mu, eps, src,
                                     _dp(ta) if ta is not None else None, _dp(out)))
        return out

    def internal_grid(self, snd: Sounder, opt: FMOptions):
        nu0, dhi, den = C.c_double(), C.c_double(), C.c_int64()
        n = self.lib.orc_internal_grid(C.byref(snd), C.byref(opt), C.byref(nu0), C.byref(dhi),
                                       C.byref(den))
        vals = np.empty(n)
        self.lib.orc_grid_values(nu0.value, dhi.value, den.value, 0, n, _dp(vals))
        return vals, dhi.value

    def forward_model(self, profile, linelists, snd: Sounder, opt: FMOptions, channels=None,
                      y0=None, return_tau=False, lm=None):
        """forward_model (src/Sensor/sounder.jl:233-360) on channels [c0, c1).

        profile: dict(p=[n_lev], T=[n_lev], vmr={mol: [n_lev]}); linelists: {mol: lines};
        y0: {mol: per-line VP_Y coefficient} (line mixing on the CO2 list);
        lm: (species, fn) with fn(T, p_atm, grid) -> the relmat line-mixing perturbation
        (opt.line_mixing 2 or 3)."""
        if lm is not None:
            species, fn = lm

            def cb(user, T, p_atm, g, n, out):
                try:
                    grid = np.ctypeslib.as_array(g, shape=(n,)).copy()
                    np.ctypeslib.as_array(out, shape=(n,))[:] = fn(T, p_atm, grid)
                    return 0
                except Exception:  # reported as a failed call
                    return -1
            ccb = LM_CALLBACK(cb)
            self.lib.orc_set_lm_callback(int(species), ccb, None)
            try:
                return self.forward_model(profile, linelists, snd, opt, channels, y0, return_tau)
            finally:
                self.lib.orc_set_lm_callback(0, LM_CALLBACK(), None)
        p = np.ascontiguousarray(profile["p"], dtype=np.float64)
        T = np.ascontiguousarray(profile["T"], dtype=np.float64)
        psp = np.array(sorted(profile["vmr"]), dtype=np.int32)
        pv = np.ascontiguousarray(np.stack([np.asarray(profile["vmr"][s], dtype=np.float64)
                                            for s in psp]))
        lsp = np.array(sorted(linelists), dtype=np.int32)
        lists = [_lines(linelists[s]) for s in lsp]
        off = np.zeros(len(lists) + 1, dtype=np.int64)
        off[1:] = np.cumsum([len(l) for l in lists])
        lines = np.zeros(int(off[-1]), dtype=LINE_DTYPE)  # concatenate() would drop the padding
        for k, l in enumerate(lists):
            lines[off[k]:off[k + 1]] = l
        assert lines.dtype.itemsize == 56
        yy = None
        if y0 is not None:
            yy = np.zeros(len(lines))
            for k, s in enumerate(lsp):
                if s in y0:
                    yy[off[k]:off[k + 1]] = y0[s]
        c0, c1 = (0, 0) if channels is None else channels
        nch = snd.n_channels if channels is None else c1 - c0
        R = np.empty(nch)
        BT = np.empty(nch)
        nw = C.c_int64()
        tau = None
        if return_tau:
            gvals, _ = self.internal_grid(snd, opt)
            tau = np.empty((len(p) - 1) * len(gvals))  # upper bound
        self._check(self.lib.orc_forward_model(
            len(p), _dp(p), _dp(T), len(psp), psp.ctypes.data, _dp(pv), len(lsp),
            lsp.ctypes.data, off.ctypes.data, lines.ctypes.data,
            yy.ctypes.data if yy is not None else None, C.byref(snd), C.byref(opt), c0, c1,
            _dp(R), _dp(BT), tau.ctypes.data if tau is not None else None, C.byref(nw)))
        if return_tau:
            return R, BT, tau[:(len(p) - 1) * nw.value].reshape(len(p) - 1, nw.value)
        return R, BT

    # -- Jacobians -----------------------------------------------------------
    def analytic_jacobian(self, profile, linelists, snd: Sounder, opt: FMOptions, retrieved=(),
                          include_T=True, include_tsfc=True, include_eps=True, log_vmr=True,
                          vmr_coupling=True, observable="bt", channels=None, y0=None):
        """analytic_jacobian (src/Estimation/vmr_jacobian.jl:152-505) -> (K [n_ch, n_state], y).

        State layout as StateVectorSpec (state_vector.jl:253-309): [T][VMR blocks in
        `retrieved` order][T_sfc][eps]."""
        p = np.ascontiguousarray(profile["p"], dtype=np.float64)
        T = np.ascontiguousarray(profile["T"], dtype=np.float64)
        psp = np.array(sorted(profile["vmr"]), dtype=np.int32)
        pv = np.ascontiguousarray(np.stack([np.asarray(profile["vmr"][s], dtype=np.float64)
                                            for s in psp]))
        lsp = np.array(sorted(linelists), dtype=np.int32)
        lists = [_lines(linelists[s]) for s in lsp]
        off = np.zeros(len(lists) + 1, dtype=np.int64)
        off[1:] = np.cumsum([len(l) for l in lists])
        lines = np.zeros(int(off[-1]), dtype=LINE_DTYPE)
        for k, l in enumerate(lists):
            lines[off[k]:off[k + 1]] = l
        yy = None
        if y0 is not None:
            yy = np.zeros(len(lines))
            for k, s in enumerate(lsp):
                if s in y0:
                    yy[off[k]:off[k + 1]] = y0[s]
        retr = np.array(list(retrieved), dtype=np.int32)
        n_lev = len(p)
        n_state = (n_lev if include_T else 0) + n_lev * len(retr) + int(include_tsfc) + int(include_eps)
        c0, c1 = (0, 0) if channels is None else channels
        nch = snd.n_channels if channels is None else c1 - c0
        K = np.zeros((n_state, nch))
        y = np.empty(nch)
        self._check(self.lib.orc_analytic_jacobian(
            n_lev, _dp(p), _dp(T), len(psp), psp.ctypes.data, _dp(pv), len(lsp), lsp.ctypes.data,
            off.ctypes.data, lines.ctypes.data, yy.ctypes.data if yy is not None else None,
            C.byref(snd), C.byref(opt), len(retr), retr.ctypes.data if len(retr) else None,
            int(include_T), int(include_tsfc), int(include_eps), int(log_vmr), int(vmr_coupling),
            0 if observable == "bt" else 1, c0, c1, _dp(K), _dp(y)))
        return np.ascontiguousarray(K.T), y

    def fd_jacobian(self, profile, linelists, snd: Sounder, opt_kw: dict, retrieved=(),
                    include_T=True, include_tsfc=True, include_eps=True, T_sfc=None, eps_sfc=1.0,
                    steps=None, observable="bt", channels=None, y0=None, lm=None):
        """finite_difference_jacobian (src/Estimation/jacobian_fd.jl:111-165), central,
        with dptmn = 0 unless opt_kw overrides it.  Log-VMR state for retrieved species;
        lm as forward_model's (relmat line mixing)."""
        n_lev = len(profile["p"])
        base_T = np.asarray(profile["T"], dtype=np.float64)
        labels = []
        x0 = []
        if include_T:
            labels += [("T", j) for j in range(n_lev)]
            x0 += list(base_T)
        for s in retrieved:
            labels += [("v", s, j) for j in range(n_lev)]
            x0 += list(np.log(np.maximum(profile["vmr"][s], 1e-30)))
        Ts0 = base_T[0] if T_sfc is None else T_sfc
        if include_tsfc:
            labels.append(("Ts",))
            x0.append(Ts0)
        if include_eps:
            labels.append(("e",))
            x0.append(eps_sfc)
        x0 = np.array(x0)
        kw = dict(dptmn=0.0)
        kw.update(opt_kw)

        def run(x):
            T = base_T.copy()
            vmr = {s: np.asarray(v, dtype=np.float64).copy() for s, v in profile["vmr"].items()}
            Ts, es = (x[0] if include_T else base_T[0]), eps_sfc
            i = 0
            if include_T:
                T = x[:n_lev].copy()
                i = n_lev
            for s in retrieved:
                vmr[s] = np.exp(x[i:i + n_lev])
                i += n_lev
            Ts = T[0]
            if include_tsfc:
                Ts = x[i]
                i += 1
            if include_eps:
                es = x[i]
            o = fm_options(T_sfc=Ts, eps_sfc=es, **kw)
            R, BT = self.forward_model(dict(p=profile["p"], T=T, vmr=vmr), linelists, snd, o,
                                       channels=channels, y0=y0, lm=lm)
            return BT if observable == "bt" else R

        y_0 = run(x0)
        K = np.zeros((len(y_0), len(x0)))
        for i in range(len(x0)):
            h = steps[i]
            xp, xm = x0.copy(), x0.copy()
            xp[i] += h
            xm[i] -= h
            K[:, i] = (run(xp) - run(xm)) / (2 * h)
        return K, y_0, labels


def build(force: bool = False):
    """Compile liboracle.so with the Makefile beside this file."""
    so = HERE / "liboracle.so"
    if so.exists() and not force:
        return so
    subprocess.run(["make", "-C", str(HERE)] + (["-B"] if force else []), check=True,
                   stdout=subprocess.DEVNULL)
    return so


def num_threads() -> int:
    return Oracle(load_tables=False).lib.orc_num_threads()


if __name__ == "__main__":
    build(force=True)
    print("built", HERE / "liboracle.so", "threads:", num_threads(), os.cpu_count())
