"""irsounderlbl.jl_b200 -- the line-by-line forward path of IRSounderLBL.jl on one B200.

Host-side mirror of the reference interface (same names, argument meanings and
error behaviour as the Julia package) over the C ABI of ``libirs_b200.so``:

    compute_voigt_cross_sections   src/CrossSections/voigt.jl:375-462
    forward_model                  src/Sensor/sounder.jl:233-360
    Sounder / IASIInstrument ...   src/Sensor/sounder.jl:33-128
    ViewingGeometry, scan angles   src/Sensor/geometry.jl:18-101
    VoigtMethod                    voigt.jl:32-36
    VPYLineMixing, VPWLineMixing,  line_mixing.jl (relmat.py: data types, readers,
    relmat operators                W(T), Y(T), eigenmodes, pole sums)

Every computation runs in the CUDA library; nothing here evaluates physics
beyond argument marshalling and the scalar geometry helpers.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from enum import IntEnum
from pathlib import Path
from typing import Dict, Iterable, Optional, Sequence

import numpy as np

from . import _lib
from ._lib import (IRS_FP64, IRS_MIXED, IRS_MIXED_DIRECT, LINE_DTYPE, FMOptions, IRSError, Profile, StageTimes,
                   check, dptr)

DATA = Path(__file__).resolve().parent / "data"


class VoigtMethod(IntEnum):
    """src/CrossSections/voigt.jl:32-36"""
    Weideman = 1
    PseudoVoigt = 2
    FullFaddeeva = 3


Weideman, PseudoVoigt, FullFaddeeva = VoigtMethod.Weideman, VoigtMethod.PseudoVoigt, VoigtMethod.FullFaddeeva


class GasSpecies(IntEnum):
    """src/Atmosphere/species.jl:6-16 (values are HITRAN molecule ids)"""
    H2O = 1
    CO2 = 2
    O3 = 3
    N2O = 4
    CO = 5
    CH4 = 6
    O2 = 7
    SO2 = 9
    NH3 = 11


H2O, CO2, O3, N2O, CO, CH4 = (GasSpecies.H2O, GasSpecies.CO2, GasSpecies.O3, GasSpecies.N2O,
                              GasSpecies.CO, GasSpecies.CH4)

PRECISION = {"fp64": IRS_FP64, "mixed": IRS_MIXED, "mixed_direct": IRS_MIXED_DIRECT}
APODIZATION = {"gaussian": 0, "norton_beer_weak": 1, "norton_beer_medium": 2, "norton_beer_strong": 3}
CONTINUA = {"h2o": 1, "co2": 2, "co2_cia": 4, "n2": 8, "o2": 16}


# ------------------------------------------------------------------ types
class HITRANLinelist:
    """HITRANLinelist (src/HITRAN/linelist.jl:51-56): lines sorted by wavenumber."""

    def __init__(self, lines: np.ndarray):
        lines = np.asarray(lines)
        order = np.argsort(lines["wavenumber"], kind="stable")
        out = np.zeros(len(lines), dtype=LINE_DTYPE)  # zeroed padding, 56-byte records
        for name in LINE_DTYPE.names:
            out[name] = lines[name][order]
        self.lines = out
        self.molecules = set(int(m) for m in np.unique(self.lines["mol_id"]))
        self.nu_min = float(self.lines["wavenumber"].min()) if len(self.lines) else 0.0
        self.nu_max = float(self.lines["wavenumber"].max()) if len(self.lines) else 0.0

    def __len__(self):
        return len(self.lines)


@dataclass
class AtmosphericProfile:
    """src/Atmosphere/profiles.jl:12-17 (levels surface-first, hPa, K, km)."""
    pressure: np.ndarray
    temperature: np.ndarray
    altitude: np.ndarray
    vmr: Dict[int, np.ndarray]


@dataclass
class Sounder:
    """src/Sensor/sounder.jl:33-56"""
    nu_min: float
    nu_max: float
    dnu: float
    n_channels: int
    opd_max: float
    fwhm_gauss: float

    @staticmethod
    def make(nu_min, nu_max, dnu, opd_max=None, fwhm_gauss=0.0, n_channels=None) -> "Sounder":
        n = round((nu_max - nu_min) / dnu) + 1 if n_channels is None else int(n_channels)
        return Sounder(float(nu_min), float(nu_max), float(dnu), n,
                       1.0 / (2.0 * dnu) if opd_max is None else float(opd_max), float(fwhm_gauss))

    def c_struct(self) -> _lib.Sounder:
        s = _lib.Sounder()
        s.nu_min, s.nu_max, s.dnu = self.nu_min, self.nu_max, self.dnu
        s.n_channels, s.opd_max, s.fwhm_gauss = self.n_channels, self.opd_max, self.fwhm_gauss
        return s


def IASIInstrument(fwhm_gauss: float = 0.5) -> Sounder:  # sounder.jl:65-68
    return Sounder.make(645.0, 2760.0, 0.25, opd_max=2.0, fwhm_gauss=fwhm_gauss)


def IASINGInstrument(fwhm_gauss: float = 0.25) -> Sounder:  # sounder.jl:86-89
    return Sounder.make(645.0, 2760.0, 0.125, opd_max=4.0, fwhm_gauss=fwhm_gauss)


def CrISInstrument(band: str = "full", fwhm_gauss: float = 0.0) -> Sounder:  # sounder.jl:102-110
    rng = {"full": (650.0, 2550.0), "lwir": (650.0, 1095.0), "mwir": (1210.0, 1750.0),
           "swir": (2155.0, 2550.0)}
    if band not in rng:
        raise IRSError(f"CrIS band must be :full, :lwir, :mwir, or :swir; got :{band}")
    return Sounder.make(*rng[band], 0.625, opd_max=0.8, fwhm_gauss=fwhm_gauss)


def MTGIRSInstrument(band: str = "full", fwhm_gauss: float = 0.0) -> Sounder:  # sounder.jl:121-128
    rng = {"full": (700.0, 2175.0), "lwir": (700.0, 1210.0), "mwir": (1600.0, 2175.0)}
    if band not in rng:
        raise IRSError(f"MTG-IRS band must be :full, :lwir, or :mwir; got :{band}")
    return Sounder.make(*rng[band], 0.625, opd_max=0.8, fwhm_gauss=fwhm_gauss)


@dataclass
class ViewingGeometry:
    """src/Sensor/geometry.jl:18-34"""
    zenith_angle: float
    azimuth_angle: float = 0.0
    mu: float = field(init=False)

    def __post_init__(self):
        if not (0.0 <= self.zenith_angle < 90.0):
            raise IRSError(f"Viewing zenith angle must be in [0, 90); got {self.zenith_angle}°")
        self.mu = math.cos(math.radians(self.zenith_angle))


def nadir_geometry() -> ViewingGeometry:
    return ViewingGeometry(0.0)


def scan_angle_to_local_zenith(scan_angle: float, h_sat_km: float = 817.0,
                               R_earth_km: float = 6371.0) -> float:
    """geometry.jl:92-101"""
    s = (R_earth_km + h_sat_km) / R_earth_km * math.sin(math.radians(abs(scan_angle)))
    if s > 1.0:
        raise IRSError(f"scan_angle {scan_angle}° exceeds limb angle from h={h_sat_km} km")
    return math.degrees(math.asin(s))


# ------------------------------------------------------------------ context
def _read_tips(path=DATA / "tips2024_q.csv"):
    out = {}
    for line in open(path):
        if line.startswith("#"):
            continue
        p = line.strip().split(",")
        out[(int(p[0]), int(p[1]))] = np.array([float(v) for v in p[2:]])
    return out


def _read_cols(path):
    rows = [l.strip().split(",") for l in open(path).readlines()[1:] if l.strip()]
    return np.ascontiguousarray(np.array(rows, dtype=np.float64).T)


class B200Context:
    """One CUDA context of libirs_b200 on `device` with the bundled tables loaded.

    Plays the role of the reference's `backend=` seam (strategy.jl:21-75): pass it
    as `backend=` or let the module-level default be created on first use."""

    def __init__(self, device: int = 0, load_tables: bool = True):
        self.lib = _lib.load()
        h = C.c_void_p()
        check(self.lib.irs_create(device, C.byref(h)))
        self.h = h
        self.device = device
        self._lists: Dict[int, tuple] = {}
        self._relmat_key = None
        if load_tables:
            self.load_tables()

    def load_tables(self):
        for (mol, iso), q in _read_tips().items():
            q = np.ascontiguousarray(q)
            check(self.lib.irs_set_partition_table(self.h, mol, iso, 70, len(q), dptr(q)))
        nu, cs, cf, te = _read_cols(DATA / "mt_ckd43_h2o_coeffs.csv")
        self._h2o = (nu, cs, cf, te)
        check(self.lib.irs_set_continuum_h2o(self.h, len(nu), *(dptr(a) for a in self._h2o)))
        nu, s, xf, td = _read_cols(DATA / "mt_ckd_co2_coeffs.csv")
        self._co2 = (nu, s, xf, td)
        check(self.lib.irs_set_continuum_co2(self.h, len(nu), *(dptr(a) for a in self._co2)))

    def upload_linelist(self, species: int, ll: HITRANLinelist, y0: Optional[np.ndarray] = None):
        key = (id(ll), None if y0 is None else id(y0))
        if self._lists.get(int(species), (None,))[0] == key:
            return
        lines = np.ascontiguousarray(ll.lines, dtype=LINE_DTYPE)
        if lines.dtype.itemsize != 56:
            raise IRSError("HITRANLine records must be 56 bytes (the isbits layout)")
        yy = None if y0 is None else np.ascontiguousarray(y0, dtype=np.float64)
        if yy is not None and len(yy) != len(lines):
            raise IRSError("VPYLineMixing.y0 must have one entry per CO2 line")
        check(self.lib.irs_upload_linelist(self.h, int(species), lines.ctypes.data, len(lines),
                                           dptr(yy) if yy is not None else None))
        self._lists[int(species)] = (key, ll, y0)

    def set_cia(self, pair: int, blocks):
        """A HITRAN CIA table (pair 1 CO2-CO2, 2 N2-N2, 3 O2-O2) as load_cia_table returns it;
        None or [] removes it."""
        blocks = blocks or []
        T = np.array([b[0] for b in blocks], dtype=np.float64)
        off = np.zeros(len(blocks) + 1, dtype=np.int64)
        off[1:] = np.cumsum([len(b[1]) for b in blocks])
        nu = np.ascontiguousarray(np.concatenate([b[1] for b in blocks]) if blocks else np.zeros(0), dtype=np.float64)
        sg = np.ascontiguousarray(np.concatenate([b[2] for b in blocks]) if blocks else np.zeros(0), dtype=np.float64)
        check(self.lib.irs_set_cia(self.h, int(pair), len(blocks), dptr(T) if len(T) else None,
                                   off.ctypes.data_as(C.POINTER(C.c_int64)), dptr(nu) if len(nu) else None,
                                   dptr(sg) if len(sg) else None))

    def upload_relmat(self, data, whitelist=frozenset(), min_band_strength: float = 0.0, bands=None):
        """Hand HITRANRelmatData (optionally a subset of its bands) to the library."""
        bands = data.bands if bands is None else bands
        key = (id(data), tuple(id(b) for b in bands), frozenset(whitelist), float(min_band_strength))
        if self._relmat_key == key:
            return
        from .relmat import _CRelmat
        c = _CRelmat(bands, data.wtfit, set(whitelist))
        check(self.lib.irs_upload_relmat(self.h, int(data.species), c.bands, c.n_bands, c.wt, c.n_wt,
                                         float(min_band_strength)))
        self._relmat_key = key
        self._relmat_ref = (data, bands)

    def stage_times(self) -> StageTimes:
        t = StageTimes()
        check(self.lib.irs_last_stage_times(self.h, C.byref(t)))
        return t

    def close(self):
        if getattr(self, "h", None):
            self.lib.irs_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default: Optional[B200Context] = None


def default_context() -> B200Context:
    global _default
    if _default is None:
        _default = B200Context()
    return _default


# ----------------------------------------------------------- operators
def compute_voigt_cross_sections(nu_grid, linelist: HITRANLinelist, T: float, p_atm: float, *,
                                 vmr_self: float = 0.0, cutoff: float = 25.0, backend=None,
                                 method: VoigtMethod = FullFaddeeva, x_far: float = 122.0,
                                 precision: str = "fp64") -> np.ndarray:
    """compute_voigt_cross_sections (src/CrossSections/voigt.jl:375-462), cm^2/molecule."""
    ctx = backend or default_context()
    grid = np.ascontiguousarray(getattr(nu_grid, "nu", nu_grid), dtype=np.float64)
    mols = linelist.molecules
    if len(mols) != 1:
        raise IRSError("compute_voigt_cross_sections takes a single-molecule line list here")
    sp = next(iter(mols))
    ctx.upload_linelist(sp, linelist)
    out = np.empty(len(grid))
    check(ctx.lib.irs_cross_sections(ctx.h, sp, dptr(grid), len(grid), float(T), float(p_atm),
                                     float(vmr_self), float(cutoff), int(method), float(x_far),
                                     PRECISION[precision], dptr(out)))
    return out


def fm_options(internal_dnu=0.001, high_res_factor=None, cutoff=25.0, lm_cutoff=None, dptmn=1e-6,
               apply_continuum=True, continua=("h2o", "co2", "co2_cia", "n2", "o2"),
               with_ils=True, apodization="gaussian", line_mixing=None,
               T_method="logp_at_pcg", source_function="cim", method=FullFaddeeva,
               x_far=122.0, precision="fp64") -> FMOptions:
    """forward_model keyword arguments (src/Sensor/sounder.jl:233-252) as the C struct."""
    if apodization not in APODIZATION:
        raise IRSError(f"Unknown apodization {apodization}; expected :gaussian or one of "
                       f"{[k for k in APODIZATION if k != 'gaussian']}")
    if T_method not in ("logp_at_pcg", "mass_weighted"):
        raise IRSError(f"T_method must be :logp_at_pcg or :mass_weighted, got :{T_method}")
    if source_function not in ("cim", "toon"):
        raise IRSError(f"source_function must be :toon or :cim, got :{source_function}")
    o = FMOptions()
    o.internal_dnu = -1.0 if internal_dnu is None else float(internal_dnu)
    o.high_res_factor = int(high_res_factor or 0)
    o.apply_continuum = int(bool(apply_continuum))
    o.continua = sum(CONTINUA[c] for c in continua)
    o.with_ils = int(bool(with_ils))
    o.apodization = APODIZATION[apodization]
    o.line_mixing = 0 if line_mixing is None else int(line_mixing.mode)
    o.T_method = 0 if T_method == "logp_at_pcg" else 1
    o.source_function = 0 if source_function == "cim" else 1
    o.method = int(method)
    o.precision = PRECISION[precision]
    o.cutoff = float(cutoff)
    o.lm_cutoff = float(cutoff if lm_cutoff is None else lm_cutoff)
    o.dptmn = float(dptmn)
    o.x_far = float(x_far)
    return o


class _ProfileBatch:
    """Keeps the numpy buffers behind an array of irs_profile structs alive."""

    def __init__(self, profs: Sequence[AtmosphericProfile], T_sfcs, mus, epss):
        self.keep = []
        self.arr = (Profile * len(profs))()
        for k, pr in enumerate(profs):
            p = np.ascontiguousarray(pr.pressure, dtype=np.float64)
            T = np.ascontiguousarray(pr.temperature, dtype=np.float64)
            sp = np.array(sorted(int(s) for s in pr.vmr), dtype=np.int32)
            vmr = np.ascontiguousarray(np.stack([np.asarray(pr.vmr[s], dtype=np.float64) for s in sp])
                                       if len(sp) else np.zeros((0, len(p))))
            self.keep += [p, T, sp, vmr]
            c = self.arr[k]
            c.n_lev, c.n_species = len(p), len(sp)
            c.pressure, c.temperature = dptr(p), dptr(T)
            c.species = sp.ctypes.data_as(C.POINTER(C.c_int32))
            c.vmr = dptr(vmr)
            c.T_sfc = float("nan") if T_sfcs[k] is None else float(T_sfcs[k])
            c.mu = float(mus[k])
            c.eps_sfc = float(epss[k])


def sounder_grid(s: Sounder) -> np.ndarray:
    """Channel wavenumbers (sounder_grid, sounder.jl:135-137)."""
    n_nu, n_ch = C.c_int64(), C.c_int64()
    o = fm_options(with_ils=False, high_res_factor=1)
    check(_lib.load().irs_grid_size(C.byref(s.c_struct()), C.byref(o), C.byref(n_nu), C.byref(n_ch)))
    return np.array([s.nu_min + i * s.dnu for i in range(n_ch.value)])


def _prepare(ctx, linelists, line_mixing):
    for sp, ll in linelists.items():
        y0 = line_mixing.y0 if (line_mixing is not None and int(sp) == 2) else None
        ctx.upload_linelist(int(sp), ll, y0)
    if line_mixing is not None and line_mixing.y0 is None:  # relaxation-matrix data
        wl = line_mixing.whitelist if line_mixing.mode == _lib.IRS_LM_RELMAT_VPW else set()
        ctx.upload_relmat(line_mixing.data, wl, line_mixing.min_band_strength)
    # species uploaded earlier but absent from this call must not contribute
    for sp in list(ctx._lists):
        if sp not in {int(s) for s in linelists}:
            empty = HITRANLinelist(np.zeros(0, LINE_DTYPE))
            ctx.upload_linelist(sp, empty)
            del ctx._lists[sp]


def forward_model_batch(profiles: Sequence[AtmosphericProfile], linelists, *, sounder: Sounder = None,
                        geoms: Optional[Sequence[ViewingGeometry]] = None, T_sfcs=None, eps_sfcs=None,
                        backend=None, line_mixing: Optional[VPYLineMixing] = None, **kw):
    """forward_model for a batch of profiles sharing one sounder and options.

    Returns (nu_out, R[n_prof, n_ch], BT[n_prof, n_ch])."""
    ctx = backend or default_context()
    sounder = sounder or IASIInstrument()
    n = len(profiles)
    geoms = geoms or [nadir_geometry()] * n
    T_sfcs = T_sfcs if T_sfcs is not None else [None] * n
    eps_sfcs = eps_sfcs if eps_sfcs is not None else [1.0] * n
    _prepare(ctx, linelists, line_mixing)
    o = fm_options(line_mixing=line_mixing, **kw)
    batch = _ProfileBatch(profiles, T_sfcs, [g.mu for g in geoms], eps_sfcs)
    s = sounder.c_struct()
    nu_out = sounder_grid(sounder)
    R = np.empty((n, len(nu_out)))
    BT = np.empty((n, len(nu_out)))
    check(ctx.lib.irs_forward_model_batch(ctx.h, batch.arr, n, C.byref(s), C.byref(o), dptr(R), dptr(BT)))
    return nu_out, R, BT


def shard_range(n: int, n_shards: int, shard: int):
    """(first, count) of the contiguous, balanced shard `shard` of n items over n_shards
    (irs_shard_range: the first n % n_shards shards take one more).  Host only."""
    first, count = C.c_int64(), C.c_int64()
    check(_lib.load().irs_shard_range(int(n), int(n_shards), int(shard), C.byref(first), C.byref(count)))
    return first.value, count.value


def forward_model_batch_multi(profiles: Sequence[AtmosphericProfile], linelists, *, backends: Sequence,
                              sounder: Sounder = None, geoms: Optional[Sequence[ViewingGeometry]] = None,
                              T_sfcs=None, eps_sfcs=None, line_mixing: Optional[VPYLineMixing] = None, **kw):
    """forward_model_batch spread over several contexts (one per GPU): contiguous shards
    of the batch, one host thread per context, gathered in batch order
    (irs_forward_model_batch_multi).  Returns (nu_out, R[n_prof, n_ch], BT[n_prof, n_ch])."""
    if not backends:
        raise IRSError("forward_model_batch_multi needs at least one context")
    sounder = sounder or IASIInstrument()
    n = len(profiles)
    geoms = geoms or [nadir_geometry()] * n
    T_sfcs = T_sfcs if T_sfcs is not None else [None] * n
    eps_sfcs = eps_sfcs if eps_sfcs is not None else [1.0] * n
    for ctx in backends:
        _prepare(ctx, linelists, line_mixing)
    o = fm_options(line_mixing=line_mixing, **kw)
    batch = _ProfileBatch(profiles, T_sfcs, [g.mu for g in geoms], eps_sfcs)
    s = sounder.c_struct()
    nu_out = sounder_grid(sounder)
    R = np.empty((n, len(nu_out)))
    BT = np.empty((n, len(nu_out)))
    hs = (C.c_void_p * len(backends))(*[ctx.h.value for ctx in backends])
    check(backends[0].lib.irs_forward_model_batch_multi(hs, len(backends), batch.arr, n, C.byref(s), C.byref(o),
                                                        dptr(R), dptr(BT)))
    return nu_out, R, BT


def distributed_batch(compute, n: int, dist=None):
    """Run a batch of n independent items over the ranks of a torch.distributed group:
    rank r computes its contiguous shard (shard_range) as compute(first, count) -> a tuple
    of arrays with the shard's items along axis 0, and every rank receives the arrays of
    the whole batch in batch order (an all-gather of the shards).  `dist` None: one
    process computes everything.  The only exchange is that gather."""
    if dist is None:
        return compute(0, n)
    world, rank = dist.get_world_size(), dist.get_rank()
    first, count = shard_range(n, world, rank)
    local = compute(first, count) if count else None
    parts = [None] * world
    dist.all_gather_object(parts, local)
    parts = [p for p in parts if p is not None]
    return tuple(np.concatenate([p[k] for p in parts], axis=0) for k in range(len(parts[0])))


def forward_model_batch_distributed(profiles: Sequence[AtmosphericProfile], linelists, *, dist=None,
                                    backend=None, sounder: Sounder = None,
                                    geoms: Optional[Sequence[ViewingGeometry]] = None, T_sfcs=None, eps_sfcs=None,
                                    line_mixing: Optional[VPYLineMixing] = None, **kw):
    """forward_model_batch over the ranks of a process group, one GPU (context) per rank:
    each rank runs its contiguous shard of the profiles and all ranks receive R and BT of
    the whole batch in batch order.  Returns (nu_out, R[n_prof, n_ch], BT[n_prof, n_ch])."""
    n = len(profiles)
    sounder = sounder or IASIInstrument()

    def pick(v, a, b):
        return None if v is None else list(v)[a:a + b]

    def compute(first, count):
        _, R, BT = forward_model_batch(profiles[first:first + count], linelists, sounder=sounder,
                                       geoms=pick(geoms, first, count), T_sfcs=pick(T_sfcs, first, count),
                                       eps_sfcs=pick(eps_sfcs, first, count), backend=backend,
                                       line_mixing=line_mixing, **kw)
        return R, BT

    R, BT = distributed_batch(compute, n, dist)
    return sounder_grid(sounder), R, BT


def forward_model(prof: AtmosphericProfile, linelists, *, sounder: Sounder = None,
                  iasi: Sounder = None, geom: ViewingGeometry = None, T_sfc: Optional[float] = None,
                  eps_sfc: float = 1.0, backend=None, line_mixing: Optional[VPYLineMixing] = None, **kw):
    """forward_model (src/Sensor/sounder.jl:233-360) -> (nu, R, BT)."""
    sounder = iasi if iasi is not None else sounder
    nu, R, BT = forward_model_batch([prof], linelists, sounder=sounder, geoms=[geom or nadir_geometry()],
                                    T_sfcs=[T_sfc], eps_sfcs=[eps_sfc], backend=backend,
                                    line_mixing=line_mixing, **kw)
    return nu, R[0], BT[0]


iasi_forward_model = forward_model

from .synthetic import afgl_atmosphere, synthetic_linelist  # noqa: E402,F401
from .estimation import (ColumnScale, FullProfile, Jacobian, PartialColumns, StateVectorSpec,  # noqa: E402,F401
                         analytic_jacobian, analytic_jacobian_batch, vjp_batch, column, default_fd_steps, dfs_partition,
                         finite_difference_jacobian, forward_model_rrule, pack_state, partial_column_basis,
                         state_labels, unpack_state, vmr_range, build_sa, scene_nedt, exclude_channels,
                         apodized_measurement_covariance, scene_measurement_covariance,
                         RetrievalResult, optimal_estimation, optimal_estimation_batch, oe_diagnostics)
from .continuum import CIA_PAIRS, load_cia_table  # noqa: E402,F401
from .hitran import (LINELIST_CACHE_VERSION, clear_linelist_cache, filter_linelist, linelist_cache_dir,  # noqa: E402,F401,E501
                     load_hitran_par, load_linelist, parse_hitran_par, set_linelist_cache_dir)
from .relmat import (BandModes, HITRANRelmatData, RelmatBand, VPWLineMixing, VPYLineMixing,  # noqa: E402,F401
                     W0B0Table, band_eff_strength, band_modes, build_w_matrix, calc_w_and_y,
                     compute_lm_dispersive_correction, compute_voigt_lm_cross_sections,
                     compute_voigt_vpw_cross_sections, compute_vpw_band_perturbation, compute_vpw_band_xsec,
                     default_vpw_whitelist, load_hitran_relmat, load_wtfit, parse_bandinfo, parse_sfile,
                     relmat_lines, vpw_perturbation)
from .iasi_l1c import (IASIL1CGranule, brightness_temperature, cloud_fraction, measurement, nfov,  # noqa: E402,F401
                       read_iasi_l1c, retrieve_granule, solar_reflection_angle)
from .noise_covariance import (SounderNoiseCovariance, load_noise_covariance, measurement_covariance,  # noqa: E402,F401,E501
                               read_iasi_ncm, subset_channels, to_bt)
from .operators import (apply_ils, dB_dT, faddeeva, faddeeva_voigt, ils_kernel, level_transmittances,  # noqa: E402,F401,E501
                        planck_radiance, schwarzschild_rte, voigt_profile)
from .robust import RobustRetrievalResult, robust_estimation, robust_estimation_batch  # noqa: E402,F401
from .surrogate import Surrogate, surrogate_features, surrogate_first_guess, surrogate_forward_batch  # noqa: E402,F401,E501
