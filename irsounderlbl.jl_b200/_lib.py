"""ctypes binding of libirs_b200.so (the C ABI of include/irs_b200.h).

The CUDA library is the only implementation: there is no CPU fallback, and a
missing or unloadable library raises immediately.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
SO = HERE / "libirs_b200.so"

IRS_WEIDEMAN, IRS_PSEUDOVOIGT, IRS_FULLFADDEEVA = 1, 2, 3
IRS_FP64, IRS_MIXED, IRS_MIXED_DIRECT = 0, 1, 2
IRS_LM_NONE, IRS_LM_PER_LINE_Y, IRS_LM_RELMAT_VPY, IRS_LM_RELMAT_VPW = 0, 1, 2, 3

# RelmatLine isbits layout (src/CrossSections/line_mixing.jl:35-47), 72 bytes
RELMAT_LINE_DTYPE = np.dtype([("isot", "i1"), ("nu", "f8"), ("ji", "i2"), ("branch", "i1"), ("gv_air", "f8"),
                              ("n_air", "f4"), ("shift", "f4"), ("e_lower", "f8"), ("dipo0", "f8"),
                              ("popu_t0", "f8"), ("dipo_t", "f8")], align=True)
assert RELMAT_LINE_DTYPE.itemsize == 72

# HITRANLine isbits layout (src/HITRAN/linelist.jl:20-31), 56 bytes
LINE_DTYPE = np.dtype({
    "names": ["mol_id", "iso_id", "wavenumber", "intensity", "a_coeff", "air_broad",
              "self_broad", "lower_energy", "temp_depend", "pressure_shift"],
    "formats": ["i1", "i1", "f8", "f8", "f8", "f4", "f4", "f8", "f4", "f4"],
    "offsets": [0, 1, 8, 16, 24, 32, 36, 40, 48, 52],
    "itemsize": 56,
})


class Sounder(C.Structure):
    _fields_ = [("nu_min", C.c_double), ("nu_max", C.c_double), ("dnu", C.c_double),
                ("n_channels", C.c_int64), ("opd_max", C.c_double), ("fwhm_gauss", C.c_double)]


class FMOptions(C.Structure):
    _fields_ = [("internal_dnu", C.c_double), ("high_res_factor", C.c_int32),
                ("apply_continuum", C.c_int32), ("continua", C.c_int32), ("with_ils", C.c_int32),
                ("apodization", C.c_int32), ("line_mixing", C.c_int32), ("T_method", C.c_int32),
                ("source_function", C.c_int32), ("method", C.c_int32), ("precision", C.c_int32),
                ("cutoff", C.c_double), ("lm_cutoff", C.c_double), ("dptmn", C.c_double),
                ("x_far", C.c_double)]


class Profile(C.Structure):
    _fields_ = [("n_lev", C.c_int32), ("n_species", C.c_int32),
                ("pressure", C.POINTER(C.c_double)), ("temperature", C.POINTER(C.c_double)),
                ("species", C.POINTER(C.c_int32)), ("vmr", C.POINTER(C.c_double)),
                ("T_sfc", C.c_double), ("mu", C.c_double), ("eps_sfc", C.c_double)]


class StateSpec(C.Structure):
    _fields_ = [("n_retrieved", C.c_int32), ("retrieved", C.POINTER(C.c_int32)),
                ("include_temperature", C.c_int32), ("include_tsfc", C.c_int32),
                ("include_emissivity", C.c_int32), ("log_vmr", C.c_int32),
                ("vmr_coupling", C.c_int32), ("observable", C.c_int32)]


class OEParams(C.Structure):
    _fields_ = [("max_iter", C.c_int32), ("max_linesearch", C.c_int32), ("method", C.c_int32),
                ("gamma0", C.c_double), ("gamma_factor", C.c_double), ("gamma_min", C.c_double),
                ("conv_factor", C.c_double), ("eps_fixed", C.c_double)]


class StageTimes(C.Structure):
    _fields_ = [("line_params_ms", C.c_double), ("line_sum_ms", C.c_double),
                ("rte_ms", C.c_double), ("ils_ms", C.c_double), ("total_ms", C.c_double),
                ("pairs", C.c_double), ("core_pairs", C.c_double), ("h2d_bytes", C.c_double),
                ("d2h_bytes", C.c_double), ("launches", C.c_double), ("evaluated_pairs", C.c_double),
                ("lm_host_ms", C.c_double), ("lm_device_ms", C.c_double)]


# every symbol the header declares, with its ctypes signature
_P = C.c_void_p
_PD = C.POINTER(C.c_double)
_PF = C.POINTER(C.c_float)
class RelmatBandC(C.Structure):  # irs_relmat_band
    _fields_ = [("lines", C.c_void_p), ("n_lines", C.c_int64), ("nu_min", C.c_double), ("nu_max", C.c_double),
                ("li", C.c_int32), ("lf", C.c_int32), ("isot", C.c_int32), ("molecule", C.c_int32),
                ("whitelisted", C.c_int32), ("_pad", C.c_int32)]


class WtfitEntryC(C.Structure):  # irs_wtfit_entry
    _fields_ = [("lli", C.c_int32), ("llf", C.c_int32), ("sub", C.c_int32), ("ji", C.c_int32),
                ("jip", C.c_int32), ("_pad", C.c_int32), ("w0r", C.c_double), ("b0r", C.c_double)]


SIGNATURES = {
    "irs_abi_version": ([], C.c_int),
    "irs_last_error": ([], C.c_char_p),
    "irs_create": ([C.c_int, C.POINTER(C.c_void_p)], C.c_int),
    "irs_destroy": ([_P], C.c_int),
    "irs_set_partition_table": ([_P, C.c_int, C.c_int, C.c_int, C.c_int, _PD], C.c_int),
    "irs_set_continuum_h2o": ([_P, C.c_int, _PD, _PD, _PD, _PD], C.c_int),
    "irs_set_continuum_co2": ([_P, C.c_int, _PD, _PD, _PD, _PD], C.c_int),
    "irs_upload_linelist": ([_P, C.c_int, _P, C.c_int64, _PD], C.c_int),
    "irs_cross_sections": ([_P, C.c_int, _PD, C.c_int64, C.c_double, C.c_double, C.c_double,
                            C.c_double, C.c_int, C.c_double, C.c_int, _PD], C.c_int),
    "irs_forward_model_batch": ([_P, C.POINTER(Profile), C.c_int, C.POINTER(Sounder),
                                 C.POINTER(FMOptions), _PD, _PD], C.c_int),
    "irs_forward_model_batch_device": ([_P, C.POINTER(Profile), C.c_int, C.POINTER(Sounder),
                                        C.POINTER(FMOptions), C.c_void_p, C.c_void_p, C.c_void_p],
                                       C.c_int),
    "irs_state_size": ([C.POINTER(StateSpec), C.c_int, C.POINTER(C.c_int64)], C.c_int),
    "irs_jacobian_batch": ([_P, C.POINTER(Profile), C.c_int, C.POINTER(Sounder), C.POINTER(FMOptions),
                            C.POINTER(StateSpec), _PD, _PD], C.c_int),
    "irs_vjp_batch": ([_P, C.POINTER(Profile), C.c_int, C.POINTER(Sounder), C.POINTER(FMOptions),
                       C.POINTER(StateSpec), _PD, _PD, _PD], C.c_int),
    "irs_oe_batch": ([_P, C.POINTER(Profile), C.c_int, C.POINTER(Sounder), C.POINTER(FMOptions),
                      C.POINTER(StateSpec), _PD, _PD, _PD, _PD, _PD, C.POINTER(OEParams), _PD, _PD, _PD,
                      C.POINTER(C.c_int32), C.POINTER(C.c_int32), _PD], C.c_int),
    "irs_forward_model_batch_multi": ([C.POINTER(C.c_void_p), C.c_int, C.POINTER(Profile), C.c_int,
                                       C.POINTER(Sounder), C.POINTER(FMOptions), _PD, _PD], C.c_int),
    "irs_shard_range": ([C.c_int64, C.c_int, C.c_int, C.POINTER(C.c_int64), C.POINTER(C.c_int64)], C.c_int),
    "irs_synchronize": ([_P], C.c_int),
    "irs_last_stage_times": ([_P, C.POINTER(StageTimes)], C.c_int),
    "irs_cross_sections_noalloc": ([_P, C.c_int64, _P, C.POINTER(C.c_int32), C.c_int, C.c_int, C.c_int, _P,
                                    C.c_int64, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int,
                                    C.c_double, _P, _P], C.c_int),
    "irs_surrogate_create": ([_P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_uint64, C.POINTER(C.c_void_p)],
                             C.c_int),
    "irs_surrogate_destroy": ([_P], C.c_int),
    "irs_surrogate_grad_size": ([_P, C.POINTER(C.c_int64)], C.c_int),
    "irs_surrogate_grad_device": ([_P, _P, _P, C.POINTER(C.c_int32), C.c_int64, C.POINTER(C.c_float),
                                   C.POINTER(C.c_double), _P], C.c_int),
    "irs_surrogate_apply_device": ([_P, C.POINTER(C.c_float), C.c_float, _P], C.c_int),
    "irs_surrogate_param_count": ([_P, C.POINTER(C.c_int64)], C.c_int),
    "irs_surrogate_get_params": ([_P, _PF], C.c_int),
    "irs_surrogate_set_params": ([_P, _PF], C.c_int),
    "irs_surrogate_set_scaling": ([_P, _PF, _PF, _PF, _PF], C.c_int),
    "irs_surrogate_set_whitening": ([_P, _PF], C.c_int),
    "irs_surrogate_train": ([_P, _PF, _PF, C.c_int64, C.c_int, C.c_int, C.c_float, C.c_uint64, _PD], C.c_int),
    "irs_surrogate_gradients": ([_P, _PF, _PF, C.c_int64, _PF, _PD], C.c_int),
    "irs_surrogate_infer": ([_P, _PF, C.c_int64, _PF, _PF], C.c_int),
    "irs_surrogate_infer_device": ([_P, _P, C.c_int64, _P, _P, _P], C.c_int),
    "irs_gemm_bf16": ([_P, _P, _P, C.c_int, C.c_int, C.c_int, _PF], C.c_int),
    "irs_oe_batch_banded": ([_P, C.POINTER(Profile), C.c_int, C.POINTER(Sounder), C.POINTER(FMOptions),
                             C.POINTER(StateSpec), _PD, _PD, C.c_int, C.POINTER(C.c_uint8), _PD, _PD, _PD,
                             C.POINTER(OEParams), _PD, _PD, _PD, C.POINTER(C.c_int32), C.POINTER(C.c_int32), _PD],
                            C.c_int),
    "irs_voigt_profile": ([_P, _PD, C.c_int64, C.c_double, C.c_double, C.c_double, C.c_int, _PD], C.c_int),
    "irs_faddeeva": ([_P, _PD, _PD, C.c_int64, _PD, _PD], C.c_int),
    "irs_faddeeva32": ([_P, _PD, _PD, C.c_int64, _PD, _PD], C.c_int),
    "irs_ils_kernel": ([_P, C.c_double, C.c_double, C.c_double, C.c_int, C.c_int64, _PD], C.c_int),
    "irs_apply_ils": ([_P, _PD, C.c_int64, C.c_double, _PD, C.c_int64, _PD], C.c_int),
    "irs_schwarzschild_rte": ([_P, _PD, C.c_int64, C.c_int, _PD, _PD, C.c_double, C.c_double, C.c_double, C.c_int,
                               _PD, _PD], C.c_int),
    "irs_set_cia": ([_P, C.c_int, C.c_int, _PD, C.POINTER(C.c_int64), _PD, _PD], C.c_int),
    "irs_upload_relmat": ([_P, C.c_int, C.POINTER(RelmatBandC), C.c_int, C.POINTER(WtfitEntryC), C.c_int64,
                           C.c_double], C.c_int),
    "irs_relmat_w_matrix": ([C.POINTER(RelmatBandC), C.POINTER(WtfitEntryC), C.c_int64, C.c_double, C.c_double,
                             _PD, _PD], C.c_int),
    "irs_relmat_y": ([C.POINTER(RelmatBandC), C.POINTER(WtfitEntryC), C.c_int64, C.c_double, C.c_double, _PD],
                     C.c_int),
    "irs_band_modes": ([C.POINTER(RelmatBandC), C.POINTER(WtfitEntryC), C.c_int64, C.c_double, C.c_double,
                        C.c_double, C.c_double, _PD, _PD, _PD, C.POINTER(C.c_int64)], C.c_int),
    "irs_vpw_band_xsec": ([_P, _PD, C.c_int64, _PD, _PD, C.c_int64, C.c_double, C.c_double, C.c_double, _PD],
                          C.c_int),
    "irs_lm_perturbation": ([_P, C.c_int, _PD, C.c_int64, C.c_double, C.c_double, C.c_double, C.c_double,
                             C.c_double, C.c_uint32, _PD], C.c_int),
    "irs_grid_size": ([C.POINTER(Sounder), C.POINTER(FMOptions), C.POINTER(C.c_int64),
                       C.POINTER(C.c_int64)], C.c_int),
}

_lib = None


def load(path: Path | str | None = None):
    """Load libirs_b200.so (built in-tree by build.py); raise if it is missing."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path or SO)
    if not p.exists():
        raise RuntimeError(f"{p} is missing: build it with `python irsounderlbl.jl_b200/build.py` "
                           "(there is no CPU fallback)")
    lib = C.CDLL(str(p))
    for name, (args, res) in SIGNATURES.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res
    if path is None:
        _lib = lib
    return lib


class IRSError(RuntimeError):
    """Raised for a non-zero status of the C ABI (the reference raises ErrorException)."""


def check(rc: int):
    if rc != 0:
        raise IRSError(f"[{rc}] " + (load().irs_last_error() or b"").decode())


def dptr(a: np.ndarray):
    return a.ctypes.data_as(_PD)


def fptr(a: np.ndarray):
    assert a.dtype == np.float32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_PF)
