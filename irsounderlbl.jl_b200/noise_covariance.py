"""Host-provided sensor noise covariance (src/Sensor/noise_covariance.jl).

SounderNoiseCovariance with the channel subset and the Planck linearisation to
brightness-temperature space.  The EUMETSAT IASI NCM product is NetCDF-4/HDF5; it is
read with h5py when that module is importable (it is not part of this image), else
read_iasi_ncm raises.  A dense Se is consumed by the reference's CPU retrieval; the GPU
retrieval here takes its diagonal.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Optional, Tuple

import numpy as np

from ._lib import IRSError

W2_TO_MW2 = 1.0e6   # noise_covariance.jl:51


@dataclass
class SounderNoiseCovariance:
    """SounderNoiseCovariance (noise_covariance.jl:34-38): space "radiance" or "bt"."""
    nu: np.ndarray
    cov: np.ndarray
    space: str


def measurement_covariance(nc: SounderNoiseCovariance) -> np.ndarray:
    """The covariance symmetrised (noise_covariance.jl:47)."""
    return 0.5 * (nc.cov + nc.cov.T)


def read_iasi_ncm(path: str, nu_window: Optional[Tuple[float, float]] = None) -> SounderNoiseCovariance:
    """read_iasi_ncm (noise_covariance.jl:66-91): Wn (m^-1) and Covariance_R (W^2) ->
    cm^-1 and mW^2, optionally the contiguous channel window only."""
    try:
        import h5py
    except ImportError as e:
        raise IRSError("reading the IASI NCM (NetCDF-4/HDF5) needs h5py, which is not installed") from e
    with h5py.File(path, "r") as h:
        if "Wn" not in h or "Covariance_R" not in h:
            raise IRSError(f"{path} is not an IASI NCM file (missing Wn / Covariance_R)")
        nu = np.asarray(h["Wn"][...], dtype=np.float64) / 100.0
        if nu_window is None:
            cov = np.asarray(h["Covariance_R"][...], dtype=np.float64)
        else:
            keep = np.flatnonzero((nu >= nu_window[0]) & (nu <= nu_window[1]))
            if len(keep) == 0:
                raise IRSError(f"ν_window {tuple(nu_window)} selects no NCM channels")
            i1, i2 = keep[0], keep[-1] + 1
            cov = np.asarray(h["Covariance_R"][i1:i2, i1:i2], dtype=np.float64)
            nu = nu[i1:i2]
    return SounderNoiseCovariance(nu, cov * W2_TO_MW2, "radiance")


def load_noise_covariance(path: str, format: str = "iasi_ncm", **kw) -> SounderNoiseCovariance:
    """load_noise_covariance (noise_covariance.jl:99-103)."""
    if format == "iasi_ncm":
        return read_iasi_ncm(path, **kw)
    raise IRSError(f"unknown noise-covariance format :{format} (supported: :iasi_ncm)")


def subset_channels(nc: SounderNoiseCovariance, nu_target, atol: float = 1e-3) -> SounderNoiseCovariance:
    """subset_channels (noise_covariance.jl:113-124): nearest channel within atol, in order."""
    nu_target = np.asarray(nu_target, dtype=np.float64)
    idx = np.empty(len(nu_target), int)
    for k, nt in enumerate(nu_target):
        j = int(np.argmin(np.abs(nc.nu - nt)))
        if abs(nc.nu[j] - nt) > atol:
            raise IRSError(f"no NCM channel within {atol} cm⁻¹ of target {nt} (nearest {nc.nu[j]})")
        idx[k] = j
    return SounderNoiseCovariance(nc.nu[idx], nc.cov[np.ix_(idx, idx)], nc.space)


def to_bt(nc: SounderNoiseCovariance, Tb, T_floor: float = 1e-6) -> SounderNoiseCovariance:
    """to_bt (noise_covariance.jl:140-152): S_bt = D S_R D, D_i = 1/max(dB/dT(nu_i, Tb_i), T_floor)."""
    from .estimation import _dB_dT
    if nc.space == "bt":
        return nc
    if nc.space != "radiance":
        raise IRSError(f"cannot convert space :{nc.space} to :bt")
    Tb = np.asarray(Tb, dtype=np.float64)
    if len(Tb) != len(nc.nu):
        raise IRSError(f"Tb length {len(Tb)} ≠ covariance channels {len(nc.nu)}; subset_channels first")
    D = 1.0 / np.maximum(_dB_dT(nc.nu, Tb), T_floor)
    return SounderNoiseCovariance(nc.nu.copy(), np.outer(D, D) * nc.cov, "bt")
