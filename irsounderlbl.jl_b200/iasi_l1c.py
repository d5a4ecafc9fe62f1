"""IASI Level-1C reader for the EPS native (.nat) product, and the batched retrieval of a
granule's fields of view (src/Sensor/iasi_l1c.jl, §8 "next": L1C -> batched OE).

The record framing (20-byte Generic Record Header: class, subclass, big-endian record
size), the MDR field offsets and the GIADR scale-factor layout are facts of the EPS
format that the reference's reader fixes (iasi_l1c.jl:22-48, 122-156); they are the
same numbers here.  The MDR fields are decoded with numpy big-endian views, one scan
line (30 steps x 4 pixels) at a time, instead of per-sample reads.
"""
from __future__ import annotations

import os
from dataclasses import dataclass, field
from typing import Dict, Optional, Sequence, Tuple

import numpy as np

from ._lib import IRSError

GRH_SIZE = 20            # Generic Record Header bytes
CLASS_MPHR, CLASS_GIADR, CLASS_MDR = 1, 5, 8
MDR_SUBCLASS = 2         # IASI L1C science MDR
NSTP, NPIX, NSPEC = 30, 4, 8700
WNO1, WNOD, NWNO = 645.0, 0.25, 8461
OFF_GEOLOC = 255893      # GGeoSondLoc [NSTP,NPIX,2] >i4 x1e-6 deg (lon, lat)
OFF_ANG_SAT = 256853     # GGeoSondAnglesMETOP [NSTP,NPIX,2] >i4 x1e-6 deg (zenith, azimuth)
OFF_ANG_SUN = 263813     # GGeoSondAnglesSun [NSTP,NPIX,2]
OFF_NSFIRST = 276782
OFF_NSLAST = 276786
OFF_SPEC = 276790        # GS1cSpect [NSTP,NPIX,NSPEC] >i2
OFF_CLDFRAC = 2728548    # GEUMAvhrr1BCldFrac [NSTP,NPIX] u1 (%)
OFF_LNDFRAC = 2728668    # GEUMAvhrr1BLandFrac [NSTP,NPIX] u1 (%)
RADFAC = 1.0e5           # W/(m^2 sr m^-1) -> mW/(m^2 sr cm^-1)
C1, C2 = 1.191042953e-5, 1.4387769   # planck.jl


def brightness_temperature(nu, R):
    """brightness_temperature (planck.jl:37-45), elementwise; 0 where R <= 0."""
    nu = np.asarray(nu, dtype=np.float64)
    R = np.asarray(R, dtype=np.float64)
    with np.errstate(divide="ignore", invalid="ignore"):
        bt = C2 * nu / np.log1p(C1 * nu ** 3 / R)
    return np.where(R > 0, bt, 0.0)


@dataclass
class IASIL1CGranule:
    """IASIL1CGranule (iasi_l1c.jl:57-100): spc is [nfov, nwno] here (row per FOV)."""
    file: str
    mph: Dict[str, str]
    wno: np.ndarray
    spc: np.ndarray
    is_bt: bool
    lat: np.ndarray
    lon: np.ndarray
    zen: np.ndarray
    azi: np.ndarray
    sza: np.ndarray
    saa: np.ndarray
    sra: np.ndarray
    cld: np.ndarray
    lnd: np.ndarray
    line: np.ndarray
    step: np.ndarray
    pix: np.ndarray


def nfov(g: IASIL1CGranule) -> int:
    return len(g.lat)


def measurement(g: IASIL1CGranule, i: int):
    """measurement (iasi_l1c.jl:320-330): (wavenumbers, spectrum of FOV i)."""
    return g.wno, g.spc[i]


def cloud_fraction(g: IASIL1CGranule) -> np.ndarray:
    return g.cld


def solar_reflection_angle(g: IASIL1CGranule) -> np.ndarray:
    return g.sra


def _solar_reflection_angle(zen, azi, sza, saa):
    """Sun-glint angle (iasi_l1c.jl:300-312): cos phi = cos ts cos ti - sin ts sin ti cos(ps - pi)."""
    r = np.radians
    c = np.cos(r(sza)) * np.cos(r(zen)) - np.sin(r(sza)) * np.sin(r(zen)) * np.cos(r(saa) - r(azi))
    return np.degrees(np.arccos(np.clip(c, -1.0, 1.0)))


def _parse_mphr(b: bytes) -> Dict[str, str]:
    out = {}
    for line in b.decode("latin-1").split("\n"):
        if not line.strip() or "=" not in line:
            continue
        k, v = line.split("=", 1)
        if k.strip():
            out[k.strip()] = v.strip()
    return out


def _parse_scalefactors(rec: bytes) -> np.ndarray:
    """GIADR scale factors (iasi_l1c.jl:122-141) -> per-sample scale over the 8700 samples."""
    be = lambda o, n: np.frombuffer(rec, ">i2", count=n, offset=o).astype(int)
    nb = int(be(20, 1)[0])
    if not 1 <= nb <= 10:
        raise IRSError(f"IASI L1C: implausible scale-band count {nb} in GIADR")
    first, last, expo = be(22, 10), be(42, 10), be(62, 10)
    off = first[0] - 1
    scale = np.ones(NSPEC)
    for b in range(nb):
        lo = min(max(first[b] - off, 1), NSPEC)
        hi = min(max(last[b] - off, 1), NSPEC)
        if lo <= hi:
            scale[lo - 1:hi] = 10.0 ** (-expo[b])
    return scale


def _default_scale() -> np.ndarray:  # iasi_l1c.jl:144-152
    scale = np.ones(NSPEC)
    for lo, hi, e in ((1, 1990, 7), (1991, 5116, 8), (5117, 8461, 9)):
        scale[lo - 1:hi] = 10.0 ** (-e)
    return scale


def read_iasi_l1c(path: str, *, bright: bool = False, wnolim: Tuple[float, float] = (WNO1, 2760.0),
                  cldlim=None, latlim=None, lonlim=None, zenlim=None, szalim=None, sralim=None,
                  max_fov: Optional[int] = None, validate: bool = True) -> IASIL1CGranule:
    """read_iasi_l1c (iasi_l1c.jl:186-272).  Radiances in mW/(m^2 sr cm^-1), or BT [K]."""
    i0 = int(round((wnolim[0] - WNO1) / WNOD))
    i1 = int(round((wnolim[1] - WNO1) / WNOD))
    if not 0 <= i0 <= i1 <= NWNO - 1:
        raise IRSError(f"wnolim {tuple(wnolim)} outside the IASI grid 645–2760 cm⁻¹")
    wno = WNO1 + np.arange(i0, i1 + 1) * WNOD

    def inwin(x, lim):
        return np.ones(np.shape(x), bool) if lim is None else (x >= lim[0]) & (x <= lim[1])

    mph: Dict[str, str] = {}
    scale = None
    cols = {k: [] for k in ("spc", "lat", "lon", "zen", "azi", "sza", "saa", "sra", "cld", "lnd", "line",
                            "step", "pix")}
    nq = NSTP * NPIX
    steps = np.repeat(np.arange(1, NSTP + 1), NPIX)
    pixs = np.tile(np.arange(1, NPIX + 1), NSTP)
    kept = 0
    with open(path, "rb") as fh:
        fsize = os.fstat(fh.fileno()).st_size
        pos = 0
        nline = 0
        while pos + GRH_SIZE <= fsize:
            fh.seek(pos)
            grh = fh.read(GRH_SIZE)
            rclass, subclass = grh[0], grh[2]
            rsize = int(np.frombuffer(grh, ">u4", count=1, offset=3)[0])
            if rsize < GRH_SIZE:
                break
            fh.seek(pos)
            rec = fh.read(rsize)
            if len(rec) != rsize:
                break
            pos += rsize
            if rclass == CLASS_MPHR:
                mph = _parse_mphr(rec[GRH_SIZE:])
            elif rclass == CLASS_GIADR and (subclass == 1 or rsize == 84):
                if scale is None:
                    scale = _parse_scalefactors(rec)
            elif rclass == CLASS_MDR and subclass == MDR_SUBCLASS:
                nline += 1
                if scale is None:
                    scale = _default_scale()
                i4 = lambda o: np.frombuffer(rec, ">i4", count=2 * nq, offset=o).reshape(nq, 2) * 1.0e-6
                geo, sat, sun = i4(OFF_GEOLOC), i4(OFF_ANG_SAT), i4(OFF_ANG_SUN)
                lon, lat = geo[:, 0], geo[:, 1]
                zen, azi, sza, saa = sat[:, 0], sat[:, 1], sun[:, 0], sun[:, 1]
                sra = _solar_reflection_angle(zen, azi, sza, saa)
                cld = np.frombuffer(rec, "u1", count=nq, offset=OFF_CLDFRAC).astype(np.float64)
                lnd = np.frombuffer(rec, "u1", count=nq, offset=OFF_LNDFRAC).astype(np.float64)
                ok = (inwin(lat, latlim) & inwin(lon, lonlim) & inwin(zen, zenlim) & inwin(sza, szalim)
                      & inwin(sra, sralim) & inwin(cld, cldlim))
                q = np.flatnonzero(ok)
                if max_fov is not None:
                    q = q[:max(0, max_fov - kept)]
                if len(q):
                    raw = np.frombuffer(rec, ">i2", count=nq * NSPEC, offset=OFF_SPEC).reshape(nq, NSPEC)
                    rad = raw[q, i0:i1 + 1].astype(np.float64) * scale[i0:i1 + 1] * RADFAC
                    cols["spc"].append(brightness_temperature(wno, rad) if bright else rad)
                    for k, v in (("lat", lat), ("lon", lon), ("zen", zen), ("azi", azi), ("sza", sza),
                                 ("saa", saa), ("sra", sra), ("cld", cld), ("lnd", lnd), ("step", steps),
                                 ("pix", pixs)):
                        cols[k].append(v[q])
                    cols["line"].append(np.full(len(q), nline))
                    kept += len(q)
                if max_fov is not None and kept >= max_fov:
                    break
    cat = {k: (np.concatenate(v) if v else np.zeros(0)) for k, v in cols.items()}
    spc = np.concatenate(cols["spc"]) if cols["spc"] else np.zeros((0, len(wno)))
    if validate and len(cat["lat"]):
        if not (np.all(np.abs(cat["lat"]) <= 90.0) and np.all(np.abs(cat["lon"]) <= 180.0)):
            raise IRSError("IASI L1C: lat/lon out of range — MDR offsets likely don't match this product "
                           "version (geoloc parse). Verify against the granule.")
        if not bright and len(wno):
            bt = float(brightness_temperature(wno[0], spc[0, 0]))
            if not 100.0 <= bt <= 400.0:
                raise IRSError(f"IASI L1C: BT={bt:.1f} K out of 100–400 K — radiance scaling/offsets likely "
                               "wrong. Verify against the granule.")
    return IASIL1CGranule(str(path), mph, wno, spc, bright, cat["lat"], cat["lon"], cat["zen"], cat["azi"],
                          cat["sza"], cat["saa"], cat["sra"], cat["cld"], cat["lnd"], cat["line"].astype(int),
                          cat["step"].astype(int), cat["pix"].astype(int))


def retrieve_granule(granule: IASIL1CGranule, spec, base_profs, linelists, *, xa, Sa, nedt_280K: float = 0.2,
                     channels: Optional[np.ndarray] = None, fovs: Optional[Sequence[int]] = None,
                     h_sat_km: float = 817.0, **oe_kw):
    """Batched optimal estimation of a granule's FOVs on the GPU: the measured BT of each
    FOV (the granule read with bright=True) is the observation, its noise the scene NEdT
    (scene_nedt at nedt_280K), its geometry the satellite zenith angle, and all FOVs run
    as one optimal_estimation_batch.  base_profs: one profile per FOV or one shared;
    channels: indices into granule.wno (default all).  The forward model's sounder is the
    IASI grid restricted to the granule's channel window."""
    from . import Sounder, ViewingGeometry
    from .estimation import optimal_estimation_batch, scene_nedt
    if not granule.is_bt:
        raise IRSError("retrieve_granule needs brightness temperatures: read the granule with bright=True")
    idx = np.arange(nfov(granule)) if fovs is None else np.asarray(fovs, int)
    ch = np.arange(len(granule.wno)) if channels is None else np.asarray(channels, int)
    y = granule.spc[np.ix_(idx, ch)]
    snd = Sounder.make(float(granule.wno[0]), float(granule.wno[-1]), WNOD, opd_max=2.0, fwhm_gauss=0.5)
    keep = np.zeros(len(granule.wno), bool)
    keep[ch] = True
    y_full = granule.spc[idx]
    se = np.stack([scene_nedt(granule.wno, b, nedt_280K=nedt_280K) ** 2 for b in y_full])
    profs = list(base_profs) if isinstance(base_profs, (list, tuple)) else [base_profs] * len(idx)
    geoms = [ViewingGeometry(float(z)) for z in granule.zen[idx]]
    r = optimal_estimation_batch(y_full, spec, profs, linelists, xa=xa, Sa=Sa, Se=se, sounder=snd, geoms=geoms,
                                 channel_mask=keep, **oe_kw)
    r["fovs"] = idx
    return r
