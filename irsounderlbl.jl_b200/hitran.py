"""HITRAN line-list ingest: the 160-character .par records, the parsed-list cache and
the list filters (src/HITRAN/linelist.jl:60-106, fetch.jl:12-33, cache.jl:9-198).

Host-side file handling, as in the reference.  The cache stores the parsed 56-byte
HITRANLine records as one .npy blob (the reference stores the same isbits vector in
a .jld2 file), keyed by the .par file's absolute path, size, mtime and the cache
version, and written through a temporary file and a rename.
"""
from __future__ import annotations

import hashlib
import os
from pathlib import Path
from typing import Iterable, Optional

import numpy as np

from ._lib import LINE_DTYPE, IRSError

LINELIST_CACHE_VERSION = 1      # cache.jl:9
_CACHE_DIR: Optional[str] = None


def parse_hitran_par(record: str) -> tuple:
    """parse_hitran_par (linelist.jl:86-106): one record -> HITRANLine fields
    (mol_id, iso_id, ν, S, A, γ_air, γ_self, E'', n_air, δ_air).  Raises ValueError on a
    malformed record; iso '0' is parsed as 0 (HITRAN's 10th isotopologue)."""
    return (int(record[0:2]), int(record[2:3]), float(record[3:15]), float(record[15:25]),
            float(record[25:35]), np.float32(record[35:40].strip()), np.float32(record[40:45].strip()),
            float(record[45:55]), np.float32(record[55:59].strip()), np.float32(record[59:67].strip()))


def _records(path: str) -> np.ndarray:
    rows = []
    with open(path) as fh:
        for rec in fh:
            rec = rec.rstrip("\n")
            if len(rec) < 67:          # short or blank records are skipped (fetch.jl:19)
                continue
            try:
                rows.append(parse_hitran_par(rec))
            except ValueError:         # malformed records are skipped (fetch.jl:26-28)
                continue
    return np.array(rows, dtype=LINE_DTYPE) if rows else np.zeros(0, dtype=LINE_DTYPE)


def load_hitran_par(filepath: str, nu_min: Optional[float] = None, nu_max: Optional[float] = None):
    """load_hitran_par (fetch.jl:12-33) -> HITRANLinelist (sorted by wavenumber)."""
    from . import HITRANLinelist
    if not os.path.isfile(filepath):
        raise IRSError(f"File not found: {filepath}")
    L = _records(filepath)
    return HITRANLinelist(_window(L, nu_min, nu_max))


def _window(L: np.ndarray, nu_min, nu_max) -> np.ndarray:
    m = np.ones(len(L), dtype=bool)
    if nu_min is not None:
        m &= L["wavenumber"] >= nu_min
    if nu_max is not None:
        m &= L["wavenumber"] <= nu_max
    return L[m]


def filter_linelist(ll, a: float, b: Optional[float] = None):
    """filter_linelist (linelist.jl:60-80): by [ν_min, ν_max] when two bounds are given,
    else by intensity >= S_min."""
    from . import HITRANLinelist
    L = ll.lines
    keep = (L["wavenumber"] >= a) & (L["wavenumber"] <= b) if b is not None else L["intensity"] >= a
    return HITRANLinelist(L[keep])


def linelist_cache_dir() -> str:
    """linelist_cache_dir (cache.jl:23-36): IRSOUNDER_LINELIST_CACHE, else the directory set
    by set_linelist_cache_dir, else ~/.cache/irsounder_b200/linelists; created if absent."""
    d = os.environ.get("IRSOUNDER_LINELIST_CACHE") or _CACHE_DIR or \
        os.path.join(os.path.expanduser("~"), ".cache", "irsounder_b200", "linelists")
    os.makedirs(d, exist_ok=True)
    return d


def set_linelist_cache_dir(path: Optional[str]) -> None:
    """set_linelist_cache_dir! (cache.jl:46-53) for this process (None clears it)."""
    global _CACHE_DIR
    _CACHE_DIR = None if path is None else str(path)


def clear_linelist_cache() -> int:
    """clear_linelist_cache (cache.jl:61-72): removes the cache blobs, returns how many."""
    d = linelist_cache_dir()
    n = 0
    for f in Path(d).glob("linelist_*.npy"):
        f.unlink()
        n += 1
    return n


def _cache_path(parpath: str) -> str:                  # cache.jl:77-81
    st = os.stat(parpath)
    key = f"{os.path.abspath(parpath)}|{st.st_size}|{st.st_mtime_ns}|{LINELIST_CACHE_VERSION}"
    return os.path.join(linelist_cache_dir(), "linelist_" + hashlib.sha1(key.encode()).hexdigest()[:16] + ".npy")


def _save_cache(cpath: str, lines: np.ndarray) -> None:  # cache.jl:83-96
    tmp = f"{cpath}.tmp.{os.getpid()}.npy"
    np.save(tmp, np.ascontiguousarray(lines, dtype=LINE_DTYPE), allow_pickle=False)
    os.replace(tmp, cpath)


def _load_cache(cpath: str) -> Optional[np.ndarray]:     # cache.jl:98-111
    if not os.path.isfile(cpath):
        return None
    try:
        a = np.load(cpath, allow_pickle=False)
        return a if a.dtype == LINE_DTYPE else None
    except (OSError, ValueError):
        return None


def load_linelist(parpath: str, isotopologues: Optional[Iterable[int]] = None, *, nu_min: Optional[float] = None,
                  nu_max: Optional[float] = None, cache: bool = True, rebuild: bool = False):
    """load_linelist (cache.jl:129-198).  With isotopologues, loads and merges
    "{base}.par" (iso 1) and "{base}_iso{k}.par"; a missing file raises."""
    from . import HITRANLinelist
    if isotopologues is not None:
        parts, missing = [], []
        for iso in isotopologues:
            f = f"{parpath}.par" if iso == 1 else f"{parpath}_iso{iso}.par"
            if not os.path.isfile(f):
                missing.append(f)
                continue
            parts.append(load_linelist(f, nu_min=nu_min, nu_max=nu_max, cache=cache, rebuild=rebuild).lines)
        if missing:
            raise IRSError("load_linelist: requested isotopologue(s) with no .par file on disk: " + ", ".join(missing)
                           + f" (base={parpath}, isotopologues={list(isotopologues)})")
        L = np.concatenate(parts) if parts else np.zeros(0, dtype=LINE_DTYPE)
        if len(L) == 0:
            raise IRSError(f"No lines found for base={parpath}, isotopologues={list(isotopologues)} "
                           "(files present but empty in the requested window)")
        return HITRANLinelist(L)
    if not os.path.isfile(parpath):
        raise IRSError(f"File not found: {parpath}")
    if cache:
        cpath = _cache_path(parpath)
        L = None if rebuild else _load_cache(cpath)
        if L is None:
            L = _records(parpath)       # the whole file; the window is applied in memory
            _save_cache(cpath, L)
    else:
        L = _records(parpath)
    return HITRANLinelist(_window(L, nu_min, nu_max))
