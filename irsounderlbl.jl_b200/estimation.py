"""State vectors and Jacobians of forward_model over the C ABI of ``libirs_b200.so``.

Host-side mirror of the reference's estimation interface:

    StateVectorSpec, pack_state, unpack_state,
    state_labels, vmr_range                   src/Estimation/state_vector.jl:253-403
    FullProfile, ColumnScale, PartialColumns,
    partial_column_basis, dfs_partition       src/Estimation/state_vector.jl:40-227
    Jacobian, column, default_fd_steps,
    finite_difference_jacobian                src/Estimation/jacobian_fd.jl:43-165
    analytic_jacobian                         src/Estimation/vmr_jacobian.jl:152-505
    forward_model rrule (pullback)            the ChainRulesCore.rrule over forward_model

The Jacobian itself (line-sum derivatives, RTE adjoint, ILS and dBT/dR channel tail)
runs in the CUDA library (irs_jacobian_batch / irs_vjp_batch); this module only packs
states, maps reduced VMR bases onto the full-profile columns and marshals buffers.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np

from . import _lib
from ._lib import IRSError, StateSpec, check, dptr

VMR_FLOOR = 1e-30  # state_vector.jl:26
SPECIES_NAME = {1: "H₂O", 2: "CO₂", 3: "O₃", 4: "N₂O", 5: "CO", 6: "CH₄", 7: "O₂", 9: "SO₂",
                11: "NH₃"}  # src/Atmosphere/species.jl:40-50


# ------------------------------------------------------------ parameterisations
@dataclass(frozen=True)
class FullProfile:
    """One log-VMR (or VMR) per level (state_vector.jl:47-50)."""
    species: int


@dataclass(frozen=True)
class ColumnScale:
    """One multiplicative column scale, VMR = VMR_ref exp(theta) (state_vector.jl:52-63)."""
    species: int


class PartialColumns:
    """N partial-column scales, VMR = VMR_ref exp(B theta) (state_vector.jl:65-100)."""

    def __init__(self, species: int, basis=None, *, pressure=None, n_blocks=None, edges_hPa=None,
                 taper="boxcar"):
        if basis is None:
            if pressure is None:
                raise IRSError("PartialColumns needs a basis or a pressure grid")
            basis = partial_column_basis(pressure, n_blocks=n_blocks, edges_hPa=edges_hPa, taper=taper)
        B = np.array(basis, dtype=np.float64, ndmin=2)
        if B.shape[1] < 1:
            raise IRSError("PartialColumns needs ≥ 1 block")
        self.species = species
        self.basis = B


def _normalize_param(p):
    return p if isinstance(p, (FullProfile, ColumnScale, PartialColumns)) else FullProfile(int(p))


def _param_basis(p, n: int):
    if isinstance(p, FullProfile):
        return None
    if isinstance(p, ColumnScale):
        return np.ones((n, 1))
    if p.basis.shape[0] != n:
        raise IRSError(f"PartialColumns basis has {p.basis.shape[0]} levels, spec expects {n}")
    return p.basis


def _blocks_equal_count(n: int, nb: int):  # state_vector.jl:122-127
    if not (1 <= nb <= n):
        raise IRSError(f"n_blocks must be in 1:{n}; got {nb}")
    e = [int(np.round(v)) for v in np.linspace(0, n, nb + 1)]  # Julia round: ties to even, as numpy
    return [range(e[m], e[m + 1]) for m in range(nb)]


def _blocks_from_edges(pressure, edges_hPa):  # state_vector.jl:130-150
    ed = sorted((float(e) for e in edges_hPa), reverse=True)
    labels = [sum(1 for e in ed if e > float(pj)) + 1 for pj in pressure]
    blocks, start = [], 0
    for j in range(1, len(labels)):
        if labels[j] != labels[j - 1]:
            blocks.append(range(start, j))
            start = j
    blocks.append(range(start, len(labels)))
    if len(blocks) != len(set(labels)):
        raise IRSError("edges_hPa produced non-contiguous blocks — is `pressure` monotonic?")
    return blocks


def _blocks_to_basis(n: int, blocks, taper: str):  # state_vector.jl:153-180
    N = len(blocks)
    B = np.zeros((n, N))
    if taper == "boxcar":
        for m, blk in enumerate(blocks):
            B[list(blk), m] = 1.0
        return B
    c = [(blk[0] + blk[-1]) / 2 for blk in blocks]  # block centres in index space
    for j in range(n):
        if j <= c[0]:
            B[j, 0] = 1.0
        elif j >= c[-1]:
            B[j, N - 1] = 1.0
        else:
            m = max(i for i, ci in enumerate(c) if ci <= j)
            wR = (j - c[m]) / (c[m + 1] - c[m])
            B[j, m] = 1.0 - wR
            B[j, m + 1] = wR
    return B


def partial_column_basis(pressure_or_n, blocks=None, *, n_blocks=None, edges_hPa=None, taper="boxcar"):
    """partial_column_basis (state_vector.jl:182-212): an n_levels x N partition of unity.

    Either ``partial_column_basis(n_levels, blocks)`` with contiguous 0-based ranges, or
    ``partial_column_basis(pressure, n_blocks=...)`` / ``(pressure, edges_hPa=...)``."""
    if taper not in ("boxcar", "tent"):
        raise IRSError(f"taper must be :boxcar or :tent; got :{taper}")
    if blocks is not None:
        n = int(pressure_or_n)
        flat = [j for b in blocks for j in b]
        if flat != list(range(n)):
            raise IRSError(f"blocks must be contiguous and cover 1:{n} exactly")
        return _blocks_to_basis(n, blocks, taper)
    pressure = np.asarray(pressure_or_n, dtype=np.float64)
    n = len(pressure)
    if edges_hPa is not None:
        if n_blocks is not None:
            raise IRSError("give exactly one of n_blocks / edges_hPa")
        blocks = _blocks_from_edges(pressure, edges_hPa)
    elif n_blocks is not None:
        blocks = _blocks_equal_count(n, n_blocks)
    else:
        raise IRSError("give exactly one of n_blocks / edges_hPa")
    return _blocks_to_basis(n, blocks, taper)


def dfs_partition(dfs, target_dfs: float = 1.0):
    """dfs_partition (state_vector.jl:215-227): contiguous 0-based level blocks of ≈ target DOF."""
    if not target_dfs > 0:
        raise IRSError("target_dfs must be positive")
    n = len(dfs)
    blocks, start, acc = [], 0, 0.0
    for j in range(n):
        acc += max(0.0, float(dfs[j]))
        if acc >= target_dfs and j < n - 1:
            blocks.append(range(start, j + 1))
            start, acc = j + 1, 0.0
    blocks.append(range(start, n))
    return blocks


# ------------------------------------------------------------------ state vector
@dataclass
class VMRBlock:
    """state_vector.jl:229-240: one retrieved gas's state slice and basis (None = identity)."""
    species: int
    basis: Optional[np.ndarray]
    m: int
    range: range


class StateVectorSpec:
    """StateVectorSpec (state_vector.jl:253-309).  Layout: [T][VMR blocks][T_sfc][eps];
    ranges are 0-based Python ranges."""

    def __init__(self, n_levels: int, species: Sequence = (), *, include_temperature: bool = True,
                 include_tsfc: bool = True, include_emissivity: bool = True, log_vmr: bool = True):
        if n_levels <= 0:
            raise IRSError("n_levels must be positive")
        self.n_levels = n_levels
        self.include_temperature = include_temperature
        self.include_tsfc = include_tsfc
        self.include_emissivity = include_emissivity
        self.log_vmr = log_vmr
        idx = 0
        self.temp_range = range(0, 0)
        if include_temperature:
            self.temp_range = range(idx, idx + n_levels)
            idx += n_levels
        self.vmr_blocks = []
        for entry in species:
            p = _normalize_param(entry)
            B = _param_basis(p, n_levels)
            m = n_levels if B is None else B.shape[1]
            self.vmr_blocks.append(VMRBlock(int(p.species), B, m, range(idx, idx + m)))
            idx += m
        self.species = [b.species for b in self.vmr_blocks]
        self.vmr_ranges = [(b.species, b.range) for b in self.vmr_blocks]
        self.tsfc_index = -1
        if include_tsfc:
            self.tsfc_index = idx
            idx += 1
        self.emis_index = -1
        if include_emissivity:
            self.emis_index = idx
            idx += 1
        self.n = idx

    def __len__(self):
        return self.n

    def __repr__(self):
        return (f"StateVectorSpec(n={self.n}, levels={self.n_levels}, T={self.include_temperature}, "
                f"species={[SPECIES_NAME.get(s, s) for s in self.species]}, T_sfc={self.include_tsfc}, "
                f"ε={self.include_emissivity}, log_vmr={self.log_vmr})")


def vmr_range(spec: StateVectorSpec, species: int) -> range:
    """state_vector.jl:311-316"""
    for sp, r in spec.vmr_ranges:
        if sp == int(species):
            return r
    raise IRSError(f"species {SPECIES_NAME.get(int(species), species)} is not in the state vector")


def state_labels(spec: StateVectorSpec):
    """state_vector.jl:324-342 (1-based level indices in the labels, as the reference)."""
    labels = []
    if spec.include_temperature:
        labels += [f"T[{i}]" for i in range(1, spec.n_levels + 1)]
    pre = "logVMR" if spec.log_vmr else "VMR"
    for b in spec.vmr_blocks:
        nm = SPECIES_NAME.get(b.species, str(b.species))
        if b.basis is None:
            labels += [f"{pre}_{nm}[{i}]" for i in range(1, spec.n_levels + 1)]
        elif b.m == 1:
            labels.append(f"logVMRscale_{nm}")
        else:
            labels += [f"logVMRscale_{nm}[{k}]" for k in range(1, b.m + 1)]
    if spec.include_tsfc:
        labels.append("T_sfc")
    if spec.include_emissivity:
        labels.append("emissivity")
    return labels


def pack_state(spec: StateVectorSpec, prof, T_sfc: Optional[float] = None, eps_sfc: float = 1.0):
    """pack_state (state_vector.jl:350-378)."""
    if len(prof.temperature) != spec.n_levels:
        raise IRSError(f"profile has {len(prof.temperature)} levels, spec expects {spec.n_levels}")
    x = np.zeros(spec.n)
    if spec.include_temperature:
        x[spec.temp_range.start:spec.temp_range.stop] = prof.temperature
    for b in spec.vmr_blocks:
        if b.species not in prof.vmr:
            raise IRSError(f"profile is missing retrieved species {b.species}")
        sl = slice(b.range.start, b.range.stop)
        if b.basis is None:
            v = np.asarray(prof.vmr[b.species], dtype=np.float64)
            x[sl] = np.log(np.maximum(v, VMR_FLOOR)) if spec.log_vmr else v
        else:
            x[sl] = 0.0
    if spec.include_tsfc:
        x[spec.tsfc_index] = prof.temperature[0] if T_sfc is None else T_sfc
    if spec.include_emissivity:
        x[spec.emis_index] = eps_sfc
    return x


def unpack_state(spec: StateVectorSpec, x, base_prof):
    """unpack_state (state_vector.jl:380-403) -> (profile, T_sfc, eps_sfc)."""
    from . import AtmosphericProfile
    x = np.asarray(x, dtype=np.float64)
    if len(x) != spec.n:
        raise IRSError(f"state vector length {len(x)} ≠ spec.n {spec.n}")
    T = (x[spec.temp_range.start:spec.temp_range.stop].copy() if spec.include_temperature
         else np.array(base_prof.temperature, dtype=np.float64))
    vmr = {s: np.array(v, dtype=np.float64) for s, v in base_prof.vmr.items()}
    for b in spec.vmr_blocks:
        xv = x[b.range.start:b.range.stop]
        if b.basis is None:
            vmr[b.species] = np.exp(xv) if spec.log_vmr else xv.copy()
        else:
            vmr[b.species] = np.asarray(base_prof.vmr[b.species]) * np.exp(b.basis @ xv)
    prof = AtmosphericProfile(np.array(base_prof.pressure, dtype=np.float64), T,
                              np.array(base_prof.altitude, dtype=np.float64), vmr)
    T_sfc = float(x[spec.tsfc_index]) if spec.include_tsfc else float(T[0])
    eps = float(x[spec.emis_index]) if spec.include_emissivity else 1.0
    return prof, T_sfc, eps


# ------------------------------------------------------------------ Jacobians
@dataclass
class Jacobian:
    """jacobian_fd.jl:43-50: K is n_y x n_x = dy/dx at x0; rows are channels."""
    K: np.ndarray
    spec: StateVectorSpec
    nu: np.ndarray
    x0: np.ndarray
    y0: np.ndarray
    observable: str

    def __repr__(self):
        return f"Jacobian({self.K.shape[0]}×{self.K.shape[1]} ∂{self.observable}/∂x, {self.spec})"


def column(jac: Jacobian, label: str) -> np.ndarray:
    """jacobian_fd.jl:58-63"""
    labels = state_labels(jac.spec)
    if label not in labels:
        raise IRSError(f'no state element labelled "{label}"')
    return jac.K[:, labels.index(label)]


def default_fd_steps(spec: StateVectorSpec, dT=0.5, dlogvmr=1e-3, dvmr=1e-9, dtsfc=0.5, deps=1e-3):
    """default_fd_steps (jacobian_fd.jl:76-92)."""
    s = np.zeros(spec.n)
    if spec.include_temperature:
        s[spec.temp_range.start:spec.temp_range.stop] = dT
    for b in spec.vmr_blocks:
        s[b.range.start:b.range.stop] = dlogvmr if (b.basis is not None or spec.log_vmr) else dvmr
    if spec.include_tsfc:
        s[spec.tsfc_index] = dtsfc
    if spec.include_emissivity:
        s[spec.emis_index] = deps
    return s


def _c_spec(spec: StateVectorSpec, log_vmr: bool, vmr_coupling: bool, observable: str):
    if len(spec.vmr_blocks) > 4:
        raise IRSError("at most 4 retrieved species")
    retr = np.array([b.species for b in spec.vmr_blocks], dtype=np.int32)
    cs = StateSpec()
    cs.n_retrieved = len(retr)
    cs.retrieved = retr.ctypes.data_as(C.POINTER(C.c_int32))
    cs.include_temperature = int(spec.include_temperature)
    cs.include_tsfc = int(spec.include_tsfc)
    cs.include_emissivity = int(spec.include_emissivity)
    cs.log_vmr = int(log_vmr)
    cs.vmr_coupling = int(vmr_coupling)
    cs.observable = 0 if observable == "bt" else 1
    return cs, retr


def _map_reduced(spec: StateVectorSpec, K_lin: np.ndarray, profiles) -> np.ndarray:
    """Map full-profile d/dVMR columns K_lin[n_prof, n_ch, n_full] onto spec's columns:
    d/dlogVMR = VMR d/dVMR (exact: the log chain is that product), then the basis B
    for reduced blocks (VMR = VMR_ref exp(B theta), vmr_jacobian.jl reduced blocks)."""
    n_lev = spec.n_levels
    out = np.zeros(K_lin.shape[:-1] + (spec.n,))
    src = 0
    if spec.include_temperature:
        out[..., spec.temp_range.start:spec.temp_range.stop] = K_lin[..., :n_lev]
        src = n_lev
    for b in spec.vmr_blocks:
        Kb = K_lin[..., src:src + n_lev]
        src += n_lev
        v = np.stack([np.asarray(p.vmr[b.species], dtype=np.float64) for p in profiles])  # [P, n_lev]
        if b.basis is None:
            out[..., b.range.start:b.range.stop] = Kb * v[:, None, :] if spec.log_vmr else Kb
        else:
            out[..., b.range.start:b.range.stop] = (Kb * v[:, None, :]) @ b.basis
    for k in (spec.tsfc_index, spec.emis_index):
        if k >= 0:
            out[..., k] = K_lin[..., src]
            src += 1
    return out


def _check_observable(observable):
    if observable not in ("bt", "radiance"):
        raise IRSError(f"observable must be :bt or :radiance, got :{observable}")


def analytic_jacobian_batch(profiles, linelists, spec: StateVectorSpec, *, sounder=None, geoms=None,
                            T_sfcs=None, eps_sfcs=None, observable="bt", vmr_coupling=True, backend=None,
                            line_mixing=None, **kw):
    """analytic_jacobian (vmr_jacobian.jl:152-505) for a batch of profiles on the GPU.

    Returns (nu, K[n_prof, n_ch, n_state], y[n_prof, n_ch]).  The line set is frozen
    (dptmn = 0) as the reference does; the line sum is FP32 with Kahan-compensated
    tiles, transmittances and radiance derivatives FP64."""
    from . import (IASIInstrument, _prepare, _ProfileBatch, default_context, fm_options, nadir_geometry,
                   sounder_grid)
    _check_observable(observable)
    ctx = backend or default_context()
    sounder = sounder or IASIInstrument()
    n = len(profiles)
    for p in profiles:
        if len(p.temperature) != spec.n_levels:
            raise IRSError(f"profile has {len(p.temperature)} levels, spec expects {spec.n_levels}")
        for b in spec.vmr_blocks:
            if b.species not in p.vmr:
                raise IRSError(f"profile is missing retrieved species {b.species}")
    geoms = geoms or [nadir_geometry()] * n
    T_sfcs = T_sfcs if T_sfcs is not None else [None] * n
    eps_sfcs = eps_sfcs if eps_sfcs is not None else [1.0] * n
    _prepare(ctx, linelists, line_mixing)
    kw.pop("dptmn", None)
    o = fm_options(line_mixing=line_mixing, dptmn=0.0, **kw)
    reduced = any(b.basis is not None for b in spec.vmr_blocks)
    # reduced blocks are computed as full-profile d/dVMR columns and mapped on the host
    cs, keep = _c_spec(spec, spec.log_vmr and not reduced, vmr_coupling, observable)
    batch = _ProfileBatch(profiles, T_sfcs, [g.mu for g in geoms], eps_sfcs)
    s = sounder.c_struct()
    nu = sounder_grid(sounder)
    n_full = C.c_int64()
    check(ctx.lib.irs_state_size(C.byref(cs), spec.n_levels, C.byref(n_full)))
    Kc = np.empty((n, n_full.value, len(nu)))
    y = np.empty((n, len(nu)))
    check(ctx.lib.irs_jacobian_batch(ctx.h, batch.arr, n, C.byref(s), C.byref(o), C.byref(cs), dptr(Kc),
                                     dptr(y)))
    K = np.ascontiguousarray(np.transpose(Kc, (0, 2, 1)))  # [n_prof, n_ch, n_full]
    if reduced:
        K = _map_reduced(spec, K, profiles)
    return nu, K, y


def analytic_jacobian(prof, linelists, spec: StateVectorSpec, *, sounder=None, iasi=None, geom=None,
                      T_sfc: Optional[float] = None, eps_sfc: float = 1.0, observable="bt",
                      vmr_coupling=True, backend=None, line_mixing=None, **kw) -> Jacobian:
    """analytic_jacobian (vmr_jacobian.jl:152-505) -> Jacobian."""
    sounder = iasi if iasi is not None else sounder
    from . import nadir_geometry
    nu, K, y = analytic_jacobian_batch([prof], linelists, spec, sounder=sounder,
                                       geoms=[geom or nadir_geometry()], T_sfcs=[T_sfc], eps_sfcs=[eps_sfc],
                                       observable=observable, vmr_coupling=vmr_coupling, backend=backend,
                                       line_mixing=line_mixing, **kw)
    x0 = pack_state(spec, prof, T_sfc=T_sfc, eps_sfc=eps_sfc)
    return Jacobian(np.asarray(K[0]), spec, nu, x0, y[0], observable)


def finite_difference_jacobian(prof, linelists, spec: StateVectorSpec, *, T_sfc: Optional[float] = None,
                               eps_sfc: float = 1.0, observable="bt", steps=None, method="central",
                               fm_kwargs=None, backend=None, geom=None, verbose=False) -> Jacobian:
    """finite_difference_jacobian (jacobian_fd.jl:111-165).

    All perturbed states go to the GPU forward model as one batch (2 n_state + 1
    profiles for :central), instead of one forward_model call per perturbation."""
    from . import forward_model_batch, nadir_geometry
    _check_observable(observable)
    if method not in ("central", "forward"):
        raise IRSError(f"method must be :central or :forward, got :{method}")
    steps = default_fd_steps(spec) if steps is None else np.asarray(steps, dtype=np.float64)
    if len(steps) != spec.n:
        raise IRSError(f"steps length {len(steps)} ≠ spec.n {spec.n}")
    labels = state_labels(spec)
    for i, d in enumerate(steps):
        if d == 0.0:
            raise IRSError(f"zero FD step for state element {i + 1} ({labels[i]})")
    kw = dict(dptmn=0.0)
    kw.update(fm_kwargs or {})
    x0 = pack_state(spec, prof, T_sfc=T_sfc, eps_sfc=eps_sfc)
    xs = [x0]
    for i in range(spec.n):
        xp = x0.copy()
        xp[i] += steps[i]
        xs.append(xp)
        if method == "central":
            xm = x0.copy()
            xm[i] -= steps[i]
            xs.append(xm)
    states = [unpack_state(spec, x, prof) for x in xs]
    g = geom or nadir_geometry()
    nu, R, BT = forward_model_batch([s[0] for s in states], linelists, geoms=[g] * len(states),
                                    T_sfcs=[s[1] for s in states], eps_sfcs=[s[2] for s in states],
                                    backend=backend, **kw)
    Y = BT if observable == "bt" else R
    y0 = Y[0]
    K = np.empty((len(y0), spec.n))
    for i in range(spec.n):
        if method == "central":
            K[:, i] = (Y[1 + 2 * i] - Y[2 + 2 * i]) / (2 * steps[i])
        else:
            K[:, i] = (Y[1 + i] - y0) / steps[i]
    return Jacobian(K, spec, nu, x0, y0, observable)


def forward_model_rrule(prof, linelists, spec: StateVectorSpec, *, sounder=None, geom=None,
                        T_sfc: Optional[float] = None, eps_sfc: float = 1.0, observable="bt", backend=None,
                        line_mixing=None, **kw):
    """The ChainRulesCore.rrule of forward_model with respect to the packed state:
    returns (y, pullback) with pullback(dy) = K^T dy (irs_vjp_batch on the GPU)."""
    from . import (IASIInstrument, _prepare, _ProfileBatch, default_context, fm_options, nadir_geometry,
                   sounder_grid)
    _check_observable(observable)
    if any(b.basis is not None for b in spec.vmr_blocks):
        jac = analytic_jacobian(prof, linelists, spec, sounder=sounder, geom=geom, T_sfc=T_sfc,
                                eps_sfc=eps_sfc, observable=observable, backend=backend,
                                line_mixing=line_mixing, **kw)
        return jac.y0, lambda dy: jac.K.T @ np.asarray(dy, dtype=np.float64)
    ctx = backend or default_context()
    sounder = sounder or IASIInstrument()
    _prepare(ctx, linelists, line_mixing)
    kw.pop("dptmn", None)
    o = fm_options(line_mixing=line_mixing, dptmn=0.0, **kw)
    g = geom or nadir_geometry()
    batch = _ProfileBatch([prof], [T_sfc], [g.mu], [eps_sfc])
    cs, keep = _c_spec(spec, spec.log_vmr, True, observable)
    s = sounder.c_struct()
    n_ch = len(sounder_grid(sounder))
    y = np.empty(n_ch)
    # the forward value comes from the same call as the first pullback
    cache = {}

    def pullback(dy):
        dy = np.ascontiguousarray(dy, dtype=np.float64)
        if dy.shape != (n_ch,):
            raise IRSError(f"cotangent has shape {dy.shape}, expected ({n_ch},)")
        dx = np.empty(spec.n)
        check(ctx.lib.irs_vjp_batch(ctx.h, batch.arr, 1, C.byref(s), C.byref(o), C.byref(cs), dptr(dy),
                                    dptr(dx), dptr(y)))
        cache["y"] = y.copy()
        return dx

    pullback(np.zeros(n_ch))
    return cache["y"], pullback
