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


def vjp_batch(profiles, linelists, spec: StateVectorSpec, dy, *, sounder=None, geoms=None, T_sfcs=None,
              eps_sfcs=None, observable="bt", vmr_coupling=True, backend=None, line_mixing=None, **kw):
    """Pullbacks dx = K^T dy of a batch (irs_vjp_batch: reverse mode on the GPU, K is never
    formed).  dy is [n_prof, n_ch]; returns (y[n_prof, n_ch], dx[n_prof, n_state])."""
    from . import (IASIInstrument, _prepare, _ProfileBatch, default_context, fm_options, nadir_geometry,
                   sounder_grid)
    _check_observable(observable)
    ctx = backend or default_context()
    sounder = sounder or IASIInstrument()
    n = len(profiles)
    nu = sounder_grid(sounder)
    dy = np.ascontiguousarray(np.broadcast_to(np.asarray(dy, dtype=np.float64), (n, len(nu))))
    geoms = geoms or [nadir_geometry()] * n
    T_sfcs = T_sfcs if T_sfcs is not None else [None] * n
    eps_sfcs = eps_sfcs if eps_sfcs is not None else [1.0] * n
    _prepare(ctx, linelists, line_mixing)
    kw.pop("dptmn", None)
    o = fm_options(line_mixing=line_mixing, dptmn=0.0, **kw)
    reduced = any(b.basis is not None for b in spec.vmr_blocks)
    cs, keep = _c_spec(spec, spec.log_vmr and not reduced, vmr_coupling, observable)
    batch = _ProfileBatch(profiles, T_sfcs, [g.mu for g in geoms], eps_sfcs)
    s = sounder.c_struct()
    n_full = C.c_int64()
    check(ctx.lib.irs_state_size(C.byref(cs), spec.n_levels, C.byref(n_full)))
    dx = np.empty((n, n_full.value))
    y = np.empty((n, len(nu)))
    check(ctx.lib.irs_vjp_batch(ctx.h, batch.arr, n, C.byref(s), C.byref(o), C.byref(cs), dptr(dy), dptr(dx),
                                dptr(y)))
    if reduced:  # the reduced columns are linear maps of the full ones: the same map on dx
        dx = _map_reduced(spec, dx[:, None, :], profiles)[:, 0, :]
    return y, dx


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


# ------------------------------------------------------------------ a-priori and noise
def _corr(kernel: str, r):
    """sa_builder.jl:28-32"""
    if kernel == "exponential":
        return np.exp(-r)
    if kernel == "matern32":
        return (1.0 + np.sqrt(3.0) * r) * np.exp(-np.sqrt(3.0) * r)
    if kernel == "matern52":
        return (1.0 + np.sqrt(5.0) * r + 5.0 * r * r / 3.0) * np.exp(-np.sqrt(5.0) * r)
    return np.exp(-0.5 * r * r)


def _resolve_sigma(sig, n, name):
    if np.isscalar(sig):
        if not sig > 0:
            raise IRSError(f"{name} must be positive")
        return np.full(n, float(sig))
    v = np.asarray(sig, dtype=np.float64)
    if len(v) != n:
        raise IRSError(f"{name} must be a scalar or length n_levels={n}; got {len(v)}")
    if not np.all(v > 0):
        raise IRSError(f"{name} entries must all be positive")
    return v


def build_sa(spec: StateVectorSpec, base_prof, sigma_T=2.0, L_T=1.0, sigma_vmr=0.5, L_vmr=1.0, sigma_col=0.2,
             sigma_tsfc=2.0, sigma_emis=0.02, kernel="matern52", jitter=0.0) -> np.ndarray:
    """build_sa (sa_builder.jl:101-153): block a-priori covariance correlated in log-pressure.
    sigma_vmr / L_vmr / sigma_col may be dicts keyed by species."""
    if kernel not in ("matern52", "matern32", "exponential", "sqexp"):
        raise IRSError(f"kernel must be :matern52, :matern32, :exponential, or :sqexp; got :{kernel}")
    p = np.asarray(base_prof.pressure, dtype=np.float64)
    if len(p) != spec.n_levels:
        raise IRSError(f"base_prof has {len(p)} levels, spec expects {spec.n_levels}")
    if not np.all(p > 0):
        raise IRSError("pressures must be positive for log-pressure correlation")
    if jitter < 0:
        raise IRSError("jitter must be ≥ 0")
    logp = np.log(p)
    dist = np.abs(logp[:, None] - logp[None, :])
    Sa = np.zeros((spec.n, spec.n))

    def per_species(v, s, what):
        if isinstance(v, dict):
            if s not in v:
                raise IRSError(f"{what} has no entry for {SPECIES_NAME.get(s, s)}")
            return v[s]
        return v

    if spec.include_temperature:
        sg = _resolve_sigma(sigma_T, spec.n_levels, "σ_T")
        r = spec.temp_range
        Sa[r.start:r.stop, r.start:r.stop] = np.outer(sg, sg) * _corr(kernel, dist / float(L_T))
    for b in spec.vmr_blocks:
        sl = slice(b.range.start, b.range.stop)
        if b.basis is None:
            sg = _resolve_sigma(per_species(sigma_vmr, b.species, "σ_vmr"), spec.n_levels, "σ_vmr")
            L = float(per_species(L_vmr, b.species, "L_vmr"))
            if not L > 0:
                raise IRSError("L_vmr must be positive")
            Sa[sl, sl] = np.outer(sg, sg) * _corr(kernel, dist / L)
        else:
            sc = _resolve_sigma(per_species(sigma_col, b.species, "σ_col"), b.m, "σ_col")
            Sa[sl, sl] = np.diag(sc ** 2)
    if spec.include_tsfc:
        Sa[spec.tsfc_index, spec.tsfc_index] = float(sigma_tsfc) ** 2
    if spec.include_emissivity:
        Sa[spec.emis_index, spec.emis_index] = float(sigma_emis) ** 2
    if jitter > 0:
        Sa[np.diag_indices(spec.n)] *= 1.0 + jitter
    return Sa


def _dB_dT(nu, T):
    """planck.jl:67-71 (host copy for covariance set-up)."""
    c1, c2 = 1.191042953e-5, 1.4387769
    x = c2 * nu / T
    ex = np.exp(x)
    return c1 * c2 * nu ** 4 * ex / (T * T * (ex - 1.0) ** 2)


def _ils_noise_autocorr(dnu_sample: float, fwhm_gauss: float, max_lag: int = 4) -> np.ndarray:
    """_ils_noise_autocorr (covariance.jl:28-36): channel-lag correlation of the Gaussian
    apodisation weights exp(-(k dnu)^2 / 2 s^2), s = fwhm / (2 sqrt(2 ln 2))."""
    if fwhm_gauss <= 0.0:
        return np.array([1.0] + [0.0] * max_lag)
    s = fwhm_gauss / (2.0 * np.sqrt(2.0 * np.log(2.0)))
    K = max_lag + 6
    w = np.exp(-((np.arange(-K, K + 1) * dnu_sample) ** 2) / (2.0 * s * s))
    R0 = float(np.sum(w * w))
    return np.array([1.0] + [float(np.sum(w[:len(w) - k] * w[k:])) / R0 for k in range(1, max_lag + 1)])


def apodized_measurement_covariance(nu, sigma, dnu_sample: float = 0.25, fwhm_gauss: float = 0.5,
                                    max_lag: int = 4) -> np.ndarray:
    """apodized_measurement_covariance (covariance.jl:63-81): Se[i, j] = s_i s_j rho(lag),
    lag = round(|nu_i - nu_j| / dnu_sample) <= max_lag (banded for contiguous channels)."""
    nu = np.asarray(nu, dtype=np.float64)
    n = len(nu)
    sv = np.full(n, float(sigma)) if np.ndim(sigma) == 0 else np.asarray(sigma, dtype=np.float64)
    if len(sv) != n:
        raise IRSError(f"σ must be a scalar or length(ν)={n}; got {len(sv)}")
    rho = _ils_noise_autocorr(dnu_sample, fwhm_gauss, max_lag)
    lag = np.rint(np.abs(nu[:, None] - nu[None, :]) / dnu_sample).astype(np.int64)
    Se = np.where(lag <= max_lag, np.outer(sv, sv) * rho[np.minimum(lag, max_lag)], 0.0)
    return Se


def scene_measurement_covariance(nu, Tb_scene, nedt_280K=0.25, T_ref=280.0, **kw) -> np.ndarray:
    """scene_measurement_covariance (covariance.jl:125-130): scene NEdT on the diagonal,
    apodisation correlations off it."""
    return apodized_measurement_covariance(nu, scene_nedt(nu, Tb_scene, nedt_280K, T_ref), **kw)


def scene_nedt(nu, Tb_scene, nedt_280K=0.25, T_ref=280.0) -> np.ndarray:
    """scene_nedt (covariance.jl:106-117): NEdT at the scene BT from the NEdT at T_ref."""
    nu = np.asarray(nu, dtype=np.float64)
    Tb = np.asarray(Tb_scene, dtype=np.float64)
    if Tb.shape != nu.shape:
        raise IRSError(f"Tb_scene must match length(ν)={len(nu)}; got {len(Tb)}")
    n0 = np.broadcast_to(np.asarray(nedt_280K, dtype=np.float64), nu.shape)
    return n0 * _dB_dT(nu, float(T_ref)) / _dB_dT(nu, Tb)


def exclude_channels(nu, *ranges) -> np.ndarray:
    """exclude_channels (optimal_estimation.jl): keep-mask dropping channels inside any (lo, hi)."""
    nu = np.asarray(nu, dtype=np.float64)
    keep = np.ones(len(nu), bool)
    for lo, hi in ranges:
        keep &= ~((nu >= lo) & (nu <= hi))
    return keep


# ------------------------------------------------------------------ optimal estimation
@dataclass
class RetrievalResult:
    """RetrievalResult (optimal_estimation.jl:53-72)."""
    x: np.ndarray
    spec: StateVectorSpec
    converged: bool
    n_iter: int
    cost: float
    S_hat: np.ndarray
    A: np.ndarray
    G: Optional[np.ndarray]
    K: Optional[np.ndarray]
    dof: float
    dfn: float
    H: float
    S_noise: Optional[np.ndarray]
    S_smoothing: np.ndarray
    chi2: float
    y_fit: np.ndarray
    nu: np.ndarray
    channel_mask: np.ndarray


def _se_inverse(Se, n_ch, keep):
    Se = np.asarray(Se, dtype=np.float64)
    if Se.ndim == 2:
        if Se.shape != (n_ch, n_ch):
            raise IRSError(f"Se must be n_y×n_y with n_y = {n_ch}")
        if np.any(Se - np.diag(np.diag(Se))):
            raise IRSError("a dense Se is not supported on this path: pass its diagonal")
        Se = np.diag(Se)
    if Se.shape != (n_ch,):
        raise IRSError(f"Se must have {n_ch} variances")
    if np.any(Se[keep] <= 0):
        raise IRSError("Se variances must be positive")
    w = np.zeros(n_ch)
    w[keep] = 1.0 / Se[keep]
    return w, Se


def optimal_estimation_batch(ys, spec: StateVectorSpec, base_profs, linelists, *, xa, Sa, Se, x0=None,
                             channel_mask=None, method="levenberg_marquardt", max_iter=15, max_linesearch=8,
                             gamma0=1.0, gamma_factor=3.0, gamma_min=1e-4, conv_factor=1e-1, observable="bt",
                             eps_fixed=1.0, fm_kwargs=None, sounder=None, geoms=None, backend=None,
                             line_mixing=None):
    """optimal_estimation (optimal_estimation.jl:142-291) for a batch of scenes on the GPU.

    ys [n_scene, n_ch]; xa [n_scene, n] (or [n]); Sa [n, n] shared; Se: per-channel
    variances [n_scene, n_ch] or [n_ch], or covariance matrices [n_scene, n_ch, n_ch] or
    one [n_ch, n_ch] (a square 2-D Se is always a covariance).  A non-diagonal covariance
    must be banded (half-width <= 32, as the apodised Se of apodized_measurement_covariance):
    the library factors it and retrieves on whitened residuals and Jacobians.  Returns
    dict(x, y_fit, M, n_iter, converged, cost, nu, ...)."""
    from . import (IASIInstrument, _prepare, _ProfileBatch, default_context, fm_options, nadir_geometry,
                   sounder_grid)
    if method not in ("levenberg_marquardt", "gauss_newton"):
        raise IRSError(f"method must be :levenberg_marquardt or :gauss_newton, got :{method}")
    _check_observable(observable)
    if any(b.basis is not None for b in spec.vmr_blocks):
        raise IRSError("reduced VMR blocks are not supported by the batched retrieval")
    ctx = backend or default_context()
    sounder = sounder or IASIInstrument()
    nu = sounder_grid(sounder)
    n_ch, n = len(nu), spec.n
    ys = np.ascontiguousarray(np.atleast_2d(ys), dtype=np.float64)
    S = len(ys)
    if ys.shape[1] != n_ch:
        raise IRSError(f"y has {ys.shape[1]} channels, the sounder {n_ch}")
    xa = np.ascontiguousarray(np.broadcast_to(np.asarray(xa, dtype=np.float64), (S, n)))
    x0 = xa.copy() if x0 is None else np.ascontiguousarray(np.broadcast_to(np.asarray(x0, np.float64), (S, n)))
    Sa = np.asarray(Sa, dtype=np.float64)
    if Sa.shape != (n, n):
        raise IRSError(f"Sa must be {n}×{n}")
    keep = np.ones(n_ch, bool) if channel_mask is None else np.asarray(channel_mask, bool)
    if len(keep) != n_ch:
        raise IRSError(f"channel_mask length {len(keep)} ≠ length(y) {n_ch}")
    if not keep.any():
        raise IRSError("channel_mask excludes every channel")
    Se = np.asarray(Se, dtype=np.float64)
    Se_mats = None
    if Se.ndim == 3 or (Se.ndim == 2 and Se.shape == (n_ch, n_ch)):
        Se_mats = np.broadcast_to(Se, (S, n_ch, n_ch)) if Se.ndim == 2 else Se
        if Se_mats.shape != (S, n_ch, n_ch):
            raise IRSError(f"Se must be n_y×n_y with n_y = {n_ch}, per scene or shared")
        off = Se_mats - np.eye(n_ch)[None] * np.diagonal(Se_mats, axis1=1, axis2=2)[:, :, None]
        if not np.any(off):
            Se, Se_mats = np.diagonal(Se_mats, axis1=1, axis2=2), None
    w = None
    if Se_mats is None:
        Se_rows = np.broadcast_to(Se, (S, n_ch)) if Se.ndim == 1 or (Se.ndim == 2 and Se.shape == (S, n_ch)) else None
        if Se_rows is None:
            raise IRSError("Se must be [n_ch] or [n_scene, n_ch] variances, or n_ch×n_ch covariances")
        w = np.ascontiguousarray(np.stack([_se_inverse(Se_rows[k], n_ch, keep)[0] for k in range(S)]))
    else:
        ii, jj = np.nonzero(np.any(Se_mats != 0.0, axis=0))
        bw = int(np.max(np.abs(ii - jj))) if len(ii) else 0
        if bw > 32:
            raise IRSError(f"a covariance Se of band half-width {bw} is not supported on the GPU path (at most 32)")
        band = np.zeros((S, n_ch, bw + 1))
        for k in range(bw + 1):
            band[:, k:, k] = np.diagonal(Se_mats, offset=-k, axis1=1, axis2=2)
        band = np.ascontiguousarray(band)
    Sa_inv = np.ascontiguousarray(np.linalg.inv(Sa))
    base_profs = list(base_profs) if isinstance(base_profs, (list, tuple)) else [base_profs] * S
    geoms = geoms or [nadir_geometry()] * S
    kw = dict(fm_kwargs or {})
    kw.pop("dptmn", None)
    prec = kw.pop("precision", "mixed")
    _prepare(ctx, linelists, line_mixing)
    o = fm_options(line_mixing=line_mixing, dptmn=0.0, precision=prec, **kw)
    batch = _ProfileBatch(base_profs, [None] * S, [g.mu for g in geoms], [eps_fixed] * S)
    cs, keep_ref = _c_spec(spec, spec.log_vmr, True, observable)
    prm = _lib.OEParams()
    prm.max_iter, prm.max_linesearch = int(max_iter), int(max_linesearch)
    prm.method = 0 if method == "levenberg_marquardt" else 1
    prm.gamma0, prm.gamma_factor, prm.gamma_min = float(gamma0), float(gamma_factor), float(gamma_min)
    prm.conv_factor, prm.eps_fixed = float(conv_factor), float(eps_fixed)
    s = sounder.c_struct()
    x = np.empty((S, n))
    y_fit = np.empty((S, n_ch))
    M = np.empty((S, n, n))
    n_iter = np.empty(S, np.int32)
    conv = np.empty(S, np.int32)
    cost = np.empty(S)
    I32 = C.POINTER(C.c_int32)
    if w is not None:
        check(ctx.lib.irs_oe_batch(ctx.h, batch.arr, S, C.byref(s), C.byref(o), C.byref(cs), dptr(ys), dptr(w),
                                   dptr(xa), dptr(Sa_inv), dptr(x0), C.byref(prm), dptr(x), dptr(y_fit), dptr(M),
                                   n_iter.ctypes.data_as(I32), conv.ctypes.data_as(I32), dptr(cost)))
    else:
        kp = np.ascontiguousarray(keep.astype(np.uint8))
        check(ctx.lib.irs_oe_batch_banded(ctx.h, batch.arr, S, C.byref(s), C.byref(o), C.byref(cs), dptr(ys),
                                          dptr(band), band.shape[2] - 1, kp.ctypes.data_as(C.POINTER(C.c_uint8)),
                                          dptr(xa), dptr(Sa_inv), dptr(x0), C.byref(prm), dptr(x), dptr(y_fit),
                                          dptr(M), n_iter.ctypes.data_as(I32), conv.ctypes.data_as(I32),
                                          dptr(cost)))
    return dict(x=x, y_fit=y_fit, M=M, n_iter=n_iter, converged=conv.astype(bool), cost=cost, nu=nu, w=w,
                Se=Se_mats, Sa_inv=Sa_inv, keep=keep)


def _banded_solver(Se_k):
    """x -> Se_k^-1 x through the banded Cholesky factor of Se_k (scipy.linalg)."""
    from scipy.linalg import cho_solve_banded, cholesky_banded
    n = len(Se_k)
    ii, jj = np.nonzero(Se_k)
    bw = int(np.max(np.abs(ii - jj))) if len(ii) else 0
    ab = np.zeros((bw + 1, n))
    for k in range(bw + 1):
        ab[bw - k, k:] = np.diagonal(Se_k, offset=k)
    c = cholesky_banded(ab)
    return lambda x: cho_solve_banded((c, False), x)


def oe_diagnostics(M, Sa, Sa_inv=None):
    """Rodgers diagnostics from M = K^T Se^-1 K (optimal_estimation.jl:257-282):
    (S_hat, A, dof, H, S_smoothing)."""
    Sa_inv = np.linalg.inv(Sa) if Sa_inv is None else Sa_inv
    S_hat = np.linalg.inv(Sa_inv + M)
    A = S_hat @ M
    dof = float(np.trace(A))
    n = len(A)
    _, ld = np.linalg.slogdet(np.eye(n) - A)
    H = -0.5 * ld / np.log(2.0)
    ImA = np.eye(n) - A
    return S_hat, A, dof, float(H), ImA @ Sa @ ImA.T


def optimal_estimation(y, spec: StateVectorSpec, base_prof, linelists, *, xa, Sa, Se, channel_mask=None, x0=None,
                       method="levenberg_marquardt", max_iter=15, max_linesearch=8, gamma0=1.0, gamma_factor=3.0,
                       gamma_min=1e-4, conv_factor=1e-1, observable="bt", eps_fixed=1.0, fm_kwargs=None,
                       sounder=None, geom=None, backend=None, line_mixing=None, verbose=False) -> RetrievalResult:
    """optimal_estimation (optimal_estimation.jl:142-291) -> RetrievalResult, one scene."""
    from . import nadir_geometry
    r = optimal_estimation_batch(np.atleast_2d(y), spec, [base_prof], linelists, xa=np.asarray(xa)[None],
                                 Sa=Sa, Se=Se, x0=None if x0 is None else
                                 np.asarray(x0)[None], channel_mask=channel_mask, method=method, max_iter=max_iter,
                                 max_linesearch=max_linesearch, gamma0=gamma0, gamma_factor=gamma_factor,
                                 gamma_min=gamma_min, conv_factor=conv_factor, observable=observable,
                                 eps_fixed=eps_fixed, fm_kwargs=fm_kwargs, sounder=sounder,
                                 geoms=[geom or nadir_geometry()], backend=backend, line_mixing=line_mixing)
    x = r["x"][0]
    M = r["M"][0]
    keep = r["keep"]
    S_hat, A, dof, H, S_smooth = oe_diagnostics(M, np.asarray(Sa, np.float64), r["Sa_inv"])
    # K at the solution (full channel grid) for the gain matrix and the noise budget
    prof, Ts, es = unpack_state(spec, x, base_prof)
    kw = dict(fm_kwargs or {})
    kw.pop("dptmn", None)
    kw.pop("precision", None)
    jac = analytic_jacobian(prof, linelists, spec, sounder=sounder, geom=geom, T_sfc=Ts,
                            eps_sfc=es if spec.include_emissivity else eps_fixed, observable=observable,
                            backend=backend, line_mixing=line_mixing, **kw)
    Kk = jac.K[keep]
    resid = (np.atleast_2d(y)[0] - r["y_fit"][0])[keep]
    if r["w"] is not None:
        wk = r["w"][0][keep]
        G = S_hat @ (Kk * wk[:, None]).T
        S_noise = (G * (1.0 / wk)[None, :]) @ G.T
        chi2 = float(np.sum(resid * wk * resid))
    else:  # banded covariance: Se^-1 by its banded Cholesky factor on the kept channels
        Se_k = r["Se"][0][np.ix_(keep, keep)]
        solve = _banded_solver(Se_k)
        G = S_hat @ solve(Kk).T
        S_noise = G @ Se_k @ G.T
        chi2 = float(resid @ solve(resid))
    m = int(keep.sum())
    return RetrievalResult(x=x, spec=spec, converged=bool(r["converged"][0]), n_iter=int(r["n_iter"][0]),
                           cost=float(r["cost"][0]), S_hat=S_hat, A=A, G=G, K=jac.K, dof=dof, dfn=m - dof, H=H,
                           S_noise=S_noise, S_smoothing=S_smooth, chi2=chi2, y_fit=r["y_fit"][0], nu=r["nu"],
                           channel_mask=keep)
