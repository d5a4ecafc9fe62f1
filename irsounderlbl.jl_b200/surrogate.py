"""MLP surrogate of forward_model: profile + scan angle -> channel brightness temperatures.

No counterpart in the reference.  The network (n_in -> n_layers x n_hidden GELU ->
n_out) runs on the tcgen05 tensor cores through ``libirs_b200.so`` (BF16 weights and
activations, FP32 accumulation, FP32 master weights and Adam); it is trained only on
spectra of the GPU line-by-line path, which is also its fallback for inputs whose
out-of-distribution score exceeds the threshold and the judge of its error on a
held-out share of every batch.

Input features (152 for 50 levels): T [n_lev], log VMR H2O [n_lev], log VMR O3
[n_lev], T_sfc, scan angle (degrees).
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence

import numpy as np

from . import _lib
from ._lib import IRSError, check, dptr, fptr

VMR_FLOOR = 1e-30


def surrogate_features(profiles, scan_angles, T_sfcs=None) -> np.ndarray:
    """[n, 3 n_lev + 2] float32 features of the profiles (T, log H2O, log O3, T_sfc, angle)."""
    n = len(profiles)
    T_sfcs = T_sfcs if T_sfcs is not None else [None] * n
    rows = []
    for p, a, ts in zip(profiles, scan_angles, T_sfcs):
        T = np.asarray(p.temperature, dtype=np.float64)
        h = np.log(np.maximum(np.asarray(p.vmr[1], dtype=np.float64), VMR_FLOOR))
        o = np.log(np.maximum(np.asarray(p.vmr[3], dtype=np.float64), VMR_FLOOR))
        rows.append(np.concatenate([T, h, o, [T[0] if ts is None else ts, float(a)]]))
    return np.ascontiguousarray(np.array(rows, dtype=np.float32))


class Surrogate:
    """One MLP on one GPU context (irs_surrogate_* of the C ABI)."""

    def __init__(self, ctx=None, n_in: int = 152, n_hidden: int = 1024, n_layers: int = 4, n_out: int = 8461,
                 seed: int = 1003):
        from . import default_context
        self.ctx = ctx or default_context()
        self.lib = self.ctx.lib
        self.n_in, self.n_hidden, self.n_layers, self.n_out = n_in, n_hidden, n_layers, n_out
        h = C.c_void_p()
        check(self.lib.irs_surrogate_create(self.ctx.h, n_in, n_hidden, n_layers, n_out, seed, C.byref(h)))
        self.h = h
        self.ood_threshold = np.inf
        self.x_mean = np.zeros(n_in, np.float32)
        self.x_sd = np.ones(n_in, np.float32)
        self.y_mean = np.zeros(n_out, np.float32)
        self.y_sd = np.ones(n_out, np.float32)

    # -------------------------------------------------------------- parameters
    def param_count(self) -> int:
        n = C.c_int64()
        check(self.lib.irs_surrogate_param_count(self.h, C.byref(n)))
        return n.value

    def get_params(self) -> np.ndarray:
        p = np.empty(self.param_count(), np.float32)
        check(self.lib.irs_surrogate_get_params(self.h, fptr(p)))
        return p

    def set_params(self, p: np.ndarray):
        p = np.ascontiguousarray(p, dtype=np.float32)
        if p.shape != (self.param_count(),):
            raise IRSError(f"parameter vector has shape {p.shape}, expected ({self.param_count()},)")
        check(self.lib.irs_surrogate_set_params(self.h, fptr(p)))

    def layer_shapes(self):
        dims = [self.n_in] + [self.n_hidden] * self.n_layers + [self.n_out]
        return [(dims[l + 1], dims[l]) for l in range(len(dims) - 1)]

    def unflatten(self, p: np.ndarray):
        """[(W, b)] per layer from the flat parameter vector."""
        out, k = [], 0
        for o, i in self.layer_shapes():
            W = p[k:k + o * i].reshape(o, i)
            k += o * i
            b = p[k:k + o]
            k += o
            out.append((W, b))
        return out

    # -------------------------------------------------------------- scaling / OOD
    def fit_scaling(self, X: np.ndarray, Y: np.ndarray, ood_quantile: float = 0.999, ood_margin: float = 2.0):
        """Input/output standardisation, the whitening matrix of the scaled inputs and
        the OOD threshold (ood_margin x the ood_quantile of the training scores)."""
        X = np.asarray(X, dtype=np.float64)
        Y = np.asarray(Y, dtype=np.float64)
        self.x_mean = X.mean(0).astype(np.float32)
        self.x_sd = np.maximum(X.std(0), 1e-6 * np.maximum(np.abs(X).max(0), 1.0)).astype(np.float32)
        self.y_mean = Y.mean(0).astype(np.float32)
        self.y_sd = np.maximum(Y.std(0), 1e-3).astype(np.float32)
        check(self.lib.irs_surrogate_set_scaling(self.h, fptr(self.x_mean), fptr(self.x_sd), fptr(self.y_mean),
                                                 fptr(self.y_sd)))
        Z = (X - self.x_mean) / self.x_sd
        cov = np.cov(Z, rowvar=False) + 1e-9 * np.eye(self.n_in)
        w, V = np.linalg.eigh(cov)
        w = np.maximum(w, 1e-4 * w.max())
        W = np.ascontiguousarray((V / np.sqrt(w)) @ V.T, dtype=np.float32)
        check(self.lib.irs_surrogate_set_whitening(self.h, fptr(W)))
        _, s = self.predict(X.astype(np.float32))
        self.ood_threshold = float(ood_margin * np.quantile(s, ood_quantile))
        return self.ood_threshold

    # -------------------------------------------------------------- training
    def train(self, X: np.ndarray, Y: np.ndarray, epochs: int = 10, batch: int = 256, lr: float = 1e-3,
              seed: int = 1003) -> np.ndarray:
        X = np.ascontiguousarray(X, dtype=np.float32)
        Y = np.ascontiguousarray(Y, dtype=np.float32)
        self._check(X, Y)
        losses = np.zeros(epochs)
        check(self.lib.irs_surrogate_train(self.h, fptr(X), fptr(Y), len(X), batch, epochs, lr, seed, dptr(losses)))
        return losses

    def gradients(self, X: np.ndarray, Y: np.ndarray):
        X = np.ascontiguousarray(X, dtype=np.float32)
        Y = np.ascontiguousarray(Y, dtype=np.float32)
        self._check(X, Y)
        g = np.empty(self.param_count(), np.float32)
        loss = C.c_double()
        check(self.lib.irs_surrogate_gradients(self.h, fptr(X), fptr(Y), len(X), fptr(g), C.byref(loss)))
        return g, loss.value

    def _check(self, X, Y=None):
        if X.ndim != 2 or X.shape[1] != self.n_in:
            raise IRSError(f"inputs have shape {X.shape}, expected (n, {self.n_in})")
        if Y is not None and (Y.shape != (len(X), self.n_out)):
            raise IRSError(f"targets have shape {Y.shape}, expected ({len(X)}, {self.n_out})")

    # -------------------------------------------------------------- inference
    def predict(self, X: np.ndarray, out: np.ndarray | None = None, ood: np.ndarray | None = None):
        """(BT [n, n_out] float32, OOD score [n]).  `out` and `ood`, when given, are
        filled in place and returned: a serving loop that reuses them (page-locked, for
        example numpy views of pinned torch tensors) skips the allocation, first-touch
        page faults and pageable staging of a fresh 4 x n x n_out-byte result per call."""
        X = np.ascontiguousarray(X, dtype=np.float32)
        self._check(X)
        if out is None:
            out = np.empty((len(X), self.n_out), np.float32)
        if ood is None:
            ood = np.empty(len(X), np.float32)
        for a, shape in ((out, (len(X), self.n_out)), (ood, (len(X),))):
            if a.shape != shape or a.dtype != np.float32 or not a.flags.c_contiguous or not a.flags.writeable:
                raise ValueError(f"predict: output must be a writeable C-contiguous float32 array of shape {shape}")
        check(self.lib.irs_surrogate_infer(self.h, fptr(X), len(X), fptr(out), fptr(ood)))
        return out, ood

    def predict_device(self, X, out, ood, stream=None):
        """Inference between device tensors (torch, float32, C-contiguous, on this
        surrogate's device): X [n, n_in] -> out [n, n_out], ood [n], ordered on `stream`
        (a torch.cuda.Stream; the current one when None)."""
        import torch
        n = X.shape[0]
        for t, shape in ((X, (n, self.n_in)), (out, (n, self.n_out)), (ood, (n,))):
            if (tuple(t.shape) != shape or t.dtype != torch.float32 or not t.is_cuda or not t.is_contiguous()
                    or t.device.index != self.ctx.device):
                raise ValueError(f"predict_device: need a contiguous float32 tensor of shape {shape} on cuda:"
                                 f"{self.ctx.device}")
        st = stream if stream is not None else torch.cuda.current_stream(X.device)
        check(self.lib.irs_surrogate_infer_device(self.h, C.c_void_p(X.data_ptr()), n, C.c_void_p(out.data_ptr()),
                                                  C.c_void_p(ood.data_ptr()), C.c_void_p(st.cuda_stream)))
        return out, ood

    def close(self):
        if getattr(self, "h", None):
            self.lib.irs_surrogate_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------------ data parallel
def cosine_lr(lr: float, epoch: int, epochs: int) -> float:
    """The learning-rate schedule of irs_surrogate_train: cosine from lr down to lr/100."""
    if epochs <= 1:
        return float(lr)
    lo = 0.01 * lr
    return float(lo + 0.5 * (lr - lo) * (1.0 + np.cos(np.pi * epoch / (epochs - 1))))


def dp_rows(n_local: int, batch: int, epoch: int, step: int, seed: int, rank: int) -> np.ndarray:
    """Local rows of mini-batch `step` of `epoch` on `rank`: a permutation of the rank's
    own samples seeded by (seed, epoch, rank), cut into full batches.  The global
    mini-batch is the concatenation of every rank's rows."""
    perm = np.random.Generator(np.random.PCG64([int(seed), int(epoch), int(rank)])).permutation(n_local)
    return np.ascontiguousarray(perm[step * batch:(step + 1) * batch], dtype=np.int32)


def train_data_parallel(grad_fn, apply_fn, n_local: int, *, batch: int, epochs: int, lr: float, seed: int,
                        rank: int, world: int, all_reduce, steps_per_epoch: int = None):
    """Data-parallel Adam over `world` ranks, one model replica per rank.

    Each step every rank takes `batch` rows of its own samples (dp_rows), grad_fn(rows)
    returns the gradient of 0.5 mean((y' - t')^2) over them (a tensor, any device) and
    the local loss, the gradients are averaged over the ranks by all_reduce (an in-place
    sum: NCCL on GPUs, gloo in tests; equal local batches make the average the gradient
    of the concatenated global batch) and apply_fn(gradient, lr) takes one Adam step on
    the replica.  Every rank takes the same number of steps (collectives stay matched):
    steps_per_epoch, or n_local // batch, which must then agree on every rank.

    Returns the loss per epoch (the mean over steps of the global-batch loss)."""
    import torch
    n_steps = steps_per_epoch if steps_per_epoch is not None else n_local // batch
    if n_steps < 1 or n_steps * batch > n_local:
        raise IRSError(f"{n_local} local samples do not fill {n_steps} batches of {batch}")
    losses = np.zeros(epochs)
    for ep in range(epochs):
        lr_ep = cosine_lr(lr, ep, epochs)
        tot = 0.0
        for st in range(n_steps):
            g, loss = grad_fn(dp_rows(n_local, batch, ep, st, seed, rank))
            g.mul_(1.0 / world)
            all_reduce(g)
            apply_fn(g, lr_ep)
            tot += float(loss)
        t = torch.tensor([tot / n_steps / world], dtype=torch.float64)
        all_reduce(t)
        losses[ep] = float(t.item())
    return losses


class DataParallelSurrogate:
    """One Surrogate replica per rank of a torch.distributed process group (NCCL, one
    GPU per rank): its training data stays resident on the rank's device and each step
    all-reduces the flat gradient in place before the Adam update, through
    irs_surrogate_grad_device / irs_surrogate_apply_device on the current torch stream.
    Peer memory is reached only by NCCL."""

    def __init__(self, sur: Surrogate, dist=None):
        import torch
        self.sur, self.dist = sur, dist
        self.torch = torch
        n = C.c_int64()
        check(sur.lib.irs_surrogate_grad_size(sur.h, C.byref(n)))
        self.grad = torch.zeros(n.value, dtype=torch.float32, device="cuda")
        self.world = dist.get_world_size() if dist is not None else 1
        self.rank = dist.get_rank() if dist is not None else 0

    def _all_reduce(self, t):
        if self.dist is None:
            return
        if t.device.type == "cpu":  # the loss scalar
            g = t.to("cuda")
            self.dist.all_reduce(g)
            t.copy_(g.cpu())
        else:
            self.dist.all_reduce(t)

    def train(self, X_local: np.ndarray, Y_local: np.ndarray, *, epochs: int, batch: int, lr: float = 1e-3,
              seed: int = 1003, steps_per_epoch: int = None) -> np.ndarray:
        torch = self.torch
        sur = self.sur
        X = torch.from_numpy(np.ascontiguousarray(X_local, dtype=np.float32)).to("cuda")
        Y = torch.from_numpy(np.ascontiguousarray(Y_local, dtype=np.float32)).to("cuda")
        sur._check(X_local, Y_local)
        idx = torch.empty(batch, dtype=torch.int32, device="cuda")
        loss = C.c_double()

        def grad_fn(rows):
            idx.copy_(torch.from_numpy(rows))
            st = torch.cuda.current_stream().cuda_stream
            check(sur.lib.irs_surrogate_grad_device(sur.h, C.c_void_p(X.data_ptr()), C.c_void_p(Y.data_ptr()),
                                                    C.cast(C.c_void_p(idx.data_ptr()), C.POINTER(C.c_int32)),
                                                    len(rows), C.cast(C.c_void_p(self.grad.data_ptr()),
                                                                      C.POINTER(C.c_float)),
                                                    C.byref(loss), C.c_void_p(st)))
            return self.grad, loss.value

        def apply_fn(g, lr_ep):
            st = torch.cuda.current_stream().cuda_stream
            check(sur.lib.irs_surrogate_apply_device(sur.h, C.cast(C.c_void_p(g.data_ptr()), C.POINTER(C.c_float)),
                                                     C.c_float(lr_ep), C.c_void_p(st)))

        return train_data_parallel(grad_fn, apply_fn, len(X_local), batch=batch, epochs=epochs, lr=lr, seed=seed,
                                   rank=self.rank, world=self.world, all_reduce=self._all_reduce,
                                   steps_per_epoch=steps_per_epoch)


def surrogate_forward_batch(sur: Surrogate, profiles: Sequence, scan_angles, linelists, *, sounder=None,
                            T_sfcs=None, holdout: float = 0.01, seed: int = 0, backend=None, **lbl_kw):
    """Brightness temperatures of a batch from the surrogate, with the line-by-line path
    as fallback for OOD inputs and as judge on a held-out share.

    Returns dict(BT [n, n_ch], lbl_mask [n] (rows computed by LBL), ood [n],
    holdout_index, holdout_rms, holdout_max)."""
    from . import ViewingGeometry, forward_model_batch, scan_angle_to_local_zenith
    X = surrogate_features(profiles, scan_angles, T_sfcs)
    BT, ood = sur.predict(X)
    BT = BT.astype(np.float64)
    n = len(profiles)
    fall = ood > sur.ood_threshold
    rng = np.random.Generator(np.random.PCG64(seed))
    n_hold = int(np.ceil(holdout * n)) if holdout > 0 else 0
    cand = np.flatnonzero(~fall)
    hold = rng.choice(cand, size=min(n_hold, len(cand)), replace=False) if n_hold else np.zeros(0, int)
    need = np.union1d(np.flatnonzero(fall), hold).astype(int)
    res = dict(ood=ood, lbl_mask=fall, holdout_index=hold, holdout_rms=None, holdout_max=None)
    if len(need):
        geoms = [ViewingGeometry(scan_angle_to_local_zenith(float(scan_angles[i]))) for i in need]
        T_need = [None if T_sfcs is None else T_sfcs[i] for i in need]
        _, _, BT_lbl = forward_model_batch([profiles[i] for i in need], linelists, sounder=sounder, geoms=geoms,
                                           T_sfcs=T_need, backend=backend, **lbl_kw)
        pos = {int(i): k for k, i in enumerate(need)}
        if len(hold):
            d = np.stack([BT[i] - BT_lbl[pos[int(i)]] for i in hold])
            res["holdout_rms"] = float(np.sqrt(np.mean(d ** 2)))
            res["holdout_max"] = float(np.max(np.abs(d)))
        for i in np.flatnonzero(fall):
            BT[i] = BT_lbl[pos[int(i)]]
    res["BT"] = BT
    return res


def _state_feature_columns(spec, n_in: int):
    """The surrogate input column of every state element when the state is the
    full-profile [T][log VMR H2O][log VMR O3][T_sfc][eps] layout the features share
    (-1: no feature, as eps), else None."""
    n_lev = spec.n_levels
    if n_in != 3 * n_lev + 2:
        return None
    cols = np.full(spec.n, -1, dtype=np.int64)
    if spec.include_temperature:
        cols[spec.temp_range.start:spec.temp_range.stop] = np.arange(n_lev)
    for b in spec.vmr_blocks:
        if b.basis is not None or not spec.log_vmr or int(b.species) not in (1, 3):
            return None
        off = n_lev if int(b.species) == 1 else 2 * n_lev
        cols[b.range.start:b.range.stop] = off + np.arange(n_lev)
    if spec.tsfc_index >= 0:
        cols[spec.tsfc_index] = 3 * n_lev
    return cols


def _first_guess_columns(sur, ys, spec, base_list, scan_angles, xa, Sa, Se, n_iter, step, cols):
    """surrogate_first_guess when the state maps onto feature columns: the perturbed
    inputs are the scene's features moved in one column, all scenes' 2 n + 1 samples go
    to the network in one device-to-device call, and K, K^T W K and the Gauss-Newton
    systems of all scenes are formed and solved as batched FP64 tensors on the
    surrogate's device (only the state -> feature rows are built on the host)."""
    import torch
    from .estimation import unpack_state
    dev = torch.device("cuda", sur.ctx.device)
    f64 = dict(dtype=torch.float64, device=dev)
    S, n = ys.shape[0], spec.n
    has = cols >= 0
    j = np.flatnonzero(has)
    jt, cj = torch.as_tensor(j, device=dev), torch.as_tensor(cols[j], device=dev)
    w = torch.as_tensor(np.ascontiguousarray(1.0 / np.asarray(Se, dtype=np.float64)), **f64)  # [S, n_ch]
    Sa_inv = torch.as_tensor(np.linalg.inv(Sa), **f64)
    ys_t = torch.as_tensor(np.ascontiguousarray(ys, dtype=np.float64), **f64)
    xa_t = torch.as_tensor(np.ascontiguousarray(xa, dtype=np.float64), **f64)
    x = np.array(xa, dtype=np.float64)
    # one set of buffers for every iteration's batched inference (S (2 n + 1) rows); a
    # perturbed input is the float64 sum rounded once to float32
    Xp = torch.empty((S, 2 * n + 1, sur.n_in), dtype=torch.float32, device=dev)
    out = torch.empty((S * (2 * n + 1), sur.n_out), dtype=torch.float32, device=dev)
    ood = torch.empty(S * (2 * n + 1), dtype=torch.float32, device=dev)
    for _ in range(n_iter):
        rows = [unpack_state(spec, x[s_], base_list[s_]) for s_ in range(S)]
        F0 = torch.as_tensor(surrogate_features([r[0] for r in rows], scan_angles, [r[1] for r in rows]),
                             device=dev)  # float32 [S, n_in]
        Xp.copy_(F0[:, None, :].expand(-1, 2 * n + 1, -1))
        c64 = F0[:, cj].double()
        Xp[:, 1 + 2 * jt, cj] = (c64 + step).float()
        Xp[:, 2 + 2 * jt, cj] = (c64 - step).float()
        sur.predict_device(Xp.view(-1, sur.n_in), out, ood)
        F = out.view(S, 2 * n + 1, -1).double()
        KT = (F[:, 1::2] - F[:, 2::2]) / (2 * step)  # K^T: [S, n, n_ch]
        KT[:, torch.as_tensor(~has, device=dev)] = 0.0
        KtW = KT * w[:, None, :]
        H = Sa_inv + KtW @ KT.transpose(1, 2)
        dx = torch.as_tensor(x, **f64) - xa_t
        r = ys_t - F[:, 0] + torch.einsum("sjc,sj->sc", KT, dx)
        g = torch.einsum("sjc,sc->sj", KtW, r)
        x = (xa_t + torch.linalg.solve(H, g[..., None])[..., 0]).cpu().numpy()
    return x


def surrogate_first_guess(sur: Surrogate, ys, spec, base_profs, scan_angles, *, xa, Sa, Se, n_iter: int = 4,
                          step: float = 1e-2):
    """First guesses of a batched retrieval from the surrogate: Gauss-Newton MAP steps
    (Rodgers 2000, eq. 5.9) with F and K both from the network (K by central
    differences of batched inferences, 2 n_state + 1 samples per scene).  The state is
    the full-profile [T][log VMR H2O / O3][T_sfc] layout of StateVectorSpec.

    Returns x0 [n_scene, n_state]."""
    from .estimation import unpack_state
    ys = np.atleast_2d(np.asarray(ys, dtype=np.float64))
    S, n = len(ys), spec.n
    xa = np.broadcast_to(np.asarray(xa, dtype=np.float64), (S, n))
    Se = np.broadcast_to(np.asarray(Se, dtype=np.float64), ys.shape)
    base_list = list(base_profs) if isinstance(base_profs, (list, tuple)) else [base_profs] * S
    cols = _state_feature_columns(spec, sur.n_in)
    if cols is not None:
        return _first_guess_columns(sur, ys, spec, base_list, scan_angles, xa, Sa, Se, n_iter, step, cols)
    w = 1.0 / Se
    Sa_inv = np.linalg.inv(Sa)
    base_profs = list(base_profs) if isinstance(base_profs, (list, tuple)) else [base_profs] * S
    x = xa.copy()

    def feats(xs, idx):
        rows = []
        for x_, i in zip(xs, idx):
            p, Ts, _ = unpack_state(spec, x_, base_profs[i])
            rows.append((p, Ts, scan_angles[i]))
        return surrogate_features([r[0] for r in rows], [r[2] for r in rows], [r[1] for r in rows])

    for _ in range(n_iter):
        pert, idx = [], []
        for s_ in range(S):
            pert.append(x[s_])
            idx.append(s_)
            for j in range(n):
                for sg in (1.0, -1.0):
                    xp = x[s_].copy()
                    xp[j] += sg * step
                    pert.append(xp)
                    idx.append(s_)
        F, _ = sur.predict(feats(pert, idx))
        F = F.astype(np.float64).reshape(S, 2 * n + 1, -1)
        for s_ in range(S):
            F0 = F[s_, 0]
            K = ((F[s_, 1::2] - F[s_, 2::2]) / (2 * step)).T  # [n_ch, n]
            KtW = K.T * w[s_]
            H = Sa_inv + KtW @ K
            g = KtW @ (ys[s_] - F0 + K @ (x[s_] - xa[s_]))
            x[s_] = xa[s_] + np.linalg.solve(H, g)
    return x
