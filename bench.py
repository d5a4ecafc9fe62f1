#!/usr/bin/env python
"""IASI spectra/s on B200: the line-by-line forward model on 400,000 synthetic lines.

Workload ("iasi-400k"): 400,000 lines over H2O, CO2, O3, N2O, CO, CH4 in
645-2760 cm^-1, IASI sounder (8461 channels, Gaussian apodization), 0.0025 cm^-1
internal grid (858,801 points), the six AFGL 50-level profiles (49 layers),
FullFaddeeva, 25 cm^-1 cutoff, DPTMIN 1e-6, :cim source,
MT-CKD H2O and CO2 continua (CIA tables are not bundled and contribute zero, as
in the reference without them).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One process per GPU (torchrun for N > 1).  A step is one global batch of 24 profiles
(the six AFGL profiles x 4) split into contiguous shards over the ranks (strong
scaling; no data-path collective); a weak-scaling line (the six profiles on every
rank) is reported beside it.  `value` is the mixed (FP32 + Kahan) path with line
lists resident in HBM, device-timed with CUDA events (max over ranks); `e2e` goes
through the host C-ABI call with host buffers; the plain FP64 kernel's spectra/s is
reported beside it.  `--impl reference` times the reference algorithm's CPU
implementation (the FP64 C++ restatement under oracle/, all host threads) on a
bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
N_PROF = 6
GLOBAL_BATCH = 4 * N_PROF  # profiles per step over all GPUs: the six AFGL profiles x 4
FAR_PAIR_FLOPS = 10     # d (2), d^2, d^2+b^2, rcp, pedestal FMA (2), value FMA (2), accumulate
CORE_PAIR_FLOPS = 70    # far-pair ops + FP32 Faddeeva (continued fraction / Weideman-16 branch)
FP32_LANES = 148 * 128  # B200: 148 SMs x 128 FP32 lanes


def _package():
    sys.path.insert(0, str(ROOT))
    import __graft_entry__ as ge
    return ge._package()


# metric, unit and workload description shared by both arms (the driver compares the
# two lines only when they agree)
METRIC = "IASI spectra/s (line-by-line forward_model, 400k lines)"


def workload_config():
    return {"workload": "iasi-400k", "lines": 400000, "species": 6, "grid_dnu": 0.0025, "n_nu": 858801,
            "layers": 49, "channels": 8461, "profiles": "the 6 AFGL 50-level profiles",
            "batch": "24 profiles per step (the 6 AFGL profiles x 4), split over the GPUs", "method": "FullFaddeeva",
            "cutoff": 25.0, "dptmn": 1e-6, "continua": "h2o,co2",
            "l2": "working set (line parameters ~4 GB, tau 1 GB) >> L2"}


def _workload_kw():
    return dict(internal_dnu=0.0025, cutoff=25.0, dptmn=1e-6, apply_continuum=True,
                with_ils=True, apodization="gaussian", T_method="logp_at_pcg",
                source_function="cim")


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during a region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                       "-lms", "200", "-i", str(self.idx)],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.p is not None:
            self.p.terminate()
            try:
                self.out, _ = self.p.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()
                self.out = ""
        else:
            self.out = ""

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in (self.out or "").splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def _physical_gpu(local_rank: int) -> int:
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        try:
            return int(vis.split(",")[local_rank])
        except (ValueError, IndexError):
            pass
    return local_rank


def _traffic_from_profiles():
    """DRAM bytes per launch of the line-sum kernel from the committed ncu summary."""
    p = ROOT / "profiles" / "linesum_mixed_iasi400k.txt"
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        if line.startswith("traffic_bytes_per_launch_full:"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


def cpu_sample(seconds_target: float = 8.0):
    """Oracle (reference algorithm, FP64, all host threads) on a channel window of the
    same workload; scaled to full spectra by internal grid points."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as orc
    pkg = _package()
    o = orc.Oracle()
    lists = pkg.synthetic.lists_iasi_400k()
    prof = pkg.afgl_atmosphere("us_standard")
    snd = orc.sounder(645.0, 2760.0, 0.25, opd_max=2.0, fwhm_gauss=0.5)
    opt = orc.fm_options(**_workload_kw())
    n_full = 858801
    ll = {s: l.lines for s, l in lists.items()}
    pr = dict(p=prof.pressure, T=prof.temperature, vmr=prof.vmr)
    # size the window: time a small one first, then grow to about `seconds_target`
    c0 = 3000
    t0 = time.perf_counter()
    o.forward_model(pr, ll, snd, opt, channels=(c0, c0 + 8))
    t_small = time.perf_counter() - t0
    n_small = 8 * 100 + 12800 + 1
    per_pt = t_small / n_small
    n_ch = max(8, int((seconds_target / per_pt - 12801) / 100))
    n_ch = min(n_ch, 8461 - c0)
    n_pts = n_ch * 100 + 12800 + 1

    def run():
        t = time.perf_counter()
        o.forward_model(pr, ll, snd, opt, channels=(c0, c0 + n_ch))
        return time.perf_counter() - t

    return run, n_pts, n_full, orc.num_threads(), c0, n_ch


def reference_arm(args, rank):
    if rank != 0:
        return
    run, n_pts, n_full, cores, c0, n_ch = cpu_sample()
    for _ in range(args.warmup):
        run()
    ts = [run() for _ in range(args.steps)]
    t = sum(ts) / len(ts)
    v = n_pts / n_full / t
    line = {
        "impl": "reference", "metric": METRIC,
        "value": v, "unit": "spectra/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded line lists, AFGL profiles)",
        "config": workload_config(),
        "cpu_baseline": {"value": v, "unit": "spectra/s", "cores": cores, "kind": "port",
                         "sample": f"one AFGL profile, channels {c0}..{c0 + n_ch - 1} ({n_pts} internal grid "
                                   f"points of {n_full}), scaled by grid points"},
        "e2e": {"value": v, "unit": "spectra/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def reduce_max(dist, x: float, device: str) -> float:
    """Max of a per-rank scalar over the process group (the timing rule for N > 1);
    `dist` None means one process."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def weak_scaling_value(world: int, profiles_per_rank: int, ms_per_step: float) -> float:
    """Whole-job spectra/s: every rank runs its own profiles (no data-path collective),
    the step time is the max over ranks."""
    return world * profiles_per_rank / (ms_per_step / 1e3)


def _peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return json.loads(p.read_text()), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


def oe_config4(pkg, ctx, n_sc: int = 1024, n_train: int = 16384):
    """Config 4: batched optimal estimation of n_sc scenes of the perturbed-AFGL sampler
    on the 5,000-line CO2 list (221 channels, MT-CKD continua), state T + log H2O + T_sfc
    (101), NEdT 0.2 K at 280 K, Sa from build_sa (0.5 K, 30 %, 3-level correlation).
    First guesses from the MLP surrogate (trained here on n_train GPU-LBL spectra of the
    same sampler, another seed), then Levenberg-Marquardt on the mixed LBL path with the
    analytic Jacobian and FP64 Cholesky; the same retrieval from the a priori beside it."""
    l5 = pkg.synthetic.lists_5k_co2()
    s5 = pkg.Sounder.make(645.0, 700.0, 0.25, opd_max=2.0, fwhm_gauss=0.5)
    kw5 = dict(internal_dnu=0.0025, apply_continuum=True, continua=("h2o", "co2"))
    base = pkg.afgl_atmosphere("us_standard")
    spec5 = pkg.StateVectorSpec(50, [pkg.H2O], include_emissivity=False)
    xa = pkg.pack_state(spec5, base)
    L3 = 3.0 * float(np.median(np.abs(np.diff(np.log(base.pressure)))))  # 3-level correlation in ln p
    Sa = pkg.build_sa(spec5, base, sigma_T=0.5, L_T=L3, sigma_vmr=0.3, L_vmr=L3)

    def scenes(n, seed):  # the sampler's T and H2O on the US-standard pressure grid
        prof, ang = pkg.synthetic.perturbed_profiles(n, seed=seed)
        sc = [pkg.AtmosphericProfile(base.pressure, p.temperature, base.altitude, {**base.vmr, 1: p.vmr[1]})
              for p in prof]
        return sc, ang, [pkg.ViewingGeometry(pkg.scan_angle_to_local_zenith(a)) for a in ang]

    truth, ang, geoms = scenes(n_sc, 1004)
    nu5, _, bt5 = pkg.forward_model_batch(truth, l5, sounder=s5, geoms=geoms, backend=ctx, dptmn=0.0, **kw5)
    rng = np.random.default_rng(1004)
    se = np.stack([pkg.scene_nedt(nu5, b, nedt_280K=0.2) ** 2 for b in bt5])
    y = bt5 + np.sqrt(se) * rng.standard_normal(bt5.shape)
    # the surrogate: trained only on GPU-LBL spectra
    t0 = time.perf_counter()
    tr, tr_ang, tr_geoms = scenes(n_train, 1005)
    _, _, bt_tr = pkg.forward_model_batch(tr, l5, sounder=s5, geoms=tr_geoms, backend=ctx, precision="mixed",
                                          **kw5)
    X = pkg.surrogate_features(tr, tr_ang)
    sur = pkg.Surrogate(ctx, n_in=X.shape[1], n_hidden=512, n_layers=3, n_out=bt_tr.shape[1], seed=1004)
    sur.fit_scaling(X, bt_tr)
    sur.train(X, bt_tr.astype(np.float32), epochs=200, batch=256, lr=1e-3, seed=1004)
    t_train = time.perf_counter() - t0
    t0 = time.perf_counter()
    x0 = pkg.surrogate_first_guess(sur, y, spec5, [base] * n_sc, ang, xa=xa, Sa=Sa, Se=se)
    t_fg = time.perf_counter() - t0
    sur.close()
    okw = dict(sounder=s5, geoms=geoms, backend=ctx, fm_kwargs=kw5)
    pkg.optimal_estimation_batch(y[:64], spec5, [base] * 64, l5, xa=xa, Sa=Sa, Se=se[:64], max_iter=1,
                                 sounder=s5, geoms=geoms[:64], backend=ctx, fm_kwargs=kw5)  # workspaces
    res = {}
    for name, start in (("surrogate", x0), ("a_priori", None)):
        t0 = time.perf_counter()
        r = pkg.optimal_estimation_batch(y, spec5, [base] * n_sc, l5, xa=xa, Sa=Sa, Se=se, x0=start, **okw)
        res[name] = (time.perf_counter() - t0, r)
    t_oe, r = res["surrogate"]
    hist = np.bincount(r["n_iter"].astype(int))
    hist_a = np.bincount(res["a_priori"][1]["n_iter"].astype(int))
    return {
        "metric": "retrieved scenes/s (batched LM optimal estimation from the surrogate's first guess: GPU "
                  "forward + analytic Jacobian + FP64 Cholesky)",
        "value": n_sc / (t_oe + t_fg), "unit": "scenes/s", "scenes": n_sc,
        "converged": int(r["converged"].sum()),
        "timing": "host wall clock: surrogate first guess + retrieval (training not included)",
        "first_guess_s": t_fg, "retrieval_s": t_oe, "surrogate_training_s": t_train,
        "iterations": {"mean": float(r["n_iter"].mean()), "max": int(r["n_iter"].max()),
                       "histogram": {str(k): int(v) for k, v in enumerate(hist) if v}},
        "from_a_priori": {"value": n_sc / res["a_priori"][0], "converged": int(res["a_priori"][1]["converged"].sum()),
                          "iterations_mean": float(res["a_priori"][1]["n_iter"].mean()),
                          "histogram": {str(k): int(v) for k, v in enumerate(hist_a) if v}},
        "config": {"workload": "oe-5k-co2 (config 4 scenes on the 5,000-line list)", "lines": 5000,
                   "channels": len(nu5), "n_state": spec5.n,
                   "prior": "build_sa matern52, sigma_T 0.5 K, sigma_logH2O 0.3, L = 3 x median |d ln p|",
                   "noise": "diagonal Se from scene_nedt(0.2 K at 280 K)",
                   "first_guess": f"MLP surrogate 152 -> 3 x 512 -> 221 trained on {n_train} GPU-LBL spectra",
                   "scenes": "perturbed-AFGL sampler (seed 1004) on the US-standard pressure grid, scan angles"}}


def surrogate_iasi_accuracy(pkg, ctx, lists, n_train: int = 12288, n_test: int = 256, epochs: int = 200):
    """The config-3 network (152 -> 4 x 1024 GELU -> 8461) trained only on n_train GPU-LBL
    IASI spectra (400k lines, mixed precision, the perturbed-AFGL sampler with scan angles)
    and judged by LBL on n_test held-out spectra of the same sampler."""
    t0 = time.perf_counter()
    profs, ang = pkg.synthetic.perturbed_profiles(n_train + n_test, seed=2025)
    geoms = [pkg.ViewingGeometry(pkg.scan_angle_to_local_zenith(a)) for a in ang]
    BT = pkg.forward_model_batch(profs, lists, sounder=pkg.IASIInstrument(), geoms=geoms, backend=ctx,
                                 precision="mixed", **_workload_kw())[2]
    t_lbl = time.perf_counter() - t0
    X = pkg.surrogate_features(profs, ang)
    tr, te = slice(0, n_train), slice(n_train, None)
    t0 = time.perf_counter()
    sur = pkg.Surrogate(ctx, n_in=X.shape[1], n_hidden=1024, n_layers=4, n_out=BT.shape[1], seed=3)
    sur.fit_scaling(X[tr], BT[tr])
    sur.train(X[tr], BT[tr].astype(np.float32), epochs=epochs, batch=256, lr=1e-3, seed=4)
    t_train = time.perf_counter() - t0
    P, ood = sur.predict(X[te])
    sur.close()
    d = P - BT[te]
    per = np.sqrt(np.mean(d ** 2, axis=1))
    clim = float(np.sqrt(np.mean((BT[tr].mean(0) - BT[te]) ** 2)))
    return {"metric": "held-out BT RMS of the MLP surrogate against GPU LBL (IASI, 8461 channels)",
            "value": float(np.sqrt(np.mean(d ** 2))), "unit": "K", "higher_is_better": False,
            "per_profile_median_K": float(np.median(per)), "per_profile_p95_K": float(np.quantile(per, 0.95)),
            "max_K": float(np.max(np.abs(d))), "climatology_rms_K": clim,
            "held_out_flagged_ood": int(np.sum(ood > sur.ood_threshold)),
            "lbl_spectra_s": t_lbl, "training_s": t_train,
            "config": {"workload": "mlp-152-4x1024-8461 on iasi-400k spectra", "train_spectra": n_train,
                       "held_out_spectra": n_test, "epochs": epochs, "batch": 256,
                       "lr": "1e-3, cosine to 1e-5", "sampler": "perturbed AFGL (seed 2025), scan 0-48 deg"}}


def bench_extras(pkg, ctx, lists, snd, torch, stream):
    """Surrogate inference, analytic Jacobian and batched optimal estimation, each on a
    bounded workload of its configuration (stated in its `config`)."""
    out = {}
    peaks, src = _peaks()
    # ---- MLP surrogate: 152 -> 4 x 1024 GELU -> 8461, batches of 4096, BF16 tcgen05
    n_in, n_hid, n_lay, n_out, B = 152, 1024, 4, 8461, 4096
    sur = pkg.Surrogate(ctx, n_in=n_in, n_hidden=n_hid, n_layers=n_lay, n_out=n_out, seed=1003)
    X = torch.randn((B, n_in), device="cuda", dtype=torch.float32)
    Y = torch.empty((B, n_out), device="cuda", dtype=torch.float32)
    ood = torch.empty((B,), device="cuda", dtype=torch.float32)

    def infer():
        pkg.check(ctx.lib.irs_surrogate_infer_device(sur.h, C.c_void_p(X.data_ptr()), B, C.c_void_p(Y.data_ptr()),
                                                     C.c_void_p(ood.data_ptr()), C.c_void_p(stream.cuda_stream)))

    for _ in range(3):
        infer()
    torch.cuda.synchronize()
    reps = 20
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(reps):
        infer()
    b.record(stream)
    torch.cuda.synchronize()
    t = a.elapsed_time(b) / reps / 1e3
    flop = 2.0 * B * (n_in * n_hid + (n_lay - 1) * n_hid * n_hid + n_hid * n_out)
    # end to end through Surrogate.predict with page-locked input and output buffers
    # reused across calls, as a serving loop holds them (the tensors own the memory)
    Xt = torch.from_numpy(np.random.default_rng(0).standard_normal((B, n_in)).astype(np.float32)).pin_memory()
    Pt = torch.empty((B, n_out), dtype=torch.float32).pin_memory()
    Ot = torch.empty((B,), dtype=torch.float32).pin_memory()
    Xh, Ph, Oh = Xt.numpy(), Pt.numpy(), Ot.numpy()
    sur.predict(Xh, out=Ph, ood=Oh)
    t0 = time.perf_counter()
    for _ in range(5):
        sur.predict(Xh, out=Ph, ood=Oh)
    te = (time.perf_counter() - t0) / 5
    out["surrogate"] = {
        "metric": "IASI spectra/s (MLP surrogate inference, batches of 4096)", "value": B / t, "unit": "spectra/s",
        "ms_per_batch": t * 1e3, "dtype": "bf16 weights/activations, fp32 accumulation (tcgen05)",
        "config": {"workload": "mlp-152-4x1024-8461", "batch": B, "weights": "seeded random (throughput only)"},
        "roofline": {"bound": "tensor", "achieved": flop / t / 1e12, "peak": peaks["bf16_tflops"],
                     "unit": "TFLOP/s", "frac": flop / t / 1e12 / peaks["bf16_tflops"],
                     "peak_source": f"{src} bf16_tflops", "flop_per_batch": flop},
        "e2e": {"value": B / te, "unit": "spectra/s", "h2d_bytes_per_step": Xh.nbytes,
                "d2h_bytes_per_step": B * n_out * 4 + B * 4,
                "timing": "host wall clock around Surrogate.predict, page-locked input and output buffers "
                          "reused across calls"},
    }
    sur.close()
    c2 = pkg.B200Context(ctx.device)
    try:
        out["surrogate_accuracy"] = surrogate_iasi_accuracy(pkg, c2, lists)
    finally:
        c2.close()
    # ---- analytic Jacobian: 400k lines + VP_Y on CO2, state T + log H2O + log O3 + T_sfc
    profs, ang = pkg.synthetic.perturbed_profiles(4, seed=1002)
    geoms = [pkg.ViewingGeometry(pkg.scan_angle_to_local_zenith(x)) for x in ang]
    lm = pkg.VPYLineMixing(pkg.synthetic.vpy_y0(len(lists[2])))
    spec = pkg.StateVectorSpec(50, [pkg.H2O, pkg.O3], include_emissivity=False)
    kw = _workload_kw()
    kw.pop("dptmn")
    pkg.analytic_jacobian_batch(profs, lists, spec, sounder=snd, geoms=geoms, backend=ctx,
                                line_mixing=lm, **kw)  # warm-up at full size: workspaces sized outside the timing
    t0 = time.perf_counter()
    pkg.analytic_jacobian_batch(profs, lists, spec, sounder=snd, geoms=geoms, backend=ctx, line_mixing=lm, **kw)
    tj = time.perf_counter() - t0
    dy = np.random.default_rng(1002).standard_normal((len(profs), 8461))
    pkg.vjp_batch(profs, lists, spec, dy, sounder=snd, geoms=geoms, backend=ctx, line_mixing=lm, **kw)
    t0 = time.perf_counter()
    pkg.vjp_batch(profs, lists, spec, dy, sounder=snd, geoms=geoms, backend=ctx, line_mixing=lm, **kw)
    tv = time.perf_counter() - t0
    out["jacobian"] = {
        "metric": "IASI Jacobians/s (analytic, state T + log H2O + log O3 + T_sfc = 151, with VP_Y)",
        "value": len(profs) / tj, "unit": "jacobians/s", "timing": "host wall clock around the C-ABI call, "
        "host buffers (K is 8461 x 151 FP64 per profile)",
        "pullbacks_per_s": len(profs) / tv,
        "pullback": "irs_vjp_batch: dx = K^T dy in reverse mode on the device (K not formed)",
        # executed FP32 FLOPs from ncu's per-op instruction counters on the profiling case
        # (bench.py --profile-jacobian), not timed here
        "roofline": {"bound": "fp32", "kernel": "jg_linesum_kernel<1, 7>", "achieved": 10.3, "peak": 74.4,
                     "unit": "TFLOP/s", "frac": 10.3 / 74.4, "issue_slots_used": 0.34,
                     "measured": "ncu sass op counters, 2 profiles x 645-1000 cm^-1 x 151-element state, "
                                 "3.07e11 FP32 FLOP in 29.8 ms"},
        "config": {"workload": "iasi-400k-lm", "profiles": len(profs), "n_state": spec.n, "channels": 8461}}
    # ---- relaxation-matrix line mixing on the 400k-line IASI workload (6 AFGL profiles)
    relmat = pkg.synthetic.synthetic_relmat(n_bands=6, j_max=60)
    profs6 = [pkg.afgl_atmosphere(n) for n in pkg.synthetic.AFGL]
    kw6 = _workload_kw()
    for name, lmx in (("vpy_relmat", pkg.VPYLineMixing(relmat)), ("vpw_relmat", pkg.VPWLineMixing(relmat, n_top=5))):
        pkg.forward_model_batch(profs6, lists, sounder=snd, backend=ctx, precision="mixed", line_mixing=lmx, **kw6)
        t0 = time.perf_counter()
        pkg.forward_model_batch(profs6, lists, sounder=snd, backend=ctx, precision="mixed", line_mixing=lmx, **kw6)
        tl = time.perf_counter() - t0
        st = ctx.stage_times()
        out[name] = {
            "metric": f"IASI spectra/s (forward_model, 400k lines, mixed, {type(lmx).__name__} on relaxation-matrix "
                      "data)", "value": len(profs6) / tl, "unit": "spectra/s",
            "timing": "host wall clock around the C-ABI call, host buffers",
            "lm_host_ms": st.lm_host_ms, "lm_device_ms": st.lm_device_ms, "line_sum_ms": st.line_sum_ms,
            "config": {"workload": "iasi-400k + synthetic relmat", "relmat_bands": len(relmat.bands),
                       "relmat_lines": int(sum(len(b.lines) for b in relmat.bands)),
                       "vpw_bands": sorted(getattr(lmx, "whitelist", set())),
                       "host_threads": os.cpu_count()}}
    # the two runs below size workspaces for thousands of profiles: each gets a context of
    # its own, closed afterwards, so that memory is returned before the next measurement
    c2 = pkg.B200Context(ctx.device)
    try:
        out["optimal_estimation"] = oe_config4(pkg, c2)
    finally:
        c2.close()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--plain-steps", type=int, default=2)
    ap.add_argument("--batch", type=int, default=GLOBAL_BATCH,
                    help="profiles per step over all GPUs (split into contiguous shards per rank)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the surrogate, Jacobian and optimal-estimation measurements")
    ap.add_argument("--profile-case", action="store_true",
                    help="run a small case of the line-sum kernels for ncu: the 400k-line list, one "
                         "profile, 645-1000 cm^-1, mixed then plain FP64, twice each")
    ap.add_argument("--profile-jacobian", action="store_true",
                    help="run a small case of the Jacobian kernels for ncu: the 400k-line list with VP_Y "
                         "line mixing on CO2, two perturbed profiles, 645-1000 cm^-1, state T + log H2O + "
                         "log O3 + T_sfc, twice")
    ap.add_argument("--profile-surrogate", action="store_true",
                    help="run the MLP surrogate (152 -> 4 x 1024 -> 8461) on three batches of 4096 for ncu")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.profile_surrogate:
        pkg = _package()
        ctx = pkg.B200Context(0)
        sur = pkg.Surrogate(ctx, n_in=152, n_hidden=1024, n_layers=4, n_out=8461, seed=1003)
        X = np.random.default_rng(0).standard_normal((4096, 152)).astype(np.float32)
        for _ in range(3):
            t0 = time.perf_counter()
            Y, ood = sur.predict(X)
            print(json.dumps({"batch": 4096, "wall_s": time.perf_counter() - t0,
                              "finite": bool(np.isfinite(Y).all())}), flush=True)
        sur.close()
        ctx.close()
        return
    if args.profile_jacobian:
        pkg = _package()
        ctx = pkg.B200Context(0)
        lists = pkg.synthetic.lists_iasi_400k()
        lm = pkg.VPYLineMixing(pkg.synthetic.vpy_y0(len(lists[2])))
        snd = pkg.Sounder.make(645.0, 1000.0, 0.25, opd_max=2.0, fwhm_gauss=0.5)
        profs, ang = pkg.synthetic.perturbed_profiles(2)
        geoms = [pkg.ViewingGeometry(pkg.scan_angle_to_local_zenith(a)) for a in ang]
        spec = pkg.StateVectorSpec(len(profs[0].pressure), [pkg.H2O, pkg.O3], include_emissivity=False)
        kw = _workload_kw()
        kw.pop("dptmn")
        for _ in range(2):
            t0 = time.perf_counter()
            _, K, _ = pkg.analytic_jacobian_batch(profs, lists, spec, sounder=snd, geoms=geoms, backend=ctx,
                                                  line_mixing=lm, **kw)
            print(json.dumps({"jacobians": len(profs), "n_state": K.shape[2], "n_ch": K.shape[1],
                              "wall_s": time.perf_counter() - t0}), flush=True)
        ctx.close()
        return
    if args.profile_case:
        pkg = _package()
        ctx = pkg.B200Context(0)
        lists = pkg.synthetic.lists_iasi_400k()
        snd = pkg.Sounder.make(645.0, 1000.0, 0.25, opd_max=2.0, fwhm_gauss=0.5)
        for prec in ("mixed", "mixed", "fp64", "fp64"):
            pkg.forward_model(pkg.afgl_atmosphere(), lists, sounder=snd, backend=ctx, precision=prec,
                              method=pkg.FullFaddeeva, **_workload_kw())
            t = ctx.stage_times()
            print(json.dumps({"precision": prec, "line_sum_ms": t.line_sum_ms, "pairs": t.pairs,
                              "core_pairs": t.core_pairs}), flush=True)
        ctx.close()
        return

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        reference_arm(args, rank)
        return

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        return reduce_max(dist, x, "cuda")

    pkg = _package()
    ctx = pkg.B200Context(local)
    lists = pkg.synthetic.lists_iasi_400k()
    afgl = [pkg.afgl_atmosphere(a) for a in pkg.synthetic.AFGL][:N_PROF]
    # the global batch (strong scaling: fixed total work, contiguous shards per rank)
    profs_all = [afgl[k % N_PROF] for k in range(args.batch)]
    first, count = pkg.shard_range(args.batch, world, rank)
    if count < 1:
        raise SystemExit(f"a batch of {args.batch} profiles leaves rank {rank} of {world} without work")
    snd = pkg.IASIInstrument()
    pkg._prepare(ctx, lists, None)
    lib = ctx.lib

    def options(prec):
        return pkg.fm_options(precision=prec, method=pkg.FullFaddeeva, **_workload_kw())

    s = snd.c_struct()
    nch = 8461
    # a real (non-default) stream: the library orders its own stream after this one
    # on entry and this one after its work on exit, so events here bracket the work
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)

    class Batch:
        def __init__(self, profs):
            self.n = len(profs)
            self.b = pkg._ProfileBatch(profs, [None] * self.n, [1.0] * self.n, [1.0] * self.n)
            self.R = torch.empty((self.n, nch), dtype=torch.float64, device="cuda")
            self.BT = torch.empty_like(self.R)

        def step(self, opt):
            pkg.check(lib.irs_forward_model_batch_device(ctx.h, self.b.arr, self.n, C.byref(s), C.byref(opt),
                                                         C.c_void_p(self.R.data_ptr()),
                                                         C.c_void_p(self.BT.data_ptr()),
                                                         C.c_void_p(stream.cuda_stream)))

    def device_ms(b, opt, steps, warm):
        for _ in range(warm):
            b.step(opt)
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            b.step(opt)
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        return max_over_ranks(e0.elapsed_time(e1) / steps)

    mine = Batch(profs_all[first:first + count])  # this rank's shard of the global batch
    six = Batch(afgl)                              # the six AFGL profiles (per-rank lines)

    # ---------------- value: mixed path, inputs resident, CUDA events
    om = options("mixed")
    for _ in range(args.warmup):
        mine.step(om)
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(_physical_gpu(local)) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            mine.step(om)
        e1.record(stream)
        torch.cuda.synchronize()
    barrier()
    ms = max_over_ranks(e0.elapsed_time(e1) / args.steps)
    value = args.batch / (ms / 1e3)

    # per-stage device times (library events on its launching stream), averaged
    acc = {"line_params_ms": 0.0, "line_sum_ms": 0.0, "rte_ms": 0.0, "ils_ms": 0.0}
    for _ in range(args.steps):
        mine.step(om)
        pkg.check(lib.irs_synchronize(ctx.h))
        st = ctx.stage_times()
        for k in acc:
            acc[k] += getattr(st, k) / args.steps
    pairs, core, evald = st.pairs, st.core_pairs, st.evaluated_pairs
    launches_per_step = st.launches
    t_ls = acc["line_sum_ms"] / 1e3
    # FLOPs of the pair evaluations the kernel issued: near lines at every block point,
    # far lines at the 8 interpolation nodes (the algorithmic pair count is larger)
    flops = FAR_PAIR_FLOPS * (evald - core) + CORE_PAIR_FLOPS * core
    clocks = clk.summary()
    f_sm = (clocks["sm_mhz"] or 1965.0) * 1e6
    peak = FP32_LANES * 2 * f_sm / 1e12
    achieved = flops / t_ls / 1e12
    traffic = _traffic_from_profiles()

    # ---------------- weak scaling: the six AFGL profiles on every rank
    ms6 = device_ms(six, om, max(2, args.steps // 2), 1)
    weak = {"value": weak_scaling_value(world, N_PROF, ms6), "unit": "spectra/s", "ms_per_step": ms6,
            "profiles_per_rank": N_PROF, "scaling": "weak"}

    # ---------------- e2e: host C-ABI call, host buffers in and out
    Rh = (C.c_double * (count * nch))()
    BTh = (C.c_double * (count * nch))()
    for _ in range(2):
        pkg.check(lib.irs_forward_model_batch(ctx.h, mine.b.arr, count, C.byref(s), C.byref(om), Rh, BTh))
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        pkg.check(lib.irs_forward_model_batch(ctx.h, mine.b.arr, count, C.byref(s), C.byref(om), Rh, BTh))
    t_e2e = max_over_ranks((time.perf_counter() - t0) / args.steps)
    st = ctx.stage_times()
    e2e = {"value": args.batch / t_e2e, "unit": "spectra/s",
           "h2d_bytes_per_step": int(st.h2d_bytes), "d2h_bytes_per_step": int(st.d2h_bytes),
           "timing": "host wall clock around the synchronous C-ABI call, max over ranks"}

    # ---------------- plain FP64 and direct FP32 kernels on the six AFGL profiles
    ms64 = device_ms(six, options("fp64"), args.plain_steps, 1)
    plain = world * N_PROF / (ms64 / 1e3)
    ms_d = device_ms(six, options("mixed_direct"), args.plain_steps, 1)
    BTd = six.BT.clone()

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        run, n_pts, n_full, cores, c0, n_ch = cpu_sample()
        tc = run()
        cpu = {"value": n_pts / n_full / tc, "unit": "spectra/s", "cores": cores, "kind": "port",
               "sample": f"FP64 oracle, one AFGL profile, channels {c0}..{c0 + n_ch - 1} ({n_pts} of "
                         f"{n_full} internal grid points), scaled by grid points"}

    extras = {}
    if world == 1 and not args.no_extras:
        extras = bench_extras(pkg, ctx, lists, snd, torch, stream)
        pkg._prepare(ctx, lists, None)

    # consistency check of this run: mixed vs FP64 BT on the six AFGL profiles
    six.step(om)
    torch.cuda.synchronize()
    BTm = six.BT.clone()
    six.step(options("fp64"))
    torch.cuda.synchronize()
    d = (BTm - six.BT)
    bt_rms = float(torch.sqrt(torch.mean(d * d)).item())
    bt_max = float(d.abs().max().item())
    dd = BTm - BTd
    far_max = float(dd.abs().max().item())

    if rank == 0:
        plain_d = {"value": plain, "unit": "spectra/s", "ms_per_step": ms64, "mixed_over_plain": value / plain}
        direct_d = {"value": world * N_PROF / (ms_d / 1e3), "unit": "spectra/s", "ms_per_step": ms_d,
                    "bt_far_field_vs_direct_max_K": far_max}
        line = {
            "metric": METRIC,
            "value": value, "unit": "spectra/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f32+kahan (fp64 cumulative optical depth and transmittance)",
            "data": "synthetic (seeded line lists, AFGL profiles)",
            "config": workload_config(),
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "kernel": "linesum_mixed_kernel<3>",
                         "algorithmic_pairs_per_s": pairs / t_ls,
                         "peak_source": "148 SMs x 128 FP32 lanes x 2 FLOP x median sampled SM clock "
                                        "(MEASURED_PEAKS.json has no FP32 figure)",
                         # the comparators of the headline, as scalars
                         "plain_fp64_spectra_per_s": plain, "mixed_over_plain_fp64": value / plain,
                         "mixed_direct_spectra_per_s": direct_d["value"],
                         "bt_rms_mixed_vs_fp64_K": bt_rms, "bt_max_mixed_vs_fp64_K": bt_max,
                         "bt_max_far_field_vs_direct_K": far_max,
                         "work": {"pairs": pairs, "evaluated_pairs": evald, "core_pairs": core,
                                  "far_flops": FAR_PAIR_FLOPS, "core_flops": CORE_PAIR_FLOPS}},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": int(launches_per_step * args.steps),
            "clocks": clocks,
            "stages_ms": acc,
            "profiles_per_step": args.batch, "profiles_this_rank": count,
            "weak_scaling": weak,
        }
        # the RTE kernel against HBM: it reads the FP32 optical depths once and writes I
        rte_bytes = count * 49 * 858801 * 4 + count * 858801 * 8
        peaks, psrc = _peaks()
        line["rte"] = {"kernel": "rte_mixed_kernel", "ms_per_step": acc["rte_ms"], "bytes_per_step": rte_bytes,
                       "achieved_gbs": rte_bytes / (acc["rte_ms"] / 1e3) / 1e9, "peak_gbs": peaks["hbm_gbs"],
                       "frac": rte_bytes / (acc["rte_ms"] / 1e3) / 1e9 / peaks["hbm_gbs"],
                       "peak_source": f"{psrc} hbm_gbs"}
        line.update(extras)
        # last, so that a cut-off log still shows them
        line["plain_fp64"] = plain_d
        line["mixed_direct"] = direct_d
        line["bt_mixed_vs_fp64_K"] = {"rms": bt_rms, "max": bt_max}
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
