"""Train the IASI MLP surrogate on spectra of the GPU line-by-line path and judge it.

    python irsounderlbl.jl_b200/train_surrogate.py [--n-train N] [--n-test M] [--epochs E]
                                                   [--batch B] [--lr LR] [--out weights.npz]

Profiles come from the perturbed-AFGL sampler (T noise N(0, C), C_ij = 9 exp(-|i-j|/3);
H2O and O3 scaled by exp(N(0, 0.2^2)); scan angle U(0, 48 deg)).  Their BTs are computed
by forward_model_batch (400,000-line six-species list, IASI, mixed precision) in
batches; the network (152 -> 4 x 1024 GELU -> 8461) is trained on the tensor cores;
the held-out profiles are judged against LBL and the inference throughput is timed.
Prints one JSON line.  The LBL spectra dominate the run time.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def _package():
    if "irs_b200" in sys.modules:
        return sys.modules["irs_b200"]
    spec = importlib.util.spec_from_file_location("irs_b200", HERE / "__init__.py",
                                                  submodule_search_locations=[str(HERE)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["irs_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n-train", type=int, default=4096)
    ap.add_argument("--n-test", type=int, default=256)
    ap.add_argument("--epochs", type=int, default=300)
    ap.add_argument("--batch", type=int, default=256)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--lbl-batch", type=int, default=48)
    ap.add_argument("--seed", type=int, default=1003)
    ap.add_argument("--out", type=str, default=None)
    args = ap.parse_args()
    pkg = _package()
    ctx = pkg.B200Context()
    lists = pkg.synthetic.lists_iasi_400k()
    snd = pkg.IASIInstrument()
    n = args.n_train + args.n_test
    profs, ang = pkg.synthetic.perturbed_profiles(n, seed=args.seed)
    kw = dict(precision="mixed", internal_dnu=0.0025, apply_continuum=True, continua=("h2o", "co2"))
    t0 = time.perf_counter()
    BT = []
    for b0 in range(0, n, args.lbl_batch):
        pb = profs[b0:b0 + args.lbl_batch]
        geoms = [pkg.ViewingGeometry(pkg.scan_angle_to_local_zenith(a)) for a in ang[b0:b0 + args.lbl_batch]]
        BT.append(pkg.forward_model_batch(pb, lists, sounder=snd, geoms=geoms, backend=ctx, **kw)[2])
    BT = np.concatenate(BT)
    t_lbl = time.perf_counter() - t0
    X = pkg.surrogate_features(profs, ang)
    tr, te = slice(0, args.n_train), slice(args.n_train, n)
    sur = pkg.Surrogate(ctx, n_in=X.shape[1], n_hidden=1024, n_layers=4, n_out=BT.shape[1], seed=args.seed)
    sur.fit_scaling(X[tr], BT[tr])
    t0 = time.perf_counter()
    losses = sur.train(X[tr], BT[tr].astype(np.float32), epochs=args.epochs, batch=args.batch, lr=args.lr,
                       seed=args.seed)
    t_train = time.perf_counter() - t0
    P, ood = sur.predict(X[te])
    d = P - BT[te]
    clim = BT[tr].mean(0)
    Xb = np.repeat(X[te], (4096 + args.n_test - 1) // args.n_test, axis=0)[:4096]
    sur.predict(Xb)
    t0 = time.perf_counter()
    for _ in range(5):
        sur.predict(Xb)
    t_inf = (time.perf_counter() - t0) / 5
    per_prof = np.sqrt(np.mean(d ** 2, axis=1))
    out = {
        "n_train": args.n_train, "n_test": args.n_test, "epochs": args.epochs,
        "lbl_spectra_per_s": n / t_lbl, "train_s": t_train,
        "loss_first_last": [float(losses[0]), float(losses[-1])],
        "heldout_bt_rms_K": float(np.sqrt(np.mean(d ** 2))), "heldout_bt_max_K": float(np.max(np.abs(d))),
        "heldout_rms_per_profile_K": {"median": float(np.median(per_prof)), "p95": float(np.quantile(per_prof, 0.95))},
        "climatology_bt_rms_K": float(np.sqrt(np.mean((BT[te] - clim) ** 2))),
        "ood_threshold": sur.ood_threshold, "heldout_ood_fraction": float(np.mean(ood > sur.ood_threshold)),
        "inference_spectra_per_s_e2e": 4096 / t_inf,
    }
    print(json.dumps(out), flush=True)
    if args.out:
        np.savez(args.out, params=sur.get_params(), x_mean=sur.x_mean, x_sd=sur.x_sd, y_mean=sur.y_mean,
                 y_sd=sur.y_sd, ood_threshold=sur.ood_threshold)
    sur.close()
    ctx.close()


if __name__ == "__main__":
    main()
