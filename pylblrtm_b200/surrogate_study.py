"""Train the channel-transmittance surrogate on engine spectra and measure gated inference.

    python -m pylblrtm_b200.surrogate_study --train 100000 --eval 65536 --steps 20000 --out study.json

Steps (all on one GPU):
  1. draw ``--train`` perturbed 20-layer profiles and compute their 2,000 channel-mean
     transmittances (650-1150 cm^-1, 0.25 cm^-1 channels, grid step 0.001) with the
     float32 line-by-line engine: the training targets;
  2. train a 4-member ensemble (61 -> 1024 x 4 -> 2000, BF16, Adam, batch 4096);
  3. calibrate the gate on ``--calibrate`` further in-distribution profiles with their
     engine spectra (per-channel spread weights and a threshold such that accepted
     profiles keep the 99.9th percentile of their maximum channel error <= ``--gate``;
     ``--calibrate 0`` keeps the raw spread compared with ``--gate``);
  4. draw ``--eval`` fresh profiles plus a fraction ``--ood`` shifted by +25 K, compute
     their engine spectra (the reference values for the surrogate's errors, and the engine's
     own spectra/s),
     run the ensemble (surrogate-only spectra/s), and the gated path that recomputes
     flagged profiles with the engine (blended spectra/s);
  5. report per-profile maximum channel errors (quantiles, fraction <= 1e-3) for the
     ensemble mean, the profiles the gate accepts and the gated output, split in/out of
     distribution.

The line list is the three-gas synthetic list (200,000 lines over 600-2500 cm^-1)
restricted to the window plus the cutoff; ``--strength-scale`` multiplies every line
strength (at scale 1 every channel of this window is saturated, T < 1e-10).
"""

from __future__ import annotations

import argparse
import json
import time
from typing import Dict

import numpy as np

from . import surrogate, synthetic


def _quantiles(a: np.ndarray) -> Dict[str, float]:
    if a.size == 0:
        return {}
    q = np.quantile(a, [0.5, 0.9, 0.99, 0.999])
    return {"p50": float(q[0]), "p90": float(q[1]), "p99": float(q[2]), "p99.9": float(q[3]),
            "max": float(a.max()), "frac_le_1e-3": float(np.mean(a <= 1e-3))}


def _profile_stats(gs, raw, ref, chunk: int = 8192) -> Dict[str, np.ndarray]:
    """Per-profile statistics of the ensemble on ``raw`` features against the engine's
    ``ref`` channels: max and mean channel spread, the spread weighted by the gate's
    channel weights, and the ensemble mean's max channel error."""
    import torch
    out = {k: [] for k in ("spread_max", "spread_mean", "spread_weighted", "err_max")}
    w = gs.ch_scale
    for a in range(0, raw.shape[0], chunk):
        pred = gs.predictions(torch.as_tensor(raw[a:a + chunk], device=gs.members[0].dev))
        sp = pred.std(0, unbiased=False)
        err = (pred.mean(0) - torch.as_tensor(ref[a:a + chunk], device=sp.device)).abs().max(1).values
        out["spread_max"].append(sp.max(1).values.cpu().numpy())
        out["spread_mean"].append(sp.mean(1).cpu().numpy())
        out["spread_weighted"].append((sp * w[None, :]).max(1).values.cpu().numpy() if w is not None
                                      else sp.max(1).values.cpu().numpy())
        out["err_max"].append(err.cpu().numpy())
    return {k: np.concatenate(v) for k, v in out.items()}


def line_list(n_lines: int, problem: surrogate.SurrogateProblem, strength_scale: float):
    sd = synthetic.three_gas_lines(n_lines)
    sd = synthetic.restrict(sd, problem.nu_min - problem.cutoff, problem.nu_max + problem.cutoff)
    return synthetic.scale_strengths(sd, strength_scale) if strength_scale != 1.0 else sd


def run(n_train: int = 100_000, n_eval: int = 65_536, ood: float = 0.05, steps: int = 20_000,
        members: int = 4, batch: int = 4096, hidden: int = 1024, depth: int = 4, lr: float = 1e-3,
        strength_scale: float = 1e-4, n_lines: int = 200_000, gate: float = 1e-3, seed: int = 0,
        profiles_per_launch: int = 256, infer_batch: int = 0, n_calibrate: int = 8192, log=print,
        dump: str = None, train_widen: float = 1.3) -> dict:
    """The study; ``infer_batch`` > 0 also times surrogate-only inference on that many
    fresh profiles (features only, no engine reference)."""
    import torch
    problem = surrogate.SurrogateProblem()
    sd = line_list(n_lines, problem, strength_scale)
    rep = {"train_widen": train_widen,
           "problem": {"nu": [problem.nu_min, problem.nu_max], "step": problem.step,
                       "channel_width": problem.channel_width, "n_channels": problem.n_channels,
                       "lines": int(sd.lines["nu0"].size), "strength_scale": strength_scale, "layers": 20},
           "network": {"inputs": 61, "hidden": [hidden] * depth, "outputs": problem.n_channels,
                       "members": members, "batch": batch, "steps": steps, "lr": lr}}

    # 1. training data from the engine
    # training profiles: the workload's distribution with its temperature and H2O spreads
    # widened by train_widen (1.3 by default), so that the tails of the workload's own
    # distribution, where the network errs most, are better covered; calibration and
    # evaluation always draw from the workload's own distribution (at train_widen = 1.3
    # the in-distribution profiles above 1e-3 went from 1.2 % to 0.36 % of the 65,536)
    train = surrogate.sample_profiles(n_train, seed=seed, t_sigma=5.0 * train_widen,
                                      h2o_log_sigma=0.3 * train_widen)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    y = surrogate.engine_channels(sd, train, problem, profiles_per_launch=profiles_per_launch)
    torch.cuda.synchronize()
    t_gen = time.perf_counter() - t0
    x = train.features()
    rep["data"] = {"profiles": n_train, "seconds": t_gen, "engine_spectra_per_s": n_train / t_gen,
                   "target_quantiles": [float(v) for v in np.quantile(y, [0, 0.1, 0.5, 0.9, 1])]}
    log(f"data: {n_train} spectra in {t_gen:.1f} s")

    # 2. ensemble training (a training set smaller than one batch trains on all of it)
    batch = max(128, min(batch, n_train // 128 * 128))
    rep["network"]["batch"] = batch
    t0 = time.perf_counter()
    cfg = surrogate.TrainConfig(batch=batch, steps=steps, lr=lr, lr_final=lr * 1e-2, warmup=min(200, steps // 10),
                                seed=seed + 1)
    nets = surrogate.train_ensemble(x, y, n_members=members, cfg=cfg, hidden=hidden, depth=depth)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    rep["training"] = {"seconds": t_train, "steps_per_s": members * steps / t_train,
                       "final_mse": [float(np.mean(n.train_losses[-50:])) for n in nets]}
    log(f"training: {members} x {steps} steps in {t_train:.1f} s")

    # 3. gate calibration on a split of its own
    gs = surrogate.GatedSurrogate(nets, gate=gate)
    if n_calibrate:
        cal = surrogate.sample_profiles(n_calibrate, seed=seed + 5)
        y_cal = surrogate.engine_channels(sd, cal, problem, profiles_per_launch=profiles_per_launch)
        rep["calibration"] = surrogate.calibrate_gate(gs, cal.features(), y_cal, target=gate)
        log(f"gate calibrated on {n_calibrate} profiles: threshold {gs.gate:.3e}, "
            f"accepted {rep['calibration']['accepted']:.4f}")

    # 4. evaluation profiles and their engine spectra
    n_ood = int(round(ood * n_eval))
    ev_in = surrogate.sample_profiles(n_eval, seed=seed + 2)
    ev_ood = surrogate.sample_profiles(n_ood, seed=seed + 3, t_offset=25.0) if n_ood else None
    ev = ev_in if ev_ood is None else surrogate.ProfileBatch(
        *(np.concatenate([getattr(ev_in, f), getattr(ev_ood, f)]) for f in ("p_atm", "t", "vmr", "air_col", "mu")))
    is_ood = np.r_[np.zeros(n_eval, bool), np.ones(n_ood, bool)]
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ref = surrogate.engine_channels(sd, ev, problem, profiles_per_launch=profiles_per_launch)
    torch.cuda.synchronize()
    t_eng = time.perf_counter() - t0
    log(f"engine on {len(ev)} evaluation profiles: {t_eng:.1f} s")

    raw = torch.as_tensor(ev.features(), device=nets[0].dev)
    gs.ensemble(raw[:1024])                                       # warm-up (workspaces)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    mean, est, flag = gs.ensemble(raw)
    e1.record()
    torch.cuda.synchronize()
    t_sur = e0.elapsed_time(e1) / 1e3
    timings = {}
    out, _, _ = gs(sd, ev, problem, timings=timings)
    t_blend = timings["surrogate_s"] + timings["fallback_s"]

    mean_h, est_h, flag_h, out_h = (mean.cpu().numpy(), est.cpu().numpy(), flag.cpu().numpy(), out.cpu().numpy())
    err_sur = np.abs(mean_h - ref).max(1)
    err_gated = np.abs(out_h - ref).max(1)
    acc = ~flag_h
    rep["throughput"] = {
        "engine_spectra_per_s": len(ev) / t_eng,
        "surrogate_only_spectra_per_s": len(ev) / t_sur,
        "surrogate_only_seconds": t_sur,
        "blended_spectra_per_s": len(ev) / t_blend,
        "blended_seconds": t_blend,
        "speedup_surrogate_only": t_eng / t_sur,
        "speedup_blended": t_eng / t_blend,
        "gemm_flops_per_spectrum": 2 * sum(k * n for k, n in nets[0].dims) * members,
    }
    rep["throughput"]["surrogate_tflops"] = rep["throughput"]["gemm_flops_per_spectrum"] * len(ev) / t_sur / 1e12
    if infer_batch:
        big = torch.as_tensor(surrogate.sample_profiles(infer_batch, seed=seed + 4).features(), device=nets[0].dev)
        gs.ensemble(big)
        torch.cuda.synchronize()
        reps = 5
        e0.record()
        for _ in range(reps):
            gs.ensemble(big)
        e1.record()
        torch.cuda.synchronize()
        t_big = e0.elapsed_time(e1) / 1e3 / reps
        rep["throughput"]["infer_batch"] = {
            "profiles": infer_batch, "seconds": t_big, "spectra_per_s": infer_batch / t_big,
            "tflops": rep["throughput"]["gemm_flops_per_spectrum"] * infer_batch / t_big / 1e12,
            "launches": gs.launches}
    if dump:            # per-profile data for studying error estimates (features, spreads, errors)
        d = {"train_mean": x.mean(0), "train_cov": np.cov(x, rowvar=False), "eval_features": ev.features(),
             "eval_ood": is_ood, **{f"eval_{k}": v for k, v in _profile_stats(gs, ev.features(), ref).items()}}
        if n_calibrate:
            d.update({"cal_features": cal.features(),
                      **{f"cal_{k}": v for k, v in _profile_stats(gs, cal.features(), y_cal).items()}})
        np.savez_compressed(dump, **d)
    rep["gate"] = {"gate": gs.gate, "target": gate, "calibrated": bool(n_calibrate),
                   "flagged_in": float(flag_h[~is_ood].mean()),
                   "flagged_ood": float(flag_h[is_ood].mean()) if n_ood else None,
                   "n_flagged": int(flag_h.sum()), "n_eval": len(ev)}
    rep["errors"] = {
        "surrogate_in": _quantiles(err_sur[~is_ood]),
        "surrogate_ood": _quantiles(err_sur[is_ood]),
        "accepted": _quantiles(err_sur[acc]),
        "accepted_in": _quantiles(err_sur[acc & ~is_ood]),
        "gated_all": _quantiles(err_gated),
        "channel_abs_err_in": _quantiles(np.abs(mean_h - ref)[~is_ood].ravel()),
        "spread_vs_error_corr": float(np.corrcoef(est_h, err_sur)[0, 1]),
    }
    return rep


def infer_only(batch: int, members: int = 4, hidden: int = 1024, depth: int = 4, reps: int = 5,
               seed: int = 0) -> dict:
    """Surrogate-only inference timing with randomly initialised members (no engine, no
    training): the cost of the ensemble and gate on ``batch`` profiles."""
    import torch
    problem = surrogate.SurrogateProblem()
    nets = [surrogate.MLP(61, problem.n_channels, hidden=hidden, depth=depth, seed=seed + m)
            for m in range(members)]
    feats = surrogate.sample_profiles(batch, seed=seed).features()
    for n in nets:
        n.set_normalisation(feats.mean(0), feats.std(0))
    gs = surrogate.GatedSurrogate(nets)
    raw = torch.as_tensor(feats, device=nets[0].dev)
    gs.ensemble(raw)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        gs.ensemble(raw)
    e1.record()
    torch.cuda.synchronize()
    t = e0.elapsed_time(e1) / 1e3 / reps
    flops = 2 * sum(k * n for k, n in nets[0].dims) * members * batch
    return {"profiles": batch, "members": members, "seconds": t, "spectra_per_s": batch / t,
            "tflops": flops / t / 1e12, "launches": gs.launches}


def main(argv=None) -> None:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--train", type=int, default=100_000)
    ap.add_argument("--eval", type=int, default=65_536)
    ap.add_argument("--ood", type=float, default=0.05)
    ap.add_argument("--steps", type=int, default=20_000)
    ap.add_argument("--members", type=int, default=4)
    ap.add_argument("--batch", type=int, default=4096)
    ap.add_argument("--hidden", type=int, default=1024)
    ap.add_argument("--depth", type=int, default=4)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--strength-scale", type=float, default=1e-4)
    ap.add_argument("--lines", type=int, default=200_000)
    ap.add_argument("--gate", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--infer-batch", type=int, default=0)
    ap.add_argument("--calibrate", type=int, default=8192, help="calibration profiles for the gate (0: none)")
    ap.add_argument("--dump", default=None, help="write per-profile features, spreads and errors (.npz)")
    ap.add_argument("--train-widen", type=float, default=1.3,
                    help="factor on the training profiles' temperature and H2O spreads")
    ap.add_argument("--profiles-per-launch", type=int, default=256)
    ap.add_argument("--infer-only", action="store_true",
                    help="only time surrogate inference on --infer-batch profiles (random weights)")
    ap.add_argument("--out", default=None)
    a = ap.parse_args(argv)
    if a.infer_only:
        rep = infer_only(a.infer_batch or 65536, a.members, a.hidden, a.depth, seed=a.seed)
        print(json.dumps(rep))
        return
    rep = run(a.train, a.eval, a.ood, a.steps, a.members, a.batch, a.hidden, a.depth, a.lr, a.strength_scale,
              a.lines, a.gate, a.seed, profiles_per_launch=a.profiles_per_launch, infer_batch=a.infer_batch,
              n_calibrate=a.calibrate, dump=a.dump, train_widen=a.train_widen)
    text = json.dumps(rep, indent=1)
    print(text)
    if a.out:
        with open(a.out, "w") as f:
            f.write(text + "\n")


if __name__ == "__main__":
    main()
