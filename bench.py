#!/usr/bin/env python
"""Throughput of the line-by-line engine: Voigt line-evaluations/s and spectra/s.

Workload: 200,000 synthetic lines (H2O-, CO2-, O3-like, 50/30/20) over
600-2500 cm^-1, a 60-layer profile (61 levels uniform in ln p), grid
600-2500 cm^-1 at 0.001 cm^-1 (1,900,001 points), 25 cm^-1 cut-off, 2 cm^-1
reference tiles, mu = 0.8. A step is one full spectrum: every device stage from
levels and line parameters resident in HBM to the transmittance in HBM.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--precision fp32|fp32-direct|fp64]
    python bench.py --impl reference     # the reference's CPU path on this host

Under torchrun (``--shard wavenumber``, the default for more than one rank) the
one spectrum is split by reference tiles: rank r computes a contiguous range of
tiles from only the lines that reach them, and the transmittance pieces are
all-gathered over NCCL inside every step (strong scaling); `value` is the
spectrum's evaluations divided by the slowest rank's time. ``--shard replicas``
instead gives every rank its own spectrum (rank r uses a profile with seeded
temperature/H2O perturbations; weak scaling, no collective in the step).
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Voigt line-evals/s"
UNIT = "line-evals/s"
WORKLOAD = "three_gas_200k_lines_60_layers_600-2500cm-1_step0.001_cutoff25_tile2_mu0.8"
FLOPS_PER_EVAL_FAR = 12      # two-term far-wing form: 5 FFMA + 1 FMUL + 1 RCP (FMA = 2 flops)
# multi-level kernel, per unit of each work category (FMA = 2 flops, RCP = 1):
FLOPS_NODE = 12              # Chebyshev-node evaluation (two-term form)
FLOPS_L3 = 24                # level-3 loop evaluation (clamped five-term form by powers of 1/|z|^2: 2 FMA + max + RCP + 9 FMA)
FLOPS_NEAR = 60              # near-zone point (float continued fraction / float64 rational, average)
FLOPS_CHEB_PER_POINT = 144   # 16 + 8 Clenshaw terms for each of levels 1 and 2 (3 flops a term)
CPU_SAMPLE = (1000.0, 1000.5)  # sub-window timed on the host (all 60 layers)


# DRAM traffic of one lbl_tau_tiles_ml_f32 call on the default workload (200k lines, 60
# layers, 600-2500 cm^-1), from a single-pass ncu capture of its two launches
# (profiles/launches_three_gas_200k_fp32_ml.md): tau_far_kernel 384.53 MB read + 7.91 MB
# written, tau_ml_kernel 391.63 MB read + 451.51 MB written. Each kernel reads the 384 MB
# of line records once; tau_ml_kernel writes the 456 MB optical depth (part of it still in
# L2 when the launch ends).
TAU_ML_DRAM_BYTES = 384.532480e6 + 7.905280e6 + 391.629568e6 + 451.512064e6


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp32-direct", "fp64"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the Jacobian timing")
    ap.add_argument("--no-surrogate", action="store_true", help="skip the gated-surrogate timing")
    ap.add_argument("--no-accuracy", action="store_true", help="skip the accuracy checks")
    ap.add_argument("--shard", default="auto", choices=["auto", "wavenumber", "replicas"],
                    help="multi-rank mode (auto: wavenumber for more than one rank)")
    ap.add_argument("--no-plain", action="store_true", help="skip the float64 / direct float32 timings")
    ap.add_argument("--nu-min", type=float, default=600.0, help="grid start (smaller cases for profiling)")
    ap.add_argument("--nu-max", type=float, default=2500.0, help="grid end (smaller cases for profiling)")
    return ap.parse_args()


def workload(rank: int):
    from pylblrtm_b200 import synthetic
    sd = synthetic.three_gas_lines()
    if rank == 0:
        prof = synthetic.logp_profile()
    else:
        lv = synthetic.perturbed_levels(synthetic.logp_levels(), 1, seed=1000 + rank)
        prof = synthetic.profile_from_levels(lv, 0)
    return sd, prof


# ---------------------------------------------------------------------------- CPU side
_CPU_CACHE = {}


def _cpu_inputs(lo, hi):
    """Workload lines near the sub-window and the layers (cached per process, untimed)."""
    key = (lo, hi)
    if key not in _CPU_CACHE:
        from oracle import restate
        from pylblrtm_b200 import synthetic
        sd = synthetic.restrict(synthetic.three_gas_lines(), lo - 26.0, hi + 26.0)
        prof = synthetic.logp_profile()
        _CPU_CACHE[key] = (sd, restate.build_layers(prof.pressure_hpa, prof.temperature_k, prof.vmr))
    return _CPU_CACHE[key]


def _oracle_layer(args):
    """One layer of the oracle on a sub-window (runs in a worker process)."""
    k, lo, hi = args
    sys.path.insert(0, ROOT)
    from oracle import restate
    sd, (p, t, v, c) = _cpu_inputs(lo, hi)
    sl = slice(k, k + 1)
    nu = restate.grid(lo, hi, 0.001)
    od = restate.optical_depth(nu, sd.lines, sd.tips, sd.molar_masses, p[sl], t[sl],
                               {g: a[sl] for g, a in v.items()}, {g: a[sl] for g, a in c.items()}, 25.0, 2.0)
    n = restate.count_evals(nu, sd.lines, sd.tips, sd.molar_masses, p[sl], t[sl],
                            {g: a[sl] for g, a in v.items()}, {g: a[sl] for g, a in c.items()}, 25.0, 2.0)
    return n, od


def cpu_reference_sample(workers: int):
    """Times the oracle port of the reference path on the sub-window, all 60 layers."""
    lo, hi = CPU_SAMPLE
    jobs = [(k, lo, hi) for k in range(60)]
    if workers <= 1:
        _cpu_inputs(lo, hi)
        t0 = time.perf_counter()
        out = [_oracle_layer(j) for j in jobs]
        dt = time.perf_counter() - t0
    else:
        import multiprocessing as mp
        with mp.get_context("spawn").Pool(workers, initializer=_cpu_inputs, initargs=(lo, hi)) as pool:
            pool.map(_oracle_layer, [(0, lo, hi)] * workers)      # start-up and input generation, untimed
            t0 = time.perf_counter()
            out = pool.map(_oracle_layer, jobs, chunksize=1)
            dt = time.perf_counter() - t0
    evals = sum(n for n, _ in out)
    return evals, dt


def cpu_info():
    model = "unknown"
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return model, os.cpu_count(), len(os.sched_getaffinity(0))


def run_reference(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    model, n_cpu, n_aff = cpu_info()
    workers = n_aff
    for _ in range(a.warmup):
        pass  # the oracle has no warm-up state; the first timed step includes process start-up
    times, evals = [], 0
    for _ in range(a.steps):
        n, dt = cpu_reference_sample(workers)
        times.append(dt)
        evals = n
    t = sum(times)
    value = evals * a.steps / t
    sample = (f"oracle port of pylblrtm/forward.py:157-317, grid {CPU_SAMPLE[0]}-{CPU_SAMPLE[1]} cm^-1 "
              f"(501 points) x 60 layers of the workload, {evals:.3e} evals/step, layer-parallel over "
              f"{workers} spawn workers; CPU {model}")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": a.gpus,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 * t / a.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "sample": f"{CPU_SAMPLE[0]}-{CPU_SAMPLE[1]} cm^-1 x 60 layers"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": workers, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------- GPU side
class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu, self.rows, self.proc = gpu, [], None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def __exit__(self, *exc):
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            self.proc.wait()

    def summary(self):
        sm = [float(r[0]) for r in self.rows if len(r) >= 7 and r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if len(r) >= 7 and r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows if len(r) >= 7 for i in range(4) if r[3 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(sm)}


def adjoint_timing(torch, steps: int = 3, n_batch: int = 256, chunk: int = 32):
    """Forward vs full per-layer Jacobians on the Jacobian workload.

    Lines of the 200k-line set in 1000-1200 cm^-1, grid 1000-1200 cm^-1 at 0.001, mu 0.8;
    d/dT_layer and d/dlnVMR_layer(H2O). (1) one profile (the 60-layer base), every device
    stage of each call; (2) the batch of 256 profiles (base + correlated N(0, 5 K)
    temperature perturbations, H2O x exp(N(0, 0.3))) through the public batched APIs in
    chunks of 32 profiles: transmittance only vs transmittance + Jacobians. CUDA events,
    inputs on the host (the batched calls include their uploads).
    """
    from pylblrtm_b200 import adjoint, batch, engine, synthetic
    sd = synthetic.restrict(synthetic.three_gas_lines(), 1000.0, 1200.0)
    grid = engine.make_grid(1000.0, 1200.0, 0.001, 2.0)
    job = engine.Job(sd, engine.layer_input_from_profile(synthetic.logp_profile()), grid, 25.0)
    g = torch.ones((1, grid.n_nu), dtype=torch.float64, device="cuda")

    def timed(fn, reps=steps):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    fwd = timed(lambda: job.run("fp32", want_od=True))
    jac = timed(lambda: job.jacobian("H2O"))
    vjp = timed(lambda: job.jacobian("H2O", g_tau=g))
    lv = synthetic.perturbed_levels(synthetic.logp_levels(), n_batch, seed=4242)
    gases = ("H2O", "CO2", "O3")
    vmr = {k: lv[k] for k in gases}
    bf = timed(lambda: batch.transmittance_batch(sd, lv["p"], lv["t"], vmr, 1000.0, 1200.0, mu_view=0.8,
                                                 profiles_per_launch=chunk, as_numpy=False), reps=1)
    bj = timed(lambda: adjoint.layer_jacobians_batch(sd, lv["p"], lv["t"], vmr, 1000.0, 1200.0, mu_view=0.8,
                                                     profiles_per_launch=chunk, on_chunk=lambda sl, out: None),
               reps=1)
    return {"workload": "lines 1000-1200 cm^-1 of the 200k-line set, 60 layers, grid 1000-1200 at 0.001",
            "outputs": "od + d tau/dT_layer + d tau/dlnVMR_layer(H2O), [60, 200001] each per profile",
            "forward_ms": fwd, "jacobian_ms": jac, "vjp_ms": vjp, "jacobian_over_forward": jac / fwd,
            "batch": {"profiles": n_batch, "chunk": chunk, "forward_ms": bf, "jacobian_ms": bj,
                      "jacobian_over_forward": bj / bf, "forward_profiles_per_s": n_batch / bf * 1e3,
                      "jacobian_profiles_per_s": n_batch / bj * 1e3}}


def _errors(torch, t_test, t_ref, tau_test, tau_ref):
    """max |dT|, max and median relative tau error (points with tau_ref > 1e-12)."""
    t_test, t_ref = torch.as_tensor(t_test).double().cuda(), torch.as_tensor(t_ref).double().cuda()
    tau_test, tau_ref = torch.as_tensor(tau_test).double().cuda(), torch.as_tensor(tau_ref).double().cuda()
    m = tau_ref > 1e-12
    rel = (tau_test[m] - tau_ref[m]).abs() / tau_ref[m]
    return {"max_abs_dT": float((t_test - t_ref).abs().max()), "max_rel_tau": float(rel.max()),
            "median_rel_tau": float(rel.median()), "points": int(t_ref.numel())}


def _timed_ms(torch, fn, reps):
    """Mean CUDA-event milliseconds of ``reps`` calls of fn (on the current stream)."""
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def plain_and_accuracy(torch, job, sd, prof, grid, evals, fp32_value):
    """The comparison engines and the accuracy of the default one, on the full workload.

    (1) The plain float64 method (every admitted line at every point, Gautschi-type
    Faddeeva in float64, the reference's ``_voigt``/``phi @ S`` work done directly) and
    the direct float32 method: line-evals/s from CUDA-event times of whole spectra, and
    the default engine's ratio to each. (2) The default float32 engine against the
    float64 engine on the full 200k-line, 60-layer, 1.9M-point spectrum at full
    strength (saturated: T ~ 0 almost everywhere) and with line strengths x 1e-3 and
    x 1e-5, where T spans (0, 1) and |dT| tests something. (3) Both engines against the
    reference's own outputs (golden vectors made by running the reference) for the
    2,000-line CO2 band at full strength and x 1e-3.
    """
    from pylblrtm_b200 import engine, synthetic
    out_plain, acc = {}, {}
    run = lambda j, prec: j.run(prec, mu=[0.8], want_od=False, want_tau=True, want_trans=True)
    r64 = run(job, "fp64")                                   # also the float64 warm-up
    ms64 = _timed_ms(torch, lambda: job.run("fp64", mu=[0.8], want_od=False, want_trans=True), 1)
    out_plain["fp64_plain"] = {"ms_per_spectrum": ms64, "line_evals_per_s": evals / (ms64 * 1e-3), "steps": 1,
                               "kernel": "tau_f64_kernel (lbl_tau_tiles_f64)"}
    r32 = run(job, "fp32")
    acc["three_gas_200k_fp32_vs_fp64"] = _errors(torch, r32.trans[0], r64.trans[0], r32.tau[0], r64.tau[0])
    rd = run(job, "fp32-direct")                             # also the direct warm-up
    msd = _timed_ms(torch, lambda: job.run("fp32-direct", mu=[0.8], want_od=False, want_trans=True), 2)
    out_plain["fp32_direct"] = {"ms_per_spectrum": msd, "line_evals_per_s": evals / (msd * 1e-3), "steps": 2,
                                "kernel": "tau_f32_kernel (lbl_tau_tiles_f32)"}
    acc["three_gas_200k_fp32_direct_vs_fp64"] = _errors(torch, rd.trans[0], r64.trans[0], rd.tau[0], r64.tau[0])
    out_plain["fp32_over_fp64"] = fp32_value / out_plain["fp64_plain"]["line_evals_per_s"]
    out_plain["fp32_over_direct"] = fp32_value / out_plain["fp32_direct"]["line_evals_per_s"]
    del r64, r32, rd
    for scale in (1e-3, 1e-5):
        js = engine.Job(synthetic.scale_strengths(sd, scale), engine.layer_input_from_profile(prof), grid, 25.0)
        a64, a32 = run(js, "fp64"), run(js, "fp32")
        e = _errors(torch, a32.trans[0], a64.trans[0], a32.tau[0], a64.tau[0])
        e["T_min"], e["T_max"] = float(a64.trans[0].min()), float(a64.trans[0].max())
        e["points_T_0.01_0.99"] = int(((a64.trans[0] > 0.01) & (a64.trans[0] < 0.99)).sum())
        acc[f"three_gas_200k_x{scale:g}_fp32_vs_fp64"] = e
        del js, a64, a32
    gold_dir = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tests", "golden")
    for name, scale in (("co2_band_full", 1.0), ("co2_band_mid", 1e-3)):
        g = np.load(os.path.join(gold_dir, f"{name}.npz"))
        sdc = synthetic.co2_band()
        if scale != 1.0:
            sdc = synthetic.scale_strengths(sdc, scale)
        gc = engine.make_grid(float(g["nu_min"]), float(g["nu_max"]), float(g["step"]), float(g["tile"]))
        j = engine.Job(sdc, engine.layer_input_from_profile(synthetic.us_standard_atmosphere(["CO2"])), gc,
                       float(g["cutoff"]))
        res = {}
        for prec in ("fp32", "fp64"):
            r = j.run(prec, mu=[float(g["mu"])], want_od=False, want_tau=True, want_trans=True)
            res[prec] = _errors(torch, r.trans[0], g["T"], r.tau[0], g["tau"])
        acc[f"{name}_vs_reference"] = res
    return out_plain, acc


def surrogate_timing():
    """Gated surrogate on the 20-layer, 650-1150 cm^-1, 2,000-channel workload at its
    stated size: the 4-member 61 -> 1024x4 -> 2000 ensemble trained for 20,000 steps per
    member on 100,000 engine spectra, the gate calibrated on 16,384 further profiles,
    65,536 fresh + 5 % OOD (+25 K) profiles evaluated against the engine, and
    surrogate-only inference timed on the gated workload's 68,813 profiles.
    """
    from pylblrtm_b200 import surrogate_study
    rep = surrogate_study.run(n_train=100_000, n_eval=65_536, ood=0.05, steps=20_000, infer_batch=68813,
                              n_calibrate=16384, log=lambda *_: None)
    th, err = rep["throughput"], rep["errors"]
    return {"workload": "20-layer profiles, 650-1150 cm^-1 at 0.001, 2000 channels of 0.25 cm^-1, "
                        f"{rep['problem']['lines']} lines x {rep['problem']['strength_scale']:g} strength; "
                        "100000 training spectra (temperature and H2O spreads x 1.3), 20000 steps/member, gate calibrated "
                        "on 16384 profiles of the workload's distribution",
            "blended_ceiling": "1 / (OOD share + flagged share): about 20x with 5 % OOD",
            "gate": rep["gate"], "calibration": rep.get("calibration"),
            "max_channel_err_accepted": err["accepted"],
            "engine_spectra_per_s": th["engine_spectra_per_s"],
            "surrogate_only_spectra_per_s": th["infer_batch"]["spectra_per_s"],
            "surrogate_only_tflops": th["infer_batch"]["tflops"],
            "surrogate_only_speedup": th["infer_batch"]["spectra_per_s"] / th["engine_spectra_per_s"],
            "blended_spectra_per_s": th["blended_spectra_per_s"], "blended_speedup": th["speedup_blended"],
            "flagged_in": rep["gate"]["flagged_in"], "flagged_ood": rep["gate"]["flagged_ood"],
            "max_channel_err_in": err["surrogate_in"], "max_channel_err_gated": err["gated_all"],
            "train_steps_per_s": rep["training"]["steps_per_s"]}


def fp32_peak(torch):
    """Measured float32 FMA throughput (TFLOP/s) of this GPU with lbl_probe_fma_f32."""
    from pylblrtm_b200 import _lib
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    blocks, iters = sms * 8 * 4, 20000
    out = torch.zeros(1, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    best = None
    for _ in range(4):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        _lib.call("lbl_probe_fma_f32", out.data_ptr(), iters, blocks, s)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        best = ms if best is None else min(best, ms)
    return blocks * 256 * 8 * iters * 2 / (best * 1e-3) / 1e12


def _e2e_leg(torch, barrier, world, steps, warmup, call, h2d, d2h, api):
    """Times ``call()`` through the public API (copies and the result read-back inside),
    max over ranks; returns the e2e record without its value."""
    for _ in range(warmup):        # like the timed loop: each result lives until the next call returns
        call()
    barrier()
    t0 = time.perf_counter()
    for _ in range(steps):
        call()
    barrier()
    dt = time.perf_counter() - t0
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([dt], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dt = float(t.item())
    return dt, {"unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h), "api": api}


def main():
    a = parse()
    if a.impl == "reference":
        run_reference(a)
        return
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    mode = a.shard if a.shard != "auto" else ("wavenumber" if world > 1 else "replicas")
    if mode == "wavenumber" and a.precision != "fp32":
        raise SystemExit("--shard wavenumber needs --precision fp32")

    import pylblrtm_b200 as lbl
    from pylblrtm_b200 import engine, shard

    sd, prof = workload(rank if mode == "replicas" else 0)
    grid = engine.make_grid(a.nu_min, a.nu_max, 0.001, 2.0)
    n_tiles = -(-grid.n_nu // grid.tile_samples)
    tiles = None
    if mode == "wavenumber":
        span = shard.tile_span(n_tiles, world, rank)
        tiles = (span.start, span.stop - span.start)
        job = shard.shard_job(sd, prof, grid, 25.0, *tiles)
        counts = [max(0, min(grid.n_nu, sp.stop * grid.tile_samples) - sp.start * grid.tile_samples)
                  for sp in (shard.tile_span(n_tiles, world, r) for r in range(world))]
        piece_max = max(counts)
        gathered = torch.empty((world, piece_max), dtype=torch.float64, device="cuda")
        piece = torch.zeros(piece_max, dtype=torch.float64, device="cuda")
    else:
        job = engine.Job(sd, engine.layer_input_from_profile(prof), grid, 25.0)

    # Steps are queued back to back: each call returns once its stages are queued and its
    # error word is checked after the timed region (Job.run(defer_errors=True)), so the
    # next step's small stages queue behind this one's summation instead of waiting for it.
    def step(timer=None, count_evals=False):
        r = job.run(a.precision, mu=[0.8], want_od=False, want_trans=True, timer=timer, count_evals=count_evals,
                    tiles=tiles, defer_errors=not count_evals)
        if mode == "wavenumber" and world > 1:       # the exchange: every rank gets the whole spectrum
            piece[: r.trans.shape[1]].copy_(r.trans[0])
            dist.all_gather_into_tensor(gathered, piece)
        return r

    # evaluation count of one step (the reference tile rule), from the kernel's own counter
    r0 = step(count_evals=True)
    evals_local = r0.evals
    if world > 1:
        t = torch.tensor([evals_local], device="cuda", dtype=torch.int64)
        dist.all_reduce(t)
        evals_all = int(t.item())
    else:
        evals_all = evals_local
    # one spectrum's evaluations (every rank's share in the wavenumber split)
    evals_per_spectrum = evals_all if mode == "wavenumber" else evals_local
    r0_lines_bytes = int(getattr(job, "last_prep_bytes", 0))
    work_per_step = r0.work          # Faddeeva evaluations the kernel actually performs
    launches_per_step = job.launches + (1 if mode == "wavenumber" and world > 1 else 0)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(a.warmup):
        step().check()
    timer = {}
    barrier()
    with ClockSampler(local) as clocks:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        done = [step(timer=timer) for _ in range(a.steps)]
        e1.record()
        barrier()
    for r in done:
        r.check()                                    # every step's error word, after the timing
    ms = e0.elapsed_time(e1)
    tau_ms = [b.elapsed_time(c) for b, c in timer["tau_events"]]
    if world > 1:
        t = torch.tensor([ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    # spectra per step: one shared spectrum (wavenumber split) or one per rank (replicas)
    spectra_per_step = 1 if mode == "wavenumber" else world
    total_evals = evals_per_spectrum * spectra_per_step * a.steps
    value = total_evals / (ms * 1e-3)

    # end to end through the public API, inputs as a caller passes them (pageable NumPy
    # arrays); host->device copies and the device->host transmittance read inside the timed
    # region. The pinned variant (line arrays in page-locked memory) is reported beside it.
    e2e = e2e_pinned = None
    if not a.no_e2e:
        h2d = sum(np.asarray(v).nbytes for v in sd.lines.values()) + prof.pressure_hpa.nbytes * (2 + len(prof.vmr))
        if mode == "wavenumber":
            call = lambda s_: shard.compute_transmittance_sharded(s_, prof, a.nu_min, a.nu_max, mu_view=0.8,
                                                                  deterministic=False)
            api = "pylblrtm_b200.shard.compute_transmittance_sharded"
        else:
            call = lambda s_: lbl.compute_transmittance(s_, prof, a.nu_min, a.nu_max, mu_view=0.8)
            api = "pylblrtm_b200.compute_transmittance"
        d2h = grid.n_nu * 8                     # every rank returns the whole spectrum
        dt, e2e = _e2e_leg(torch, barrier, world, a.steps, a.warmup, lambda: call(sd), h2d, d2h + 8, api)
        e2e["value"] = evals_per_spectrum * spectra_per_step * a.steps / dt
        e2e["spectra_per_s"] = spectra_per_step * a.steps / dt
        e2e["inputs"] = "pageable NumPy arrays (as a caller passes them)"
        pin = {k: torch.from_numpy(np.ascontiguousarray(v)).pin_memory().numpy() for k, v in sd.lines.items()}
        sd_pin = lbl.SpectralData(pin, sd.tips, sd.molar_masses, sd.molecule)
        dtp, e2e_pinned = _e2e_leg(torch, barrier, world, a.steps, a.warmup, lambda: call(sd_pin), h2d, d2h + 8, api)
        e2e_pinned["value"] = evals_per_spectrum * spectra_per_step * a.steps / dtp
        e2e_pinned["spectra_per_s"] = spectra_per_step * a.steps / dtp
        e2e_pinned["inputs"] = "line arrays in page-locked host memory"

    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return
    peak = fp32_peak(torch)
    det = None
    if a.precision == "fp32" and world == 1:
        dtimer = {}
        for _ in range(2):
            job.run(a.precision, mu=[0.8], want_od=False, want_trans=True, deterministic=True, tiles=tiles)
        for _ in range(3):
            job.run(a.precision, mu=[0.8], want_od=False, want_trans=True, deterministic=True, timer=dtimer,
                    tiles=tiles)
        torch.cuda.synchronize()
        dms = [b.elapsed_time(c) for b, c in dtimer["tau_events"]]
        det = {"kernel_ms": sum(dms) / len(dms),
               "note": "bit-reproducible near-zone sums (deterministic=True); the timed default adds them "
                       "with shared-memory atomics (reproducible to ~1e-9 relative)"}
    full_size = (a.nu_min, a.nu_max) == (600.0, 2500.0)
    plain = acc = None
    if world == 1 and a.precision == "fp32" and not (a.no_plain and a.no_accuracy):
        if mode == "wavenumber":       # the comparison engines run on an unrestricted job
            job_full = engine.Job(sd, engine.layer_input_from_profile(prof), grid, 25.0)
        else:
            job_full = job
        plain, acc = plain_and_accuracy(torch, job_full, sd, prof, grid, evals_per_spectrum, value)
        if not full_size:
            acc = {k: v for k, v in acc.items() if not k.startswith("co2_band")}
        del job_full
    adj = None if (a.no_adjoint or world > 1) else adjoint_timing(torch)
    sur = None if (a.no_surrogate or world > 1) else surrogate_timing()
    tau_avg = sum(tau_ms) / len(tau_ms)
    # HBM-bound stages: algorithmic bytes / CUDA-event time
    try:
        with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "MEASURED_PEAKS.json")) as f:
            hbm_peak = float(json.load(f)["hbm_gbs"])
        hbm_source = "MEASURED_PEAKS.json hbm_gbs (copy, burst), of measured"
    except (OSError, KeyError, ValueError):
        hbm_peak = 6650.0
        hbm_source = "fallback 6650 GB/s (no MEASURED_PEAKS.json), of fallback"
    n_rows_, n_kept_, n_grp_, rec_ = timer["prep_shape"]
    prep_ms = sum(b.elapsed_time(c) for b, c in timer["prep_events"]) / len(timer["prep_events"])
    sum_ms = sum(b.elapsed_time(c) for b, c in timer["sum_events"]) / len(timer["sum_events"])
    n_out = r0.trans.shape[1]
    prep_bytes = n_rows_ * n_kept_ * rec_ + n_kept_ * 64 + n_rows_ * n_grp_ * 48
    sum_bytes = n_rows_ * n_out * (4 if a.precision != "fp64" else 8) + n_out * 8
    hbm = {"peak_gbs": hbm_peak, "peak_source": hbm_source,
           "line_prep": {"ms": prep_ms, "bytes": prep_bytes, "gbs": prep_bytes / prep_ms / 1e6,
                         "frac": prep_bytes / prep_ms / 1e6 / hbm_peak,
                         "bytes_rule": "32-B record written per (layer, line) + 64-B line record read once "
                                       "+ 48-B layer-group record per (layer, group)"},
           "layer_sum_exp": {"ms": sum_ms, "bytes": sum_bytes, "gbs": sum_bytes / sum_ms / 1e6,
                             "frac": sum_bytes / sum_ms / 1e6 / hbm_peak,
                             "bytes_rule": "od read once (4 B x layers per point) + f64 T written"}}
    if a.precision == "fp32":
        nodes, l3, near = r0.work_split
        flops = nodes * FLOPS_NODE + l3 * FLOPS_L3 + near * FLOPS_NEAR + FLOPS_CHEB_PER_POINT * n_out * 60
        flops_note = (f"{nodes:.3e} node evals x {FLOPS_NODE} + {l3:.3e} level-3 evals x {FLOPS_L3} + "
                      f"{near:.3e} near points x {FLOPS_NEAR} + Chebyshev {FLOPS_CHEB_PER_POINT}/point/layer")
    else:
        flops = work_per_step * FLOPS_PER_EVAL_FAR
        flops_note = f"{work_per_step:.3e} evaluations x {FLOPS_PER_EVAL_FAR}"
    achieved = flops / (tau_avg * 1e-3) / 1e12
    cpu = None
    if world == 1 and not a.no_cpu_baseline:
        n, dt = cpu_reference_sample(1)
        model, _, _ = cpu_info()
        cpu = {"value": n / dt, "unit": UNIT, "cores": 1, "kind": "port",
               "sample": f"oracle port, {CPU_SAMPLE[0]}-{CPU_SAMPLE[1]} cm^-1 x 60 layers ({n:.3e} evals, "
                         f"{dt:.1f} s), 1 process; CPU {model}"}
    parallelism = "single" if world == 1 else (f"wavenumber{world}" if mode == "wavenumber" else f"replicas{world}")
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": ms / a.steps, "higher_is_better": True,
        "scaling": "strong" if mode == "wavenumber" else "weak", "vs_baseline": None,
        "dtype": "f64" if a.precision == "fp64" else "f32", "data": "synthetic",
        "spectra_per_s": spectra_per_step * a.steps / (ms * 1e-3),
        "evals_per_spectrum": evals_per_spectrum,
        "config": {"workload": WORKLOAD if full_size
                   else f"{WORKLOAD} restricted to grid {a.nu_min}-{a.nu_max} cm^-1", "precision": a.precision,
                   "lines": 200000, "layers": 60, "grid_points": grid.n_nu, "parallelism": parallelism,
                   "tiles_per_rank": tiles[1] if tiles else n_tiles,
                   "l2": "inputs and outputs larger than L2 (line records 384 MB, od 456 MB)"},
        "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak,
                     "traffic": TAU_ML_DRAM_BYTES if (a.precision == "fp32" and full_size and world == 1) else None,
                     "traffic_unit": "bytes per call of both kernels (ncu dram__bytes_read.sum + dram__bytes_write.sum)",
                     "algorithmic_bytes": r0_lines_bytes + job.n_prof * job.n_lay * n_out * 4,
                     "algorithmic_bytes_rule": "32-B prepared line record per (layer, line) read once + "
                                               "float32 od written once per (layer, point)",
                     "kernel": {"fp32": "tau_far_kernel + tau_ml_kernel<0> (one lbl_tau_tiles_ml_f32 call)",
                                "fp32-direct": "tau_f32_kernel",
                                "fp64": "tau_f64_kernel"}[a.precision],
                     "faddeeva_evals_per_launch": work_per_step,
                     "kernel_ms": tau_avg,
                     "peak_source": "measured live: lbl_probe_fma_f32 (MEASURED_PEAKS.json has no fp32 entry)",
                     "flops_per_launch": flops, "flops_count": flops_note},
        "gpu_launches": launches_per_step * a.steps,
        "clocks": clocks.summary(),
        "e2e": e2e,
        "e2e_pinned": e2e_pinned,
        "cpu_baseline": cpu,
        "plain_engines": plain,
        "deterministic_mode": det,
        "accuracy": acc,
        "hbm_kernels": hbm,
        "adjoint": adj,
        "surrogate": sur,
    }
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
