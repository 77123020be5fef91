#!/usr/bin/env python
"""Benchmark: NLL evaluations per second of the coupled-channel Pc K-matrix model (6 Lambda*,
12 Pc K-matrix entries) on 500k data + 5M efficiency-weighted MC events.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl mine|reference]

One step = one evaluation of the unbinned NLL over the whole sample (data -log L plus the MC
normalisation sum) for one parameter point, inputs resident in HBM.  Under torchrun each rank holds
its own full-size event shard (weak scaling) and the three per-rank sums are all-reduced over NCCL
every step.  Prints one JSON line on rank 0.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "pwa-xib2jpsilambdak_b200"))

METRIC = "NLL evals/s, 5M-event K-matrix model: batched vs plain on B200, |dNLL|<=1e-4"
WORKLOAD = {"name": "kmatrix", "n_data": 500_000, "n_mc": 5_000_000, "w_range": (0.2, 1.0)}
# --workload full_bw: the full Breit-Wigner model (14 Lambda* up to J = 7/2, 3 narrow Pc) with the
# fixed-width Gaussian resolution (2.7 MeV on a 0.5 MeV grid) on 100k data + 1M MC events
WORKLOADS = {
    "kmatrix": dict(WORKLOAD, smearing=None,
                    text="kmatrix: 6 Lambda* BW + 4-channel Pc K-matrix (4 poles, 8 non-resonant)"),
    "full_bw": dict(name="full_bw", n_data=100_000, n_mc=1_000_000, w_range=(0.2, 1.0),
                    smearing=("gauss", 0.0027, 0.0005, 17),
                    text="full_bw: 14 Lambda* BW (J <= 7/2) + 3 narrow Pc BW, Gaussian resolution 2.7 MeV on "
                         "a 0.5 MeV grid"),
}
CPU_FRAC = 10  # the bounded CPU sample: 1/CPU_FRAC of the bench sample's data and MC events
# DRAM bytes read + written per event of a segment (table-only and exact passes together), from one
# ncu captures of the 50k data + 500k MC case (DRAM read + write of the table-only and the
# exact-capable pass of the window segment); the traffic of a launch scales with its events.
DRAM_BYTES_PER_EVENT = {1: 3120.0}
BATCH_DRAM_BYTES_PER_EVENT = {1: 38200.0}
# The resource that binds the FP64 kernels: FP64 pipe utilisation of the dominant kernel (ncu,
# sm__pipe_fp64_cycles_active as % of peak, small case of the same kernel), with its summary file.
FP64_PIPE = {("plain", 1): (0.186, "profiles/k_smeared20_kmatrix_50k_500k.md"),
             ("batch", 1): (0.112, "profiles/k_batch20_kmatrix_50k_500k.md")}


def fp64_pipe(kind: str, seg: int):
    v = FP64_PIPE.get((kind, seg))
    if v is None:
        return None
    return {"frac": v[0], "metric": "sm__pipe_fp64_cycles_active, % of peak (ncu)", "source": v[1]}


def parse():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["mine", "reference"], default="mine")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--small", action="store_true", help="1/10 of the workload (for profiling captures)")
    ap.add_argument("--exact", action="store_true", help="solve the K-matrix for every lookup (no tables)")
    ap.add_argument("--plain-only", action="store_true", help="skip the batched (Minuit gradient) measurement")
    ap.add_argument("--no-proposal", action="store_true", help="skip the learned-proposal measurement")
    ap.add_argument("--no-ensemble", action="store_true", help="skip the toy-ensemble fit measurement")
    ap.add_argument("--no-batch-tune", action="store_true",
                    help="keep one wave of blocks per event class for the batched passes (no autotuning)")
    ap.add_argument("--event-order", choices=["index", "mass"], default="index",
                    help="walk each MC event class by event index or by m(J/psi p) (pwa_ctx_set_event_order)")
    ap.add_argument("--profile-case", choices=["flow_small", "ensemble_small"],
                    help="run one small case of a kernel for a profiler capture (no bench line)")
    ap.add_argument("--ens-shape", help="ensemble_small profile case: launch shape 'warps,tile_events' "
                                         "instead of the autotuned one")
    ap.add_argument("--no-full-parity", action="store_true",
                    help="skip the FP64 oracle check of the whole sample (centre and one point per batch kind)")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="kmatrix",
                    help="kmatrix (the headline workload) or full_bw (the Breit-Wigner model with the "
                         "Gaussian resolution)")
    return ap.parse_args()


# ------------------------------------------------------------------------------ helpers
def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), float(d["bf16_tflops"]), "measured"
    return 6650.0, 1590.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle-reason samples during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def required_bytes_per_event(model) -> tuple:
    """Bytes of the reference SoA the model's amplitude reads per event (planes of d-functions for
    spins the model does not use are not needed), and the full reference row (all planes)."""
    ls = sorted({r.spin2 for r in model.lstar})
    pcs = sorted({r.spin2 for r in model.pc})
    ncm = max([4 if s == 1 else 6 for s in ls], default=0)
    planes = 3 + 8 * ncm + sum(2 * (4 if s == 1 else 6) for s in ls)
    if pcs:
        planes += 96 + sum(2 * (8 if s == 1 else 12) for s in pcs)
    full = 111 + (192 if model.NZ else 0)
    return 4 * planes, 4 * full


# ------------------------------------------------------------------------------ CPU side
def cpu_sample_from_device(dsample, frac: int = CPU_FRAC, seed: int = 5):
    """The bounded CPU sample: a seeded 1/frac of the bench sample's data and of its MC events (band
    order kept, band counts recomputed), copied to host memory.  Both CPU legs (the GPU arm's
    cpu_baseline and --impl reference) time this same selection."""
    rng = np.random.default_rng(seed)
    di = np.sort(rng.choice(dsample.nda, size=dsample.nda // frac, replace=False))
    mi = np.sort(rng.choice(dsample.nmc, size=dsample.nmc // frac, replace=False))
    return dsample.to_host(di, mi)


def bench_sample(block, wl: dict, device: int, rank: int = 0, small: bool = False):
    """The benchmark sample of this rank, generated on the GPU (seeded; identical in both arms)."""
    from pwa_b200 import gpu_sample
    frac = 10 if small else 1
    return gpu_sample.generate(block, wl["n_data"] // frac, wl["n_mc"] // frac, wl["w_range"], seed=1000 + rank,
                               device=device)


def time_reference(sample, block, steps: int, warmup: int) -> float:
    """Seconds per host_store_fx of the reference's own code built for host cores (OpenMP over all
    cores) on `sample`: `warmup` untimed calls, then the mean of `steps` timed calls."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O
    ref = O.RefHost(sample, block)
    for _ in range(max(warmup, 1)):
        ref.store_fx(block)
    t = time.perf_counter()
    for _ in range(steps):
        ref.store_fx(block)
    return (time.perf_counter() - t) / steps


def reference_arm(args):
    """--impl reference: the reference's own likelihood code (FP32, OpenMP over all host cores) on the
    bounded CPU sample of the workload (1/CPU_FRAC of the bench sample's events, drawn as the GPU
    arm's cpu_baseline draws them), reported in evals/s of the full workload."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O
    from pwa_b200 import configs, model as M
    wl = WORKLOADS[args.workload]
    mdl, vals = configs.MODELS[wl["name"]]()
    block = M.build_param_block(mdl, vals)
    if wl["smearing"]:
        print(json.dumps({"impl": "reference", "unavailable": "the reference has no Gaussian resolution model "
                                                              "(full_bw workload)"}))
        return 0
    L = O.ref_lib(block.NR, block.NZ, block.NX, build_if_missing=False)
    if L is None:
        print(json.dumps({"impl": "reference", "unavailable": "host build of the reference not found in oracle/_ref"}))
        return 0
    # input preparation (outside the timed region): the bench sample from the seeded device
    # generator, then the CPU selection; the timed code is the reference's alone
    import torch
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dsample = bench_sample(block, wl, local, small=args.small)
    smp = cpu_sample_from_device(dsample)
    n_full = dsample.n
    del dsample
    torch.cuda.empty_cache()
    t0 = time.perf_counter()
    dt = time_reference(smp, block, args.steps, args.warmup)
    run_s = time.perf_counter() - t0
    scale = n_full / smp.n
    value = 1.0 / (dt * scale)
    cores = os.cpu_count()
    out = {"metric": METRIC, "value": value, "unit": "evals/s", "n_gpus": args.gpus, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
           "config": {"workload": f"{wl['text']}, {wl['n_data']} data + {wl['n_mc']} MC events",
                      "parallelism": "host cores (OpenMP)"},
           "step": f"one host_store_fx of the reference's host build over {smp.n} events (1/{CPU_FRAC} of the "
                   f"workload: {smp.nda} data + {smp.nmc} MC drawn from the bench sample); value = 1 / "
                   f"(seconds per step x {scale:.2f})",
           "sample_scale": scale, "timed_s": round(run_s, 2),
           "cpu_baseline": {"value": value, "unit": "evals/s", "cores": cores, "kind": "reference",
                            "sample": f"{smp.nda} data + {smp.nmc} MC events drawn from the bench sample "
                                      f"(seed 5); time x{scale:.2f} to the full workload"},
           "e2e": {"value": value, "unit": "evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))
    return 0


def full_size_parity(dsample, block, ctx, labels, gblocks, bres, probe) -> dict:
    """GPU plain and batched NLL against the FP64 oracle on the whole bench sample (host cores), at
    the centre and one gradient point of every batch kind."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O
    t0 = time.perf_counter()
    host = dsample.to_host()
    rows = []
    for name in probe:
        i = 0 if name == "centre" else labels.index((name, +1))
        v_or, s_or, _, _ = O.nll(host, gblocks[i])
        v_pl = ctx.eval_nll(gblocks[i]).nll
        rows.append({"point": name, "nll_oracle": v_or, "dnll_plain": v_pl - v_or,
                     "dnll_batched": (bres[i].nll - v_or) if bres is not None else None})
    del host
    worst = max(max(abs(r["dnll_plain"]), abs(r["dnll_batched"] or 0.0)) for r in rows)
    return {"sample_events": dsample.n, "points": rows, "max_abs_dnll": worst,
            "oracle_threads": os.cpu_count(), "seconds": round(time.perf_counter() - t0, 1)}


# ------------------------------------------------------------------------------ learned proposal
PROPOSAL = {"model": "full_bw", "n_train": 10_000_000, "n_toy": 10_000_000, "n_norm": 5_000_000, "batch": 65536,
            "epochs": 16, "lr": 3e-3, "chunk": 1 << 20, "premap_mix": 0.1}
# FLOPs per event of one training step: forward (64x256 + 3 x 256^2 + 256x512), backward through the
# activations (512x256 + 3 x 256^2) and the weight gradients (512x256 + 3 x 256^2 + 256x64), 2 per MAC
PROPOSAL_FLOP_PER_ROW = 2.0 * ((64 * 256 + 3 * 256 ** 2 + 256 * 512) + (512 * 256 + 3 * 256 ** 2)
                               + (512 * 256 + 3 * 256 ** 2 + 256 * 64))


def _amp2_unit(ctx, block, x, chunk):
    """|A|^2 and the flat phase-space density at unit coordinates x (torch [7, n] on the device)."""
    import torch
    from pwa_b200 import flow
    a2, fl = [], []
    for c0 in range(0, x.shape[1], chunk):
        xs = x[:, c0:c0 + chunk].contiguous()
        (pp, pp1, pp2, ns), f = flow.events_from_unit(xs)
        sw = torch.zeros(ns, dtype=torch.float32, device=x.device)
        ctx.bind_planes(pp, pp1, pp2, sw, xs.shape[1], ns)
        a2.append(torch.as_tensor(ctx.amp2(block), device=x.device))
        fl.append(f)
        del pp, pp1, pp2
    return torch.cat(a2), torch.cat(fl)


def proposal_bench(device: int, bf16_peak: float) -> dict:
    """The learned proposal (trained on the GPU, BF16 tcgen05 GEMMs) against flat hit-or-miss on the
    full Breit-Wigner model: amplitude evaluations per accepted toy event (acceptance against 1.05 x the
    largest weight, as the hit-or-miss toy maker does with its global maximum), and amplitude evaluations
    for equal statistical error of the normalisation integral (importance sampling, weights |A|^2 flat / q)."""
    import torch
    from pwa_b200 import configs, flow, lib, model as M
    P = PROPOSAL
    mdl, vals = configs.MODELS[P["model"]]()
    block = M.build_param_block(mdl, vals)
    ctx = lib.Context(device)
    t0 = time.perf_counter()
    xt = flow.flat_unit(P["n_train"], seed=501, device=device)
    a2t, _ = _amp2_unit(ctx, block, xt, P["chunk"])
    t_data = time.perf_counter() - t0
    f = flow.Flow(device, max_batch=P["batch"], seed=11)
    torch.cuda.synchronize(device)
    t0 = time.perf_counter()
    f.fit_premap(xt, a2t, mix=P["premap_mix"])
    hist = f.train(xt, a2t, epochs=P["epochs"], batch=P["batch"], lr=P["lr"])
    torch.cuda.synchronize(device)
    t_train = time.perf_counter() - t0
    steps = len(hist)
    del xt, a2t
    # toys: candidates from q vs flat candidates
    xq, lq = f.sample(P["n_toy"], seed=502)
    a2q, flq = _amp2_unit(ctx, block, xq, P["chunk"])
    wq = a2q * flq / torch.exp(lq.double())
    xf = flow.flat_unit(P["n_toy"], seed=503, device=device)
    a2f, _ = _amp2_unit(ctx, block, xf, P["chunk"])
    g = torch.Generator(device=f"cuda:{device}").manual_seed(504)

    def accepted(w):
        mx = 1.05 * float(w.max())
        return int((torch.rand(w.numel(), generator=g, device=w.device, dtype=torch.float64) * mx < w).sum())

    acc_q, acc_f = accepted(wq), accepted(a2f)
    evals_q, evals_f = P["n_toy"] / max(acc_q, 1), P["n_toy"] / max(acc_f, 1)
    # the same in expectation: 1.05 x max weight / mean weight
    exp_q = 1.05 * float(wq.max()) / float(wq.mean())
    exp_f = 1.05 * float(a2f.max()) / float(a2f.mean())
    q999 = float(torch.quantile(wq[:1 << 24].float(), 0.999)) / float(wq.mean())
    # weighted toys (every candidate kept with weight |A|^2 flat / q, the exact amplitude deciding): the
    # amplitude evaluations per effective event, n / ESS = mean(w^2) / mean(w)^2, against the
    # evaluations per accepted event of flat hit-or-miss at the same statistical power
    per_eff_q = float((wq ** 2).mean()) / float(wq.mean()) ** 2
    # normalisation integral on the first n_norm events of each
    nn = P["n_norm"]
    wn, fn = wq[:nn], a2f[:nn]
    i_q, i_f = float(wn.mean()), float(fn.mean())
    rv_q, rv_f = float(wn.var()) / i_q ** 2, float(fn.var()) / i_f ** 2
    ctx.close()
    f.close()
    gain = evals_f / evals_q
    tflops = PROPOSAL_FLOP_PER_ROW * P["batch"] * steps / t_train / 1e12
    return {
        "model": "full_bw (14 Lambda* BW up to J = 7/2, 3 narrow Pc BW): the batched-gradient config's model",
        "network": "autoregressive 4 x 256 SiLU MLP, 64 bins per coordinate, BF16 tcgen05 GEMMs, FP32 accumulation",
        "train_events": P["n_train"], "epochs": P["epochs"], "steps": steps, "batch": P["batch"],
        "train_s": round(t_train, 3), "data_s": round(t_data, 3), "loss_first": hist[0], "loss_last": hist[-1],
        "train_tflops": round(tflops, 2),
        "train_frac_of_bf16_peak": round(tflops / bf16_peak, 4),
        "premap": f"per-coordinate piecewise-linear CDF on 1024 cells, uniform floor {P['premap_mix']}",
        "toy_candidates": P["n_toy"], "accepted_flat": acc_f, "accepted_learned": acc_q,
        "evals_per_accepted_expected_flat": round(exp_f, 3), "evals_per_accepted_expected_learned": round(exp_q, 3),
        "learned_weight_q999_over_mean": round(q999, 3),
        "weighted_toys_evals_per_effective_event": round(per_eff_q, 3),
        "weighted_toys_gain_vs_hit_or_miss": round(exp_f / per_eff_q, 3),
        "evals_per_accepted_flat": round(evals_f, 3), "evals_per_accepted_learned": round(evals_q, 3),
        "evals_per_accepted_gain": round(gain, 3), "target_gain": 10.0,
        "target_met_hit_or_miss": bool(gain >= 10.0),
        "target_met_weighted_equal_error": bool(exp_f / per_eff_q >= 10.0),
        "norm_events": nn, "norm_integral_flat": i_f, "norm_integral_learned": i_q,
        "norm_rel_diff": (i_q - i_f) / i_f,
        "norm_rel_diff_in_sigma": (i_q - i_f) / np.sqrt(float(wn.var()) / nn + float(fn.var()) / nn),
        "norm_evals_gain_equal_error": round(rv_f / rv_q, 3),
    }


# ------------------------------------------------------------------------------ toy ensemble
ENSEMBLE = {"model": "full_bw", "n_toys": 256, "size_lo": 5e3, "size_hi": 2e5, "size_seed": 42, "n_mc": 1_000_000,
            "w_range": (0.2, 1.0), "smearing": ("gauss", 0.0027, 0.0005, 17), "gen_seed": 11, "parity_toys": (0, 1, 2)}
# bytes the ensemble kernel reads per data event: the pp / pp1 / pp2 plane slots (303 floats), the
# data weight, and the cached lineshape factors (2 NR + 2 NZ + NZ (NZ + 1) doubles; NR = 14, NZ = 3)
ENSEMBLE_BYTES_PER_EVENT = 303 * 4 + 4 + (2 * 14 + 2 * 3 + 3 * 4) * 8


def ensemble_bench(device: int, hbm: float) -> dict:
    """The batched-gradient config's toy study: 256 seeded toys of the full Breit-Wigner model with sizes
    log-uniform in 5k-200k events and one 1M-event MC sample, all fitted together (every coupling but
    the reference one free), against the toy-by-toy fit through the batched numerical gradient."""
    import torch
    from pwa_b200 import configs, ensemble, fit as F, lib, model as M, toys
    P = ENSEMBLE
    mdl, vals = configs.MODELS[P["model"]]()
    block = M.build_param_block(mdl, vals)
    sizes = toys.toy_sizes(P["n_toys"], P["size_lo"], P["size_hi"], P["size_seed"])
    t0 = time.perf_counter()
    ens = toys.make_ensemble_gpu(block, sizes, P["n_mc"], P["w_range"], seed=P["gen_seed"], device=device)
    t_gen = time.perf_counter() - t0
    ctx = lib.Context(device)
    ctx.bind_device(ens.sample)
    ctx.set_smearing(*P["smearing"])
    names = ensemble.coupling_names(mdl)
    t0 = time.perf_counter()
    E = ensemble.Ensemble(ctx, ens, mdl, vals, names)
    t_setup = time.perf_counter() - t0
    fac_ms, gram_ms = E.setup_ms()
    tune = ensemble.autotune(E)
    S = np.repeat(E.s0[None, :], E.n_toys, axis=0)
    ms = []
    for _ in range(5):
        E.eval_slots(S)
        ms.append(E.last_ms())
    step_ms = float(np.median(ms[1:]))
    n_ev = int(sizes.sum())
    gbs = ENSEMBLE_BYTES_PER_EVENT * n_ev / (step_ms / 1e3) / 1e9
    torch.cuda.synchronize(device)
    t0 = time.perf_counter()
    fit = E.fit()
    t_fit = time.perf_counter() - t0
    # parity of the fitted points: the exact float blocks through the single-point evaluator
    par = []
    for t in P["parity_toys"]:
        out, _, _ = E.eval_slots(np.repeat(E.exact_slots(fit.x[t])[None, :], E.n_toys, axis=0))
        toys.select(ctx, ens, t)
        r = ctx.eval_nll(E.builder.block(dict(zip(names, fit.x[t]))))
        par.append(abs(out[t, 0] - r.nll))
    # the toy-by-toy path: one batched numerical gradient (2N+1 points over the toy's data and the MC)
    grad_s = []
    for t in (int(np.argmin(sizes)), int(np.argmax(sizes))):
        toys.select(ctx, ens, t)
        f = F.gpu_fcn(ctx, mdl, vals, names)
        X = F._grad_points(fit.x[t], np.full(len(names), 1e-3))
        f(X)
        t1 = time.perf_counter()
        f(X)
        grad_s.append(time.perf_counter() - t1)
    toys.select_all(ctx, ens)
    # Migrad-like toy-by-toy fits need at least one gradient per iteration: project with the ensemble's
    # own iteration counts (a lower bound on the sequential cost)
    seq_s = float(np.sum(fit.iterations + 1) * np.mean(grad_s))
    E.close()
    ctx.close()
    del ens
    return {
        "model": "full_bw (14 Lambda* BW, 3 narrow Pc BW), Gaussian resolution 2.7 MeV on a 0.5 MeV grid",
        "toys": P["n_toys"], "toy_sizes": "floor(exp U(ln 5e3, ln 2e5)), seed 42", "data_events": n_ev,
        "mc_events": P["n_mc"], "free_parameters": len(names), "slots": E.n_slot,
        "generate_s": round(t_gen, 3), "setup_s": round(t_setup, 3), "factor_cache_ms": round(fac_ms, 3),
        "gram_ms": round(gram_ms, 3), "launch_shape": {k: tune[k] for k in ("warps", "tile_events", "cached")},
        "step_ms": round(step_ms, 3), "step_gbs": round(gbs, 1), "step_frac_of_hbm": round(gbs / hbm, 4),
        "step_bytes_per_event": ENSEMBLE_BYTES_PER_EVENT,
        "fit_wall_s": round(t_fit, 3), "fit_calls": fit.calls, "fit_device_s": round(fit.device_ms / 1e3, 3),
        "converged": int(fit.converged.sum()), "iterations_mean": float(fit.iterations.mean()),
        "iterations_max": int(fit.iterations.max()),
        "parity_fitted_points_max_dnll": float(max(par)),
        "sequential_gradient_s": [round(x, 4) for x in grad_s],
        "sequential_projection_s": round(seq_s, 1),
        "speedup_vs_sequential_projection": round(seq_s / t_fit, 1),
        "note": "sequential projection = sum over toys of (iterations + 1) x the measured time of one "
                "batched numerical gradient (2N+1 points over the toy's window and the MC), a lower bound",
    }


# ------------------------------------------------------------------------------ profiler cases
def profile_case(name: str, device: int = 0, ens_shape: str | None = None) -> int:
    """Small runs of one kernel family for ncu captures (inputs above L2, a few GB on the device at
    most): flow_small = 12 training steps of the proposal network on 16,384-event batches (k_gemm);
    ensemble_small = an 8-toy ensemble of the full BW model (8 x 40k data events, 100k MC) and three
    ensemble steps (k_ens_data), at the launch shape `ens_shape` ("warps,tile_events") or the autotuned
    one."""
    import torch
    from pwa_b200 import configs, ensemble, flow, lib, model as M, toys
    if name == "flow_small":
        f = flow.Flow(device, max_batch=16384, seed=3)
        x = flow.flat_unit(12 * 16384, seed=5, device=device)
        w = torch.rand(x.shape[1], dtype=torch.float64, device=x.device, generator=torch.Generator(x.device).manual_seed(6))
        f.fit_premap(x, w)
        f.train(x, w, epochs=1, batch=16384, lr=1e-3)
        f.close()
    else:
        mdl, vals = configs.MODELS["full_bw"]()
        block = M.build_param_block(mdl, vals)
        ens = toys.make_ensemble_gpu(block, np.full(8, 40_000), 100_000, (0.2, 1.0), seed=7, device=device)
        ctx = lib.Context(device)
        ctx.bind_device(ens.sample)
        ctx.set_smearing("gauss", 0.0027, 0.0005, 17)
        E = ensemble.Ensemble(ctx, ens, mdl, vals, ensemble.coupling_names(mdl))
        if ens_shape:
            E.set_launch(*(int(v) for v in ens_shape.split(",")))
        else:
            ensemble.autotune(E)  # the launch shape the bench uses for this device and ensemble shape
        S = np.repeat(E.s0[None, :], E.n_toys, axis=0)
        for _ in range(3):
            E.eval_slots(S)
        print(json.dumps({"case": name, "step_ms": E.last_ms(), "events": int(ens.offsets[-1])}))
        E.close()
        ctx.close()
    torch.cuda.synchronize(device)
    return 0


# ------------------------------------------------------------------------------ GPU arm
def main():
    args = parse()
    if args.profile_case:
        return profile_case(args.profile_case, ens_shape=args.ens_shape)
    if args.impl == "reference":
        return reference_arm(args)
    import torch
    import torch.distributed as dist
    from pwa_b200 import configs, gpu_sample, lib, model as M

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)

    wl = WORKLOADS[args.workload]
    mdl, vals = configs.MODELS[wl["name"]]()
    block = M.build_param_block(mdl, vals)
    frac = 10 if args.small else 1
    nd, nm = wl["n_data"] // frac, wl["n_mc"] // frac
    t_gen = time.perf_counter()
    sample = bench_sample(block, wl, local, rank, args.small)
    t_gen = time.perf_counter() - t_gen
    ctx = lib.Context(local)
    ctx.bind_device(sample)
    ctx.set_timing(True)
    if wl["smearing"]:
        ctx.set_smearing(*wl["smearing"])
    ctx.set_lineshape_tables(not args.exact)
    ctx.set_event_order(args.event_order == "mass")
    stream = torch.cuda.ExternalStream(ctx.stream(), device=dev)
    sums = torch.zeros(3, dtype=torch.float64, device=dev)

    def step():
        r = ctx.eval_nll(block)
        if world > 1:
            sums.copy_(torch.tensor([r.data_term, r.sumint, r.sum_noint], dtype=torch.float64))
            dist.all_reduce(sums)
        return r

    for _ in range(max(args.warmup, 3)):
        r = step()
    # timed region: device time with CUDA events on the launching stream
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    clk = ClockSampler(local)
    clk.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    seg_time = {}
    seg_deferred = {}
    kernel_ms = 0.0
    launches = 0
    for _ in range(args.steps):
        r = step()
        kernel_ms += ctx.last_kernel_ms()
        launches += ctx.last_launches()
        for (kind, n, ms), n_def in zip(ctx.segments(), ctx.segments_deferred()):
            t, _ = seg_time.get(kind, (0.0, n))
            seg_time[kind] = (t + ms, n)
            seg_deferred[kind] = n_def
    e1.record(stream)
    torch.cuda.synchronize(dev)
    dev_ms = e0.elapsed_time(e1)
    # end to end through the public API (host parameter block in, result out), wall clock
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    e2e_ms = (time.perf_counter() - t0) * 1e3

    # batched: one step = one batch of the 2N+1 points of Minuit's numerical gradient
    bat = None
    if not args.plain_only:
        from pwa_b200 import gradient
        labels, gblocks = gradient.gradient_blocks(mdl, vals)
        npts = len(gblocks)
        bsums = torch.zeros((npts, 3), dtype=torch.float64, device=dev)

        def bstep():
            res, ns = ctx.eval_nll_batch(gblocks)
            if world > 1:
                bsums.copy_(torch.tensor([[x.data_term, x.sumint, x.sum_noint] for x in res], dtype=torch.float64))
                dist.all_reduce(bsums)
            return res, ns

        tune = None
        if not args.no_batch_tune:
            from pwa_b200 import autotune
            tune = autotune.tune_batch(ctx, gblocks)  # waves per event class, timed or from the cache
        for _ in range(max(args.warmup, 3)):
            bres, nstruct = bstep()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)
        b0, b1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        b0.record(stream)
        blaunch = 0
        bseg = {}
        for _ in range(args.steps):
            bres, nstruct = bstep()
            blaunch += ctx.last_launches()
            for (kind, n, _), ms in zip(ctx.segments(), ctx.batch_segment_ms()):
                t, _ = bseg.get(kind, (0.0, n))
                bseg[kind] = (t + ms, n)
        b1.record(stream)
        torch.cuda.synchronize(dev)
        bdev_ms = b0.elapsed_time(b1)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            bstep()
        be2e_ms = (time.perf_counter() - t0) * 1e3
        # |dNLL| of the batched points against one-by-one evaluation, one point of every kind
        probe = ["a_p1p1_1520", "m0_1670", "width_1810", "scRe", "a_L0_Pc4312", "p_Bp_ZM1SC1", "a_L1_ZM3SC1",
                 "g1_Pc4312", "m0_Pc4440", "g3_Pc4500", "fsc_ZM3SC2"]
        idx = [0] + [labels.index((n, +1)) for n in probe if (n, +1) in labels]
        dmax = max(abs(bres[i].nll - ctx.eval_nll(gblocks[i]).nll) for i in idx)
        bat = dict(npts=npts, nstruct=nstruct, dev_ms=bdev_ms, e2e_ms=be2e_ms, launches=blaunch, dnll=dmax,
                   nprobe=len(idx), seg=bseg, labels=labels, blocks=gblocks, res=bres, tune=tune)
    clocks = clk.stop()
    if world > 1:
        t = torch.tensor([dev_ms, e2e_ms, bat["dev_ms"] if bat else 0.0, bat["e2e_ms"] if bat else 0.0],
                         dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dev_ms, e2e_ms, bd, be = t.tolist()
        if bat:
            bat["dev_ms"], bat["e2e_ms"] = bd, be
        dist.barrier()
    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return 0

    value = world * args.steps / (dev_ms / 1e3)
    e2e = world * args.steps / (e2e_ms / 1e3)
    hbm, bf16, peak_kind = measured_peaks()
    req_b, full_b = required_bytes_per_event(mdl)
    names = {0: "k_unsmeared", 1: "k_smeared<20>", 2: "k_smeared<30>", 3: "k_smeared<150>", 4: "k_smeared<grid>",
             -1: "k_build_tables"}
    total_seg = sum(t for t, _ in seg_time.values())
    shares = {names[k]: round(t / total_seg, 4) for k, (t, n) in seg_time.items()}
    dom = max(seg_time, key=lambda k: seg_time[k][0])
    dom_ms = seg_time[dom][0] / args.steps
    dom_bytes = seg_time[dom][1] * req_b + (sample.nda * 4 if dom in (2, 3) else 0)
    achieved = dom_bytes / (dom_ms / 1e3) / 1e9
    metric = METRIC if args.workload == "kmatrix" else ("NLL evals/s, 1M-event full Breit-Wigner model with Gaussian "
                                                         "resolution: batched vs plain on B200")
    out = {"metric": metric, "value": value, "unit": "evals/s", "n_gpus": world, "steps": args.steps,
           "warmup": max(args.warmup, 3), "ms_per_step": dev_ms / args.steps, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": {"workload": f"{wl['text']}, {nd} data + {nm} MC events per GPU",
                      "global_events": world * (nd + nm),
                      "parallelism": f"dp{world} event shards, NCCL all-reduce of 3 sums per step",
                      "l2": "inputs larger than L2 (events x 828 B >> 126 MB)", "precision": "plain FP64 path",
                      "lineshapes": "exact K-matrix solves" if args.exact else "FP64 K-matrix tables, exact near "
                                                                               "thresholds",
                      "event_order": args.event_order},
           "gpu_launches": launches,
           "kernel_shares": shares,
           "segments": {names[k]: {"events": int(n), "deferred_to_exact": int(seg_deferred.get(k, 0)),
                                   "ms_per_step": round(t / args.steps, 4),
                                   "ns_per_event": round(t / args.steps / max(n, 1) * 1e6, 3)}
                        for k, (t, n) in seg_time.items()},
           "roofline": {"bound": "hbm", "kernel": names[dom], "achieved": achieved, "peak": hbm, "unit": "GB/s",
                        "frac": achieved / hbm,
                        "traffic": (DRAM_BYTES_PER_EVENT[dom] * seg_time[dom][1]
                                    if dom in DRAM_BYTES_PER_EVENT else None),
                        "traffic_unit": "bytes per step of this segment (ncu, scaled by events)",
                        "fp64_pipe": fp64_pipe("plain", dom),
                        "note": f"algorithmic bytes = {req_b} B per event (planes the model reads) of the "
                                f"{full_b} B reference row; peak {peak_kind}"},
           "e2e": {"value": e2e, "unit": "evals/s", "h2d_bytes_per_step": int(lib.load().pwa_point_table_bytes()),
                   "d2h_bytes_per_step": 48},
           "clocks": clocks, "setup_s": round(t_gen, 2)}
    if wl["smearing"] and not args.no_cpu_baseline:
        out["cpu_baseline"] = {"value": None, "unit": "evals/s", "cores": os.cpu_count(), "kind": "reference",
                               "sample": "not timed: the reference has no Gaussian resolution model"}
    elif world == 1 and not args.no_cpu_baseline:
        try:
            smp = cpu_sample_from_device(sample)
            t_ref = time_reference(smp, block, args.steps, args.warmup)
            scale = sample.n / smp.n
            out["cpu_baseline"] = {"value": 1.0 / (t_ref * scale), "unit": "evals/s", "cores": os.cpu_count(),
                                   "kind": "reference", "seconds_per_step": t_ref, "steps": args.steps,
                                   "sample": f"{smp.nda} data + {smp.nmc} MC events (1/{CPU_FRAC}) drawn from the "
                                             f"bench sample (seed 5), {args.steps} timed calls after "
                                             f"{max(args.warmup, 1)} warm-up; time x{scale:.2f} to the full "
                                             f"workload"}
            # parity on the same sample: this GPU path and the reference FP32 code vs the FP64 oracle
            sys.path.insert(0, str(ROOT / "oracle"))
            import oracle as O
            v_or, _, _, _ = O.nll(smp, block)
            c2 = lib.Context(local)
            c2.upload(smp)
            v_gpu = c2.eval_nll(block).nll
            c2.close()
            v_ref, _ = O.RefHost(smp, block).store_fx(block)
            out["parity"] = {"sample_events": smp.n, "dnll_gpu_vs_oracle": v_gpu - v_or,
                             "dnll_reference_fp32_vs_oracle": v_ref - v_or}
            del smp
        except Exception as ex:  # the baseline is reported, never required for the GPU number
            out["cpu_baseline"] = {"value": None, "unit": "evals/s", "cores": os.cpu_count(), "kind": "reference",
                                   "sample": f"failed: {ex}"}
    if world == 1 and bat and not args.no_full_parity and not wl["smearing"]:
        # every batch kind: Lambda* coupling and mass, Pc coupling, K-matrix pole coupling and mass,
        # scattering term
        probe = ["centre", "a_p1p1_1520", "m0_1670", "a_L0_Pc4312", "g1_Pc4312", "m0_Pc4440", "fsc_ZM3SC2"]
        probe = [p for p in probe if p == "centre" or (p, +1) in bat["labels"]]
        try:
            out["parity_full"] = full_size_parity(sample, block, ctx, bat["labels"], bat["blocks"], bat["res"],
                                                  probe)
        except Exception as ex:
            out["parity_full"] = {"failed": str(ex)}
    if world == 1 and not args.no_proposal:
        try:
            out["proposal"] = proposal_bench(local, bf16)
        except Exception as ex:
            out["proposal"] = {"failed": str(ex)}
    if world == 1 and not args.no_ensemble:
        try:
            out["ensemble"] = ensemble_bench(local, hbm)
        except Exception as ex:
            out["ensemble"] = {"failed": str(ex)}
    if bat:
        out = batched_line(out, bat, args, world, sample, req_b, hbm, peak_kind)
    print(json.dumps(out))
    if world > 1:
        dist.destroy_process_group()
    return 0


def batched_line(plain: dict, bat: dict, args, world: int, sample, req_b: int, hbm: float, peak_kind: str) -> dict:
    """The bench line with the batched gradient evaluation as the headline and the plain single-point
    measurement kept under "plain"."""
    from pwa_b200 import lib
    npts = bat["npts"]
    value = world * npts * args.steps / (bat["dev_ms"] / 1e3)
    e2e = world * npts * args.steps / (bat["e2e_ms"] / 1e3)
    ms_step = bat["dev_ms"] / args.steps
    # dominant kernel: the batched passes of the costliest event class (CUDA events around its launches)
    bnames = {0: "k_batch_un", 1: "k_batch<20>", 2: "k_batch<30>", 3: "k_batch<150>", 4: "k_batch<grid>"}
    seg = bat["seg"]
    dom = max(seg, key=lambda k: seg[k][0])
    dom_ms = seg[dom][0] / args.steps
    dom_ev = seg[dom][1]
    achieved = dom_ev * (req_b + 4) / (dom_ms / 1e3) / 1e9
    tot = sum(t for t, _ in seg.values())
    keep = ("value", "ms_per_step", "gpu_launches", "kernel_shares", "segments", "roofline", "e2e")
    out = {k: v for k, v in plain.items() if k not in keep}
    out["plain"] = {k: plain[k] for k in keep if k in plain}
    out["plain"]["note"] = "one step = one single-point evaluation (pwa_ctx_eval_nll)"
    pt_bytes = int(lib.load().pwa_point_table_bytes())
    out.update({
        "value": value, "ms_per_step": ms_step, "gpu_launches": bat["launches"],
        "batched_vs_plain": value / plain["value"],
        "batch": {"points_per_step": npts, "points_from_centre": bat["nstruct"],
                  "points_one_by_one": npts - bat["nstruct"],
                  "max_abs_dnll_vs_single_point": bat["dnll"], "probed_points": bat["nprobe"],
                  "step": "the 2N+1 parameter points of Minuit's numerical gradient (centre, +-h per parameter) "
                          "in one pwa_ctx_eval_nll_batch call; every point's NLL is computed in FP64",
                  "waves_per_class": ({bnames[int(k)]: w for k, w in bat["tune"]["waves"].items()}
                                      if bat.get("tune") else "1 (not tuned)"),
                  "tune_ms": ({bnames[int(k)]: v for k, v in bat["tune"]["ms"].items()}
                              if bat.get("tune") and "ms" in bat["tune"] else None)},
        "kernel_shares": {bnames[k]: round(t / tot, 4) for k, (t, n) in seg.items()},
        "segments": {bnames[k]: {"events": int(n), "ms_per_step": round(t / args.steps, 3)}
                     for k, (t, n) in seg.items()},
        "roofline": {"bound": "hbm", "kernel": bnames[dom], "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm,
                     "traffic": (BATCH_DRAM_BYTES_PER_EVENT[dom] * dom_ev if dom in BATCH_DRAM_BYTES_PER_EVENT
                                 else None),
                     "traffic_unit": "bytes per step of this segment (ncu, scaled by events)",
                     "fp64_pipe": fp64_pipe("batch", dom),
                     "note": f"algorithmic bytes = {req_b} B of planes + 4 B index per event, read once per "
                             f"batch of {npts} points; the kernel is FP64-issue bound, peak {peak_kind}"},
        "e2e": {"value": e2e, "unit": "evals/s",
                "h2d_bytes_per_step": (npts + 1) * pt_bytes + npts * (8 * 24 * 16 + 96),
                "d2h_bytes_per_step": npts * 48},
    })
    out["config"] = dict(out["config"], precision="FP64; batched points formed from the centre's per-event terms",
                         step="one Minuit gradient batch (2N+1 points)")
    return out


if __name__ == "__main__":
    sys.exit(main())
