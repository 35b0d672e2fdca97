#!/usr/bin/env python
"""Benchmark of the B200 Milne-Eddington inversion (one JSON line on stdout).

Metric: converged pixels/s on one B200 -- pixels inverted per second, counted
as converged when their chi^2 is <= 1.05 x the chi^2 the reference's FP64 C
code reaches on the same profile -- with the learned initialiser, beside the
plain LM with the reference's random restarts on the same map and GPU.  The
converged share is measured on a seeded sample of the map against the
reference core (oracle/_ref, the reference's own C sources compiled here; the
oracle restatement where it was not built).

Workload (default): the 1024x1024 Fe I 15648.5 A map (nl = 60, seeded draws of
B, theta, phi, v, Doppler width, damping, eta0, beta; S = 1; noise 1e-3),
num_run = 5, chisq_criteria = 1.5, FP32 synthesis with FP64 SVD solve and
chi^2 test, with Bounds_Dopp = 100, 400 mA and Bounds_Damp = 0.05, 1.0: the
default Doppler bounds (10-80 mA) cannot reach the drawn widths (150-350 mA),
so with them no start can fit and chisq_criteria is met by a sixth of the
pixels at best (`--bounds literal` runs that variant).

The initialiser is trained once per line and grid before the timed region
(4M profiles synthesised on the GPU from seeded draws of the same
distributions, other seeds than the map's, 20 epochs of Adam, lr 1e-3, batch
4096); its training time is reported, its inference is inside every step.

A step is one inversion of the whole map.  The map (2 GB of FP64 profiles,
larger than L2) is resident in HBM when the timed region starts; `e2e` times
the same step through the host entry point me_invert_batch with the profiles
in pinned host memory (host->device copy, inference, inversion, device->host
copy of the results).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
    torchrun --nproc-per-node N bench.py --gpus N ...   (one rank per GPU)

With N GPUs every rank inverts its own map (pixels are independent; no
collective on the data path): scaling is weak, value = all ranks' pixels /
the slowest rank's time.
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "milne-eddington_b200")
sys.path.insert(0, PKG)

import me_maps  # noqa: E402
import me_ranks  # noqa: E402

METRIC = "converged pixels/s on 1 B200 at chi2<=1.05x FP64 ref: learned-init vs plain LM"
UNIT = "pixels/s"


# ---------------------------------------------------------------------------
# CPU side: the reference's own C core (or the oracle port) on host cores.
# ---------------------------------------------------------------------------
_W = {}


def _cpu_worker_init(kind, workload, npix_max, seed, widen):
    sys.path[:0] = [os.path.join(ROOT, "tests"), PKG]
    import oracle_bind as ob
    import me_b200
    lam = me_maps.wavelengths(workload)
    _W["kind"] = kind
    if kind == "reference":
        _W["eng"] = ob.Reference(me_maps.reference_control_text(workload, widen_bounds=widen),
                                 lam, npix_max, seed=seed)
    else:
        cfg = me_b200.parse_config_text(me_maps.control_text(workload, precision="FP64",
                                                             widen_bounds=widen))
        _W["eng"] = ob.Oracle(cfg, lam)


def _cpu_worker_invert(prof):
    eng = _W["eng"]
    if _W["kind"] == "reference":
        return eng.invert(prof)
    import oracle_bind as ob
    return eng.invert(prof, rng_mode=ob.MEO_RNG_NR, nr_seed=1)


def cpu_kind(workload="fe15648_1024x1024"):
    """The reference's own core where it was built here and the workload is
    within its reach; the oracle port (the same algorithm restated, with the
    instrument-filter extension) otherwise."""
    if me_maps.WORKLOADS[workload]["ctl"].get("filter", "0") != "0":
        return "port"
    return "reference" if os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libmeref.so")) \
        else "port"


def cpu_invert(prof, workload, procs, widen):
    """Inverts prof [n][4][nl] with `procs` processes of the reference core;
    returns (results, seconds, kind)."""
    kind = cpu_kind(workload)
    n = prof.shape[0]
    procs = max(1, min(procs, n))
    chunks = np.array_split(np.arange(n), procs)
    ctx = mp.get_context("spawn")
    with ctx.Pool(procs, initializer=_cpu_worker_init,
                  initargs=(kind, workload, max(len(c) for c in chunks), 4242, widen)) as pool:
        pool.map(_cpu_worker_invert, [prof[c[:1]] for c in chunks])  # warm every worker
        t0 = time.perf_counter()
        parts = pool.map(_cpu_worker_invert, [prof[c] for c in chunks])
        dt = time.perf_counter() - t0
    return np.concatenate(parts), dt, kind


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def cpu_sample_profiles(workload, npix, seed):
    """Seeded profiles synthesised on the CPU by the oracle (FP64)."""
    sys.path[:0] = [os.path.join(ROOT, "tests")]
    import me_b200
    import oracle_bind as ob
    lam = me_maps.wavelengths(workload)
    cfg = me_b200.parse_config_text(me_maps.control_text(workload, precision="FP64"))
    o = ob.Oracle(cfg, lam)
    par = me_maps.draw_parameters(workload, npix, seed)
    return me_maps.add_noise(o.synth_many(par), me_maps.WORKLOADS[workload]["noise"], seed)


# ---------------------------------------------------------------------------
# GPU clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.path = tempfile.mktemp(suffix=".csv")

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.dev}",
                                          f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            self.proc.wait(timeout=10)
            self.f.close()

    def summary(self):
        try:
            rows = [r.split(",") for r in open(self.path).read().strip().splitlines() if r]
        except Exception:
            rows = []
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = max(mx, float(r[2]))
                for k, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(k)
            except (ValueError, IndexError):
                pass
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="fe15648_1024x1024", choices=list(me_maps.WORKLOADS))
    ap.add_argument("--bounds", default="auto", choices=["auto", "widened", "literal"],
                    help="auto: widened Doppler/damping bounds for the Fe I 15648 A maps, "
                         "the workload's own otherwise")
    ap.add_argument("--npix", type=int, default=0, help="override the map size (testing)")
    ap.add_argument("--precision", default="FP32", choices=["FP32", "FP64"])
    ap.add_argument("--sample", type=int, default=4096,
                    help="pixels of the CPU sample (reference timing + converged share)")
    ap.add_argument("--train-samples", type=int, default=4 << 20)
    ap.add_argument("--train-epochs", type=int, default=20)
    ap.add_argument("--plain-steps", type=int, default=-1, help="timed plain-LM steps (-1: K)")
    ap.add_argument("--e2e-steps", type=int, default=1)
    ap.add_argument("--fp64-sample", type=int, default=16384,
                    help="pixels of the FP32-vs-FP64 comparison of the plain algorithm (0: off)")
    ap.add_argument("--autotune", type=int, default=1,
                    help="tune each arm's plan on the map before timing (me_plan_autotune)")
    ap.add_argument("--mlp-compare", type=int, default=1,
                    help="time the initialiser's map inference with each GEMM kernel "
                         "(outside the timed region); 2: also retrain with mma.sync")
    return ap.parse_args()


def use_widened(args):
    if args.bounds == "auto":
        return me_maps.WORKLOADS[args.workload]["kind"] == "fe15648"
    return args.bounds == "widened"


def reference_arm(args):
    """The reference's own CPU implementation on this host's cores."""
    rank, _, _ = me_ranks.rank_env()
    if rank != 0:
        return 0
    w = me_maps.WORKLOADS[args.workload]
    widen = use_widened(args)
    cores = host_cores()
    # ~7 ms of one core per pixel at num_run = 5: a step of ~2 s on all cores
    npix = args.npix or max(cores * 48, 256)
    prof = cpu_sample_profiles(args.workload, npix, seed=99)
    times = []
    kind = None
    for i in range(args.warmup + args.steps):
        _, dt, kind = cpu_invert(prof, args.workload, cores, widen)
        if i >= args.warmup:
            times.append(dt)
    step = max(times)
    value = npix / step
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 0,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": step * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded draws of the workload's parameter distributions)",
            "config": {"workload": args.workload,
                       "bounds": "widened" if widen else "workload's own",
                       "pixels_per_step": npix,
                       "num_run": int(w["ctl"].get("num_run", 4)), "nl": w["nl"],
                       "init": "Init_Guess + random restarts (the reference's algorithm)",
                       "cpu_processes": cores},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind,
                             "sample": f"{npix} pixels of {args.workload} per step, "
                                       f"{cores} processes of the reference core"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def _flops(c):
    return c.get("add", 0) + c.get("mul", 0) + c.get("div", 0) + c.get("sqrt", 0)


def event_flops(fc, nl, jacobians, trials):
    """Algorithmic FLOPs of LM work (the reference algorithm, counted per event
    with a counting scalar type: tests/golden/flop_counts.json) split by the
    kernel that does it: synthesis with Jacobian + normal equations per
    Jacobian; an SVD solve of H for the first trial after each Jacobian and of
    an orthogonal U factor for every later trial; a forward synthesis + chi^2
    per trial."""
    first = jacobians
    later = max(trials - first, 0)
    return {"jac": jacobians * nl * (_flops(fc["jacobian_per_lambda"])
                                     + _flops(fc["normal_equations_per_lambda"])),
            "svd": first * _flops(fc["svd_solve_normal_matrix"])
            + later * _flops(fc["svd_solve_orthogonal"]),
            "trial": trials * nl * (_flops(fc["forward_per_lambda"])
                                    + _flops(fc["loss_per_lambda"]))}


def kernel_rooflines(st, fc, nl, peak):
    """Per-kernel algorithmic FLOP/s from a profiled batch (me_plan_set_profiling):
    the round kernels over the events the rounds did, the tail kernel over
    the rest."""
    tj, tt = st["tail_jacobians"], st["tail_trials"]
    rounds = event_flops(fc, nl, st["jacobians"] - tj, st["trials"] - tt)
    tail = event_flops(fc, nl, tj, tt)
    out = {}
    for name, ms, fl in (("jac_kernel", st["jac_ms"], rounds["jac"]),
                         ("svd_kernel", st["svd_ms"], rounds["svd"]),
                         ("trial_kernel", st["trial_ms"], rounds["trial"]),
                         ("finish_kernel", st["tail_ms"], sum(tail.values()))):
        if ms > 0:
            tf = fl / (ms / 1e3) / 1e12
            out[name] = {"ms": ms, "algorithmic_flop": fl, "tflops": tf, "frac": tf / peak}
    return out


def param_errors(res, ref):
    """Median and 99th percentile |res - ref| per parameter in G, deg, deg,
    m/s, mA, -, -, -, - (S, beta in continuum units)."""
    names = ["B_G", "theta_deg", "phi_deg", "v_m_s", "doppler_mA", "damping", "eta0", "S",
             "beta"]
    scale = [1.0, 180 / np.pi, 180 / np.pi, 1e3, 1.0, 1.0, 1.0, 1.0, 1.0]
    d = np.abs(res[:, :9] - ref[:, :9])
    d[:, 2] = np.minimum(d[:, 2], np.pi - d[:, 2])  # azimuth is folded into [0, pi)
    return {n: [float(np.median(d[:, k]) * sc), float(np.quantile(d[:, k], 0.99) * sc)]
            for k, (n, sc) in enumerate(zip(names, scale))}


def work_histograms(counts):
    """Per-pixel LM iterations and runs of a step (inverted pixels only):
    histogram bins 0..29 iterations and 30+, 1..20 runs and 21+."""
    if counts is None:
        return None
    c = counts[counts[:, 0] > 0]
    it = np.minimum(c[:, 1], 30)
    runs = np.minimum(c[:, 0], 21)
    return {"pixels": int(c.shape[0]),
            "iterations": np.bincount(it, minlength=31).tolist(),
            "runs": np.bincount(runs, minlength=22)[1:].tolist(),
            "iterations_median_p99": [float(np.median(c[:, 1])), float(np.quantile(c[:, 1], 0.99))],
            "trials_per_pixel": float(c[:, 2].mean())}


def initialiser_gemm_compare(torch, init, plan, prof, npix, stream, args, name, rank):
    """The initialiser's map inference (features, four GEMMs, decode) timed with
    each GEMM kernel on the resident map (CUDA events, mean of 5 after one
    warm-up), and with --mlp-compare 2 the training wall time with mma.sync
    beside the tcgen05 training of the run."""
    import me_b200
    out = torch.empty((npix, 9), dtype=torch.float64, device="cuda")
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    res = {"map_pixels": npix, "inference_ms": {}}
    for path in ("tcgen05", "mma_sync"):
        init.set_gemm(path)
        init.predict_device(prof.data_ptr(), npix, out.data_ptr(), stream.cuda_stream)
        e0.record(stream)
        for _ in range(5):
            init.predict_device(prof.data_ptr(), npix, out.data_ptr(), stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize()
        res["inference_ms"][path] = e0.elapsed_time(e1) / 5
    init.set_gemm("tcgen05")
    if args.mlp_compare > 1:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        other = me_b200.Initializer.train(plan, samples=args.train_samples,
                                          epochs=args.train_epochs, seed=20240607 + 7919 * rank,
                                          gemm=me_b200.GEMM_PATHS["mma_sync"],
                                          **me_maps.train_prior(name))
        torch.cuda.synchronize()
        res["train_s_mma_sync"] = time.perf_counter() - t0
        res["final_loss_mma_sync"] = other.final_loss
        other.close()
    res["gemm_launches"] = init.gemm_launches()
    return res


def timed_steps(torch, step, n, stream, dist, clk=None):
    """Runs n steps between a barrier + synchronize on both sides; returns
    (seconds, per-step stats), max over ranks."""
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    stats = []
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ctx = clk if clk is not None else _Null()
    with ctx:
        ev0.record(stream)
        for _ in range(n):
            stats.append(step())
        ev1.record(stream)
        torch.cuda.synchronize()
    if dist:
        dist.barrier()
    elapsed = me_ranks.max_over_ranks(ev0.elapsed_time(ev1) / 1e3, dist, "cuda")
    return elapsed, stats


class _Null:
    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False


def main():
    args = parse()
    if args.impl == "reference":
        return reference_arm(args)

    import torch
    import me_b200

    rank, world, local = me_ranks.rank_env()
    torch.cuda.set_device(local)
    dist = me_ranks.init("nccl", 600, torch.device("cuda", local))

    w = me_maps.WORKLOADS[args.workload]
    name = args.workload
    widen = use_widened(args)
    npix = args.npix or w["npix"]
    lam = me_maps.wavelengths(name)
    nl = lam.size
    seed = me_ranks.map_seed(rank)

    # ---- synthetic map resident in HBM: seeded draws -> GPU FP64 synthesis + noise
    gen = me_b200.Plan(me_b200.parse_config_text(me_maps.control_text(name, precision="FP64")),
                       lam, device=local)
    par_true = me_maps.draw_parameters(name, npix, seed)
    d_par = torch.from_numpy(par_true).cuda()
    prof = torch.empty((npix, 4, nl), dtype=torch.float64, device="cuda")
    gen.synthesize_device(d_par.data_ptr(), npix, prof.data_ptr())
    g = torch.Generator(device="cuda").manual_seed(seed)
    prof += w["noise"] * torch.randn(prof.shape, dtype=torch.float64, device="cuda", generator=g)
    torch.cuda.synchronize()
    gen.close()
    res = torch.zeros((npix, 10), dtype=torch.float64, device="cuda")
    res_plain = torch.zeros((npix, 10), dtype=torch.float64, device="cuda")

    ctl = me_maps.control_text(name, precision=args.precision, seed=seed, widen_bounds=widen)
    plan = me_b200.Plan(me_b200.parse_config_text(ctl), lam, device=local)
    plain = me_b200.Plan(me_b200.parse_config_text(ctl), lam, device=local)
    stream = torch.cuda.current_stream()

    # ---- the learned initialiser: trained on the GPU for this line and grid
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    torch.cuda.nvtx.range_push("train")
    init = me_b200.Initializer.train(plan, samples=args.train_samples, epochs=args.train_epochs,
                                     seed=20240607 + 7919 * rank, **me_maps.train_prior(name))
    torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0
    plan.set_initializer(init)
    tuned, tuned_plain = None, None
    if args.autotune:
        tuned = plan.autotune(prof.data_ptr(), npix, stream.cuda_stream)

    def step():
        return plan.invert_device(prof.data_ptr(), npix, res.data_ptr(), 0, stream.cuda_stream)

    def step_plain():
        return plain.invert_device(prof.data_ptr(), npix, res_plain.data_ptr(), 0,
                                   stream.cuda_stream)

    nvtx = torch.cuda.nvtx  # ranges name the phases for ncu --nvtx-include
    nvtx.range_push("warmup")
    for _ in range(args.warmup):
        step()
    nvtx.range_pop()
    clk = ClockSampler(local)
    nvtx.range_push("timed")
    elapsed, stats = timed_steps(torch, step, args.steps, stream, dist, clk)
    nvtx.range_pop()
    step_s = elapsed / args.steps
    last = stats[-1]
    kernel_ms = statistics.mean(s["kernel_ms"] for s in stats)
    init_ms = statistics.mean(s["init_ms"] for s in stats)

    # ---- per-pixel LM work of the last learned-start step
    counts_learned = plan.last_counters(npix)

    # ---- one more step with per-kernel CUDA events (outside the timed region)
    nvtx.range_push("profiled")
    plan.set_profiling(True)
    prof_stats = step()
    plan.set_profiling(False)
    nvtx.range_pop()

    # ---- the initialiser's inference with each GEMM kernel (outside the timed region)
    mlp_cmp = None
    if args.mlp_compare:
        nvtx.range_push("mlp_compare")
        mlp_cmp = initialiser_gemm_compare(torch, init, plan, prof, npix, stream, args, name,
                                           rank)
        nvtx.range_pop()

    # ---- the plain LM with the reference's restarts, same map and GPU
    plain_steps = args.steps if args.plain_steps < 0 else args.plain_steps
    plain_s, plain_last = None, None
    counts_plain = None
    if plain_steps > 0:
        if args.autotune:
            tuned_plain = plain.autotune(prof.data_ptr(), npix, stream.cuda_stream)
        step_plain()  # warm-up (slot buffers, caches)
        nvtx.range_push("plain")
        el, pst = timed_steps(torch, step_plain, plain_steps, stream, dist)
        nvtx.range_pop()
        plain_s, plain_last = el / plain_steps, pst[-1]
        counts_plain = plain.last_counters(npix)

    # ---- FP32 synthesis against the FP64 path on the GPU: the plain algorithm
    # on a seeded sample of the map, same pixels, both precisions
    fp_cmp = None
    if args.fp64_sample > 0 and args.precision == "FP32":
        ns = min(npix, args.fp64_sample)
        sel = torch.from_numpy(np.sort(np.random.default_rng(11).choice(npix, ns, replace=False)))
        sprof = prof[sel.cuda()].contiguous()
        out32 = torch.zeros((ns, 10), dtype=torch.float64, device="cuda")
        out64 = torch.zeros((ns, 10), dtype=torch.float64, device="cuda")
        ctl64 = me_maps.control_text(name, precision="FP64", seed=seed, widen_bounds=widen)
        with me_b200.Plan(me_b200.parse_config_text(ctl), lam, device=local) as p32, \
                me_b200.Plan(me_b200.parse_config_text(ctl64), lam, device=local) as p64:
            p32.invert_device(sprof.data_ptr(), ns, out32.data_ptr(), 0, stream.cuda_stream)
            p64.invert_device(sprof.data_ptr(), ns, out64.data_ptr(), 0, stream.cuda_stream)
        torch.cuda.synchronize()
        a, b = out32.cpu().numpy(), out64.cpu().numpy()
        v = b[:, 9] > 0
        ratio = a[v, 9] / b[v, 9]
        fp_cmp = {"pixels": int(ns), "param_err_median_p99": param_errors(a[v], b[v]),
                  "chi2_ratio_q01_q50_q99": [float(np.quantile(ratio, q)) for q in (0.01, 0.5, 0.99)],
                  "chi2_within_1.05": float(np.mean(ratio <= 1.05))}

    # ---- end to end through the host entry point (pinned host buffers)
    e2e = None
    if args.e2e_steps > 0:
        h_prof = torch.empty((npix, 4, nl), dtype=torch.float64, pin_memory=True)
        h_prof.copy_(prof)
        h_prof_np = h_prof.numpy()
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            _, st_e2e = plan.invert(h_prof_np)
        e2e_s = me_ranks.max_over_ranks((time.perf_counter() - t0) / args.e2e_steps, dist, "cuda")
        e2e = {"seconds": e2e_s, "h2d_ms": st_e2e["h2d_ms"], "d2h_ms": st_e2e["d2h_ms"]}

    res_np = res.cpu().numpy()
    res_plain_np = res_plain.cpu().numpy()
    out = {}
    if rank == 0:
        # ---- CPU leg: the reference core on a seeded sample of this map, timed on
        # the host cores (cpu_baseline); its chi^2 decides which of the GPU's
        # pixels count as converged (chi^2 <= 1.05 x the reference's)
        cores = host_cores()
        nb = min(npix, max(args.sample, cores * 32))
        rng = np.random.default_rng(7)
        idx = np.sort(rng.choice(npix, size=nb, replace=False))
        sample_prof = prof[idx].cpu().numpy()
        ref_res, base_dt, base_kind = cpu_invert(sample_prof, name, cores, widen)
        valid = ref_res[:, 9] > 0

        def conv(r):
            ratio = r[idx, 9][valid] / ref_res[valid, 9]
            return (float(np.mean(ratio <= 1.05)) if valid.any() else 0.0,
                    [float(np.quantile(ratio, q)) for q in (0.01, 0.5, 0.99)])

        frac, ratio_q = conv(res_np)
        frac_plain, ratio_q_plain = conv(res_plain_np) if plain_s else (None, None)
        fc = json.load(open(os.path.join(ROOT, "tests", "golden", "flop_counts.json")))[name]
        peak = fp32_peak_tflops(torch)
        kr = kernel_rooflines(prof_stats, fc, nl, peak)
        top = max(kr, key=lambda k: kr[k]["ms"])
        alg_step = sum(event_flops(fc, nl, last["jacobians"], last["trials"]).values())
        out = {"frac": frac, "ratio_q": ratio_q, "frac_plain": frac_plain,
               "ratio_q_plain": ratio_q_plain, "cpu_value": nb / base_dt, "nb": nb,
               "base_kind": base_kind, "cores": cores, "kernels": kr, "top": top,
               "alg_step": alg_step, "step_tflops": alg_step / (kernel_ms / 1e3) / 1e12,
               "clk": clk.summary(), "peak": peak,
               "err_vs_ref": param_errors(res_np[idx][valid], ref_res[valid]),
               "err_vs_truth": param_errors(res_np, par_true),
               "err_vs_truth_ref": param_errors(ref_res[valid], par_true[idx][valid])}

    if dist:
        dist.barrier()
    if rank == 0:
        pix_per_s = npix * world / step_s
        value = pix_per_s * out["frac"]
        plain_cfg = None
        if plain_s:
            plain_raw = npix * world / plain_s
            plain_cfg = {"converged_pixels_per_s": plain_raw * out["frac_plain"],
                         "raw_pixels_per_s": plain_raw, "ms_per_step": plain_s * 1e3,
                         "converged_fraction": out["frac_plain"],
                         "chi2_ratio_q01_q50_q99": out["ratio_q_plain"],
                         "runs_per_pixel": plain_last["runs"] / max(1, plain_last["valid"]),
                         "steps": plain_steps, "warmup": 1}
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_s * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32+f64 (MLP bf16)" if args.precision == "FP32" else "f64 (MLP bf16)",
            "data": "synthetic (seeded draws of the workload's parameter distributions, "
                    "GPU FP64 synthesis + Gaussian noise)",
            "config": {"workload": name, "bounds": "widened" if widen else "workload's own",
                       "pixels_per_gpu": npix,
                       "nl": nl, "num_run": int(w["ctl"].get("num_run", 4)),
                       "chisq_criteria": float(w["ctl"].get("chisq_criteria", 1.0)),
                       "precision": args.precision,
                       "init": "learned (MLP 240-256-256-256-10 GELU), then the reference's "
                               "restarts for pixels above chisq_criteria",
                       "train": {"samples": args.train_samples, "epochs": args.train_epochs,
                                 "batch": 4096, "lr": 1e-3, "seconds": train_s,
                                 "final_loss": init.final_loss},
                       "parallelism": f"pixel shards x{world}",
                       "l2": "inputs larger than L2 (2 GB of profiles per GPU)",
                       "raw_pixels_per_s": pix_per_s,
                       "converged_fraction": out["frac"],
                       "converged_sample": f"{out['nb']} seeded pixels vs the "
                                           f"{out['base_kind']} FP64 chi^2",
                       "chi2_ratio_q01_q50_q99": out["ratio_q"],
                       "runs_per_pixel": last["runs"] / max(1, last["valid"]),
                       "ended_after_learned_start": last["learned_done"] / max(1, last["valid"]),
                       "fallback_rate": 1.0 - last["learned_done"] / max(1, last["valid"]),
                       "profile_stream": {
                           "bytes_per_pixel": 4 * nl * 8 + 10 * 8,
                           "gb_per_s": npix * (4 * nl * 8 + 10 * 8) / step_s / 1e9,
                           "note": "profiles read once and results written once per step "
                                   "(HBM), far below the measured HBM bandwidth: the path is "
                                   "compute bound"},
                       "init_ms_per_step": init_ms,
                       "initialiser_gemm": mlp_cmp,
                       "autotuned": {"learned": tuned, "plain": tuned_plain},
                       "histograms": {"learned": work_histograms(counts_learned),
                                      "plain": work_histograms(counts_plain)},
                       "fp32_vs_fp64_plain": fp_cmp,
                       "plain_lm": plain_cfg,
                       "learned_vs_plain": (value / plain_cfg["converged_pixels_per_s"]
                                            if plain_cfg else None),
                       "param_err_vs_fp64_ref_median_p99": out["err_vs_ref"],
                       "param_err_vs_truth_median_p99": out["err_vs_truth"],
                       "ref_param_err_vs_truth_median_p99": out["err_vs_truth_ref"]},
            "gpu_launches": int(sum(s["launches"] for s in stats)),
            "e2e": None, "clocks": out["clk"],
            "roofline": {"bound": "fp32", "kernel": out["top"],
                         "achieved": out["kernels"][out["top"]]["tflops"],
                         "peak": out["peak"], "unit": "TFLOP/s",
                         "frac": out["kernels"][out["top"]]["frac"],
                         "traffic": None,
                         "note": "dominant kernel by device time in a profiled step (CUDA "
                                 "events around every launch): algorithmic FLOPs of the "
                                 "reference algorithm for the events it ran (counted with a "
                                 "counting scalar type) / its time; peak = FP32 FFMA rate "
                                 "measured in this run with cuBLAS SGEMM, TF32 off "
                                 "(MEASURED_PEAKS.json has no FP32 figure)",
                         "kernels": out["kernels"],
                         "step_algorithmic_tflops": out["step_tflops"],
                         "algorithmic_flop_per_step": out["alg_step"]},
            "cpu_baseline": {"value": out["cpu_value"], "unit": UNIT, "cores": out["cores"],
                             "kind": out["base_kind"],
                             "sample": f"{out['nb']} seeded pixels of the map, "
                                       f"{out['cores']} processes of the reference core"},
            "stats": {k: last[k] for k in ("valid", "runs", "iterations", "trials", "accepted",
                                           "jacobians", "redo_pixels", "launches",
                                           "learned_done")},
        }
        if e2e:
            line["e2e"] = {"value": npix * world / e2e["seconds"] * out["frac"], "unit": UNIT,
                           "h2d_bytes_per_step": npix * 4 * nl * 8,
                           "d2h_bytes_per_step": npix * 10 * 8,
                           "h2d_ms": e2e["h2d_ms"], "d2h_ms": e2e["d2h_ms"]}
        print(json.dumps(line), flush=True)
    init.close()
    plan.close()
    plain.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def fp32_peak_tflops(torch):
    """FP32 FFMA throughput of this GPU: cuBLAS SGEMM with TF32 disabled."""
    old = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        n = 8192
        a = torch.randn(n, n, device="cuda")
        b = torch.randn(n, n, device="cuda")
        for _ in range(2):
            torch.mm(a, b)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        best = 0.0
        for _ in range(3):
            e0.record()
            torch.mm(a, b)
            e1.record()
            torch.cuda.synchronize()
            best = max(best, 2 * n ** 3 / (e0.elapsed_time(e1) / 1e3) / 1e12)
        return best
    finally:
        torch.backends.cuda.matmul.allow_tf32 = old


if __name__ == "__main__":
    sys.exit(main())
