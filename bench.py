#!/usr/bin/env python
"""Benchmark of the B200 Milne-Eddington inversion (one JSON line on stdout).

Metric: converged pixels/s on one B200 -- pixels inverted per second, counted
as converged when their chi^2 is <= 1.05 x the chi^2 the reference's FP64 C
code reaches on the same profile -- with the learned initialiser, beside the
plain LM with the reference's random restarts on the same map and GPU.  The
converged share is measured on a seeded sample of the map against the
reference core (oracle/_ref, the reference's own C sources compiled here; the
oracle restatement where it was not built, and for the instrument filter the
reference does not have).

Workload (default): the 1024x1024 Fe I 15648.5 A map (nl = 60, seeded draws of
B, theta, phi, v, Doppler width, damping, eta0, beta; S = 1; noise 1e-3),
num_run = 5, chisq_criteria = 1.5, FP32 synthesis with FP64 SVD solve and
chi^2 test, with Bounds_Dopp = 100, 400 mA and Bounds_Damp = 0.05, 1.0: the
default Doppler bounds (10-80 mA) cannot reach the drawn widths (150-350 mA),
so with them no start can fit and chisq_criteria is met by a sixth of the
pixels at best (`--bounds literal` runs that variant; the default line also
reports it under `other_workloads`).

The sample pixels (4096 by default) are the same in both arms: seeded indices
into the map, the map's own parameter draws, synthesised on the host by the
reference's own Milne_Eddington_Single and given seeded host noise.  The GPU
arm writes them into its map before anything runs, inverts them with the map,
and compares them with the reference core; the reference arm (`--impl
reference`) times the reference core on exactly those pixels.

The parity block puts every GPU arm beside the reference on the sample, next
to the reference's own spread on the same pixels (another restart seed, and a
one-ulp change of the input), with per-parameter tolerances.

The initialiser is trained once per line and grid before the timed region
(4M profiles synthesised on the GPU from seeded draws of the same
distributions, other seeds than the map's, 20 epochs of Adam, lr 1e-3, batch
4096); its training time is reported, its inference is inside every step.

A step is one inversion of the whole map.  The map (2 GB of FP64 profiles,
larger than L2) is resident in HBM when the timed region starts; `e2e` times
the same step through the host entry point me_invert_batch with the profiles
and the results in pinned host memory (host->device copy, inference,
inversion, device->host copy of the results).

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

import me_maps  # noqa: E402  (pure Python: workload definitions)
import me_ranks  # noqa: E402  (pure Python: rank plumbing)

METRIC = "converged pixels/s on 1 B200 at chi2<=1.05x FP64 ref: learned-init vs plain LM"
UNIT = "pixels/s"
REF_SEED = 4242      # restart stream of the reference run that defines "converged"
REF_SEED_B = 99991   # a second restart stream: the reference's seed-to-seed spread

# Per-parameter tolerance on |GPU - reference| (units of param_errors):
# G, deg, deg, m/s, mA, -, -, continuum, -.
TOLERANCE = {"B_G": 1.0, "theta_deg": 0.1, "phi_deg": 0.1, "v_m_s": 1.0, "doppler_mA": 0.1,
             "damping": 1e-3, "eta0": 0.1, "S": 1e-3, "beta": 1e-3}


# ---------------------------------------------------------------------------
# CPU side: the reference's own C core (or the oracle port) on host cores,
# in spawned worker processes (one set-up per process, reseeded per run).
# ---------------------------------------------------------------------------
_W = {}


def _cpu_worker_init(kind, workload, npix_max, widen):
    sys.path[:0] = [os.path.join(ROOT, "tests"), PKG]
    import oracle_bind as ob
    lam = me_maps.wavelengths(workload)
    _W["kind"] = kind
    if kind == "reference":
        # the reference's own parser (RDINPUT) and INIT_INV; nothing of this
        # library is loaded in this process
        _W["eng"] = ob.Reference(me_maps.reference_control_text(workload, widen_bounds=widen),
                                 lam, npix_max, seed=REF_SEED)
    else:
        import me_b200
        cfg = me_b200.parse_config_text(me_maps.control_text(workload, precision="FP64",
                                                             widen_bounds=widen))
        _W["eng"] = ob.Oracle(cfg, lam)


def _ulp_perturb(prof):
    rng = np.random.default_rng(5)
    return prof * (1 + 2.3e-16 * rng.choice([-1, 1], prof.shape))


def _cpu_worker_invert(job):
    prof, seed, perturb = job
    eng = _W["eng"]
    if perturb:
        prof = _ulp_perturb(prof)
    if _W["kind"] == "reference":
        eng.reseed(seed)
        return eng.invert(prof)
    import oracle_bind as ob
    eng.carry[0] = 0.0
    return eng.invert(prof, rng_mode=ob.MEO_RNG_NR, nr_seed=seed)


def _cpu_worker_synth(par):
    eng = _W["eng"]
    return np.stack([eng.synth(p) for p in np.atleast_2d(par)])


def cpu_kind(workload):
    """The reference's own core where it was built here and the workload is
    within its reach; the oracle port (the same algorithm restated, with the
    instrument-filter extension) otherwise."""
    if me_maps.WORKLOADS[workload]["ctl"].get("filter", "0") != "0":
        return "port"
    return "reference" if os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libmeref.so")) \
        else "port"


class CpuPool:
    """`procs` spawned processes of the reference core (or the port) for one
    workload: host-side synthesis of sample pixels and timed inversions."""

    def __init__(self, workload, procs, npix_max, widen):
        self.kind = cpu_kind(workload)
        self.procs = max(1, procs)
        ctx = mp.get_context("spawn")
        self.pool = ctx.Pool(self.procs, initializer=_cpu_worker_init,
                             initargs=(self.kind, workload, max(1, npix_max), widen))

    def synth(self, par):
        chunks = np.array_split(np.arange(par.shape[0]), self.procs)
        return np.concatenate(self.pool.map(_cpu_worker_synth, [par[c] for c in chunks if len(c)]))

    def invert(self, prof, seed=REF_SEED, perturb=False):
        """(results, seconds): prof split in `procs` contiguous slices, each
        process one slice from a fresh restart stream (as independent
        reference processes would)."""
        chunks = [c for c in np.array_split(np.arange(prof.shape[0]), self.procs) if len(c)]
        t0 = time.perf_counter()
        parts = self.pool.map(_cpu_worker_invert, [(prof[c], seed, perturb) for c in chunks])
        return np.concatenate(parts), time.perf_counter() - t0

    def close(self):
        self.pool.close()
        self.pool.join()


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def sample_size(args, cores):
    return max(args.sample, cores * 32)


def sample_profiles(pool, workload, npix, nsample, map_seed):
    """The map's sample pixels: seeded indices, the map's own parameter draws,
    synthesised on the host by the CPU pool's core, plus seeded host noise."""
    idx = me_maps.sample_indices(npix, nsample)
    par = me_maps.draw_parameters(workload, npix, map_seed)[idx]
    prof = pool.synth(par) + me_maps.sample_noise(workload, idx.size, map_seed)
    return idx, prof


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
                    help="pixels of the sample (converged share, parity, reference arm)")
    ap.add_argument("--train-samples", type=int, default=4 << 20)
    ap.add_argument("--train-epochs", type=int, default=20)
    ap.add_argument("--plain-steps", type=int, default=-1, help="timed plain-LM steps (-1: K)")
    ap.add_argument("--e2e-steps", type=int, default=1)
    ap.add_argument("--e2e-warmup", type=int, default=1,
                    help="untimed calls of the host entry point before its timed steps")
    ap.add_argument("--fp64-sample", type=int, default=16384,
                    help="pixels of the FP32-vs-FP64 comparison of the plain algorithm (0: off)")
    ap.add_argument("--autotune", type=int, default=1,
                    help="tune each arm's plan on the map before timing (me_plan_autotune)")
    ap.add_argument("--mlp-compare", type=int, default=1,
                    help="time the initialiser's map inference with each GEMM kernel "
                         "(outside the timed region); 2: also retrain with mma.sync")
    ap.add_argument("--parity", type=int, default=1,
                    help="reference self-spread and per-parameter parity block on the sample")
    ap.add_argument("--other-workloads", default="fe6302_2048x1024,fe6173_4096x4096,literal",
                    help="comma list of further workloads measured after the headline "
                         "(N = 1 only; 'literal' = the headline map with the literal bounds); "
                         "empty: none")
    ap.add_argument("--svd-registers", type=int, default=-1,
                    help="me_plan_set_svd_registers for both arms after any autotuning "
                         "(-1: leave the default / the autotuner's choice)")
    ap.add_argument("--kernel-variant", type=int, default=-1,
                    help="me_plan_set_kernel_variant for both arms after any autotuning "
                         "(-1: leave the default / the autotuner's choice)")
    ap.add_argument("--other-budget-s", type=float, default=480.0,
                    help="wall-time budget of the further workloads; one that would start "
                         "past it is skipped")
    return ap.parse_args()


def use_widened(args, workload=None):
    if args.bounds == "auto":
        return me_maps.WORKLOADS[workload or args.workload]["kind"] == "fe15648"
    return args.bounds == "widened"


def arm_config(workload, widen, npix, nsample, precision=None):
    """The configuration both arms report: the workload and its sample."""
    w = me_maps.WORKLOADS[workload]
    return {"workload": workload, "map_pixels": npix, "nl": w["nl"],
            "num_run": int(w["ctl"].get("num_run", 4)),
            "chisq_criteria": float(w["ctl"].get("chisq_criteria", 1.0)),
            "bounds": "widened" if widen else "workload's own",
            "sample": f"{nsample} seeded pixels of the map (same in both arms)"}


def reference_arm(args):
    """The reference's own CPU implementation on this host's cores, on the
    GPU arm's sample pixels: the reference's parser, synthesis and
    INVERSION_MULTI (oracle/_ref), nothing of this library."""
    rank, _, _ = me_ranks.rank_env()
    if rank != 0:
        return 0
    name = args.workload
    widen = use_widened(args)
    cores = host_cores()
    npix = args.npix or me_maps.WORKLOADS[name]["npix"]
    nb = min(npix, sample_size(args, cores))
    pool = CpuPool(name, cores, (nb + cores - 1) // cores, widen)
    try:
        _, prof = sample_profiles(pool, name, npix, nb, me_ranks.map_seed(0))
        pool.invert(prof[:cores])  # every worker set up
        times = []
        for i in range(args.warmup + args.steps):
            _, dt = pool.invert(prof)
            if i >= args.warmup:
                times.append(dt)
    finally:
        pool.close()
    step = statistics.median(times)
    value = nb / step
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 0,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": step * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded draws of the workload's parameter distributions)",
            "config": arm_config(name, widen, npix, nb),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": pool.kind,
                             "sample": f"{nb} seeded pixels of {name} (the GPU arm's sample) "
                                       f"per step, {cores} processes of the reference core, "
                                       f"median step"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "init": "Init_Guess + random restarts (the reference's algorithm)"}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# rooflines, errors, parity
# ---------------------------------------------------------------------------
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


def kernel_rooflines(st, fc, nl, peak, peak64):
    """Per-kernel algorithmic FLOP/s from a profiled batch (me_plan_set_profiling):
    the round kernels over the events the rounds did, the tail kernel over
    the rest.  frac: of the FP32 peak; frac_of_fp64_peak: of the FP64 peak,
    the one that bounds the SVD solve (FP64 arithmetic)."""
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
            if peak64:
                out[name]["frac_of_fp64_peak"] = tf / peak64
    return out


PARAMS = ["B_G", "theta_deg", "phi_deg", "v_m_s", "doppler_mA", "damping", "eta0", "S", "beta"]


def abs_errors(res, ref):
    """|res - ref| per pixel and parameter in G, deg, deg, m/s, mA, -, -, -, -
    (the azimuth difference folded into [0, 90] deg)."""
    scale = np.array([1.0, 180 / np.pi, 180 / np.pi, 1e3, 1.0, 1.0, 1.0, 1.0, 1.0])
    d = np.abs(res[:, :9] - ref[:, :9])
    d[:, 2] = np.minimum(d[:, 2], np.pi - d[:, 2])
    return d * scale


def param_errors(res, ref):
    """Median and 99th percentile |res - ref| per parameter."""
    d = abs_errors(res, ref)
    return {n: [float(np.median(d[:, k])), float(np.quantile(d[:, k], 0.99))]
            for k, n in enumerate(PARAMS)}


def chi2_agreement(res, ref):
    """Share of the reference's inverted pixels with chi^2 <= 1.05 x the
    reference's, the chi^2 ratio quantiles, and the share identical in all
    ten outputs (1e-6 relative)."""
    v = ref[:, 9] > 0
    if not v.any():
        return {"within_1.05": 0.0, "ratio_q01_q50_q99": None, "identical": 0.0}
    ratio = res[v, 9] / ref[v, 9]
    same = np.all(np.abs(res - ref) <= 1e-6 * np.abs(ref) + 1e-12, axis=1)[v]
    return {"within_1.05": float(np.mean(ratio <= 1.05)),
            "ratio_q01_q50_q99": [float(np.quantile(ratio, q)) for q in (0.01, 0.5, 0.99)],
            "identical": float(same.mean())}


def parity_vs_reference(res, ref, spread):
    """A GPU arm against the reference on the sample: per parameter median /
    p99 |delta| and pass/fail.  A parameter passes when its median is within
    the stated tolerance or within 1.1 x the reference's own spread, and its
    p99 within 1.25 x that spread (or the tolerance): the spread is the larger
    of the reference against itself with another restart seed and with a
    one-ulp input change, on the same pixels.  (A p99 of 4096 pixels rests on
    its ~41 largest differences and varies by about 10 % between samples.)
    The chi^2 test passes when the share within 1.05 x is no more than 0.02
    below the reference's own."""
    v = ref[:, 9] > 0
    err = param_errors(res[v], ref[v])
    params = {}
    for n in PARAMS:
        med, p99 = err[n]
        smed = max(spread[k]["err"][n][0] for k in spread)
        sp99 = max(spread[k]["err"][n][1] for k in spread)
        tol = TOLERANCE[n]
        params[n] = {"median_p99": [med, p99], "tolerance": tol,
                     "ref_spread_median_p99": [smed, sp99],
                     "pass": bool(med <= max(tol, 1.1 * smed) and p99 <= max(tol, 1.25 * sp99)),
                     "within_tolerance_median": bool(med <= tol)}
    chi = chi2_agreement(res, ref)
    s_within = min(spread[k]["chi2"]["within_1.05"] for k in spread)
    chi["ref_spread_within_1.05"] = s_within
    chi["pass"] = bool(chi["within_1.05"] >= s_within - 0.02)
    return {"params": params, "chi2": chi,
            "all_pass": bool(chi["pass"] and all(p["pass"] for p in params.values()))}


def truth_recovery(res, ref, truth):
    """The learned start against the truth, beside the reference against the
    truth on the same pixels: a parameter passes when neither its median nor
    its p99 error exceeds the reference's (or the tolerance)."""
    v = ref[:, 9] > 0
    a = param_errors(res[v], truth[v])
    b = param_errors(ref[v], truth[v])
    out = {}
    for n in PARAMS:
        tol = TOLERANCE[n]
        out[n] = {"gpu_vs_truth_median_p99": a[n], "ref_vs_truth_median_p99": b[n],
                  "pass": bool(a[n][0] <= max(tol, b[n][0]) and a[n][1] <= max(tol, b[n][1]))}
    return out


def work_histograms(counts):
    """Per-pixel LM iterations and runs of a step (inverted pixels only):
    histogram bins 0..29 iterations and 30+, 1..20 runs and 21+."""
    if counts is None:
        return None
    c = counts[counts[:, 0] > 0]
    if c.shape[0] == 0:
        return None
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


def gpu_map(torch, me_b200, name, npix, seed, device):
    """A seeded map resident in HBM: the workload's parameter draws, the GPU's
    FP64 synthesis, Gaussian noise.  Returns (true parameters, profiles)."""
    w = me_maps.WORKLOADS[name]
    lam = me_maps.wavelengths(name)
    gen = me_b200.Plan(me_b200.parse_config_text(me_maps.control_text(name, precision="FP64")),
                       lam, device=device)
    par_true = me_maps.draw_parameters(name, npix, seed)
    d_par = torch.from_numpy(par_true).cuda()
    prof = torch.empty((npix, 4, lam.size), dtype=torch.float64, device="cuda")
    gen.synthesize_device(d_par.data_ptr(), npix, prof.data_ptr())
    g = torch.Generator(device="cuda").manual_seed(seed)
    prof += w["noise"] * torch.randn(prof.shape, dtype=torch.float64, device="cuda", generator=g)
    torch.cuda.synchronize()
    gen.close()
    del d_par
    return par_true, prof


# ---------------------------------------------------------------------------
# further workloads (N = 1): the other configurations, measured after the
# headline with the same method, fewer steps
# ---------------------------------------------------------------------------
def other_workload(torch, me_b200, args, key, stream, cores, init_headline):
    """One further workload: learned start (1 warm-up + 2 timed steps) and
    plain LM (1 timed step after a warm-up on a part of the map), each arm
    autotuned first on the map's first 262144 pixels, the converged share of
    each against the reference core (the port with the filter) on a seeded
    sample, iteration histograms, fallback rate."""
    if key == "literal":
        name, widen, label = args.workload, False, f"{args.workload}_literal_bounds"
    else:
        name, widen, label = key, use_widened(args, key), key
    w = me_maps.WORKLOADS[name]
    lam = me_maps.wavelengths(name)
    npix = w["npix"]
    seed = me_ranks.map_seed(0)
    t_start = time.perf_counter()
    nb = min(npix, max(1024, cores * 32))
    pool = CpuPool(name, cores, (nb + cores - 1) // cores, widen)
    try:
        idx, sprof = sample_profiles(pool, name, npix, nb, seed)
        par_true, prof = gpu_map(torch, me_b200, name, npix, seed, torch.cuda.current_device())
        prof[torch.from_numpy(idx).cuda()] = torch.from_numpy(sprof).cuda()
        res = torch.zeros((npix, 10), dtype=torch.float64, device="cuda")
        ctl = me_maps.control_text(name, precision=args.precision, seed=seed, widen_bounds=widen)
        out = {"workload": name, "bounds": "widened" if widen else "workload's own",
               "map_pixels": npix, "nl": w["nl"], "num_run": int(w["ctl"].get("num_run", 4)),
               "chisq_criteria": float(w["ctl"].get("chisq_criteria", 1.0))}
        with me_b200.Plan(me_b200.parse_config_text(ctl), lam) as plan:
            if key == "literal":
                init = init_headline  # same line, grid and prior as the headline
                out["train_s"] = 0.0
            else:
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                init = me_b200.Initializer.train(plan, samples=args.train_samples,
                                                 epochs=args.train_epochs, seed=20240607,
                                                 **me_maps.train_prior(name))
                torch.cuda.synchronize()
                out["train_s"] = time.perf_counter() - t0
            plan.set_initializer(init)
            # the autotuner on a part of the map (its time stays bounded), per arm
            tune_pix = min(npix, 262144)
            tuned_l = tuned_p = None
            if args.autotune:
                tuned_l = plan.autotune(prof.data_ptr(), tune_pix, stream.cuda_stream)

            def step():
                return plan.invert_device(prof.data_ptr(), npix, res.data_ptr(), 0,
                                          stream.cuda_stream)

            step()
            el, st = timed_steps(torch, step, 2, stream, None)
            learned_s = el / 2
            counts = plan.last_counters(npix)
            res_l = res.cpu().numpy()
            plan.set_initializer(None)
            if key != "literal":
                init.close()
            if args.autotune:
                tuned_p = plan.autotune(prof.data_ptr(), tune_pix, stream.cuda_stream)
            # plain LM: warm-up on the first eighth of the map, one timed step
            part = max(1, npix // 8)
            plan.invert_device(prof.data_ptr(), part, res.data_ptr(), 0, stream.cuda_stream)
            el_p, st_p = timed_steps(torch, step, 1, stream, None)
            plain_s = el_p
            counts_p = plan.last_counters(npix)
            res_p = res.cpu().numpy()
        del prof, res
        torch.cuda.empty_cache()
        ref_res, ref_dt = pool.invert(sprof)
    finally:
        pool.close()
    learned = chi2_agreement(res_l[idx], ref_res)
    plain = chi2_agreement(res_p[idx], ref_res)
    raw_l, raw_p = npix / learned_s, npix / plain_s
    last = st[-1]
    out.update({
        "converged_pixels_per_s": raw_l * learned["within_1.05"],
        "plain_converged_pixels_per_s": raw_p * plain["within_1.05"],
        "learned_vs_plain": (raw_l * learned["within_1.05"]) / max(1e-9, raw_p * plain["within_1.05"]),
        "raw_pixels_per_s": raw_l, "plain_raw_pixels_per_s": raw_p,
        "ms_per_step": learned_s * 1e3, "plain_ms_per_step": plain_s * 1e3,
        "steps": 2, "plain_steps": 1,
        "converged_fraction": learned["within_1.05"], "plain_converged_fraction": plain["within_1.05"],
        "chi2_ratio_q01_q50_q99": learned["ratio_q01_q50_q99"],
        "plain_chi2_ratio_q01_q50_q99": plain["ratio_q01_q50_q99"],
        "fallback_rate": 1.0 - last["learned_done"] / max(1, last["valid"]),
        "runs_per_pixel": last["runs"] / max(1, last["valid"]),
        "plain_runs_per_pixel": st_p[-1]["runs"] / max(1, st_p[-1]["valid"]),
        "histograms": {"learned": work_histograms(counts), "plain": work_histograms(counts_p)},
        "autotuned": {"learned": tuned_l, "plain": tuned_p,
                      "on_pixels": min(npix, 262144)},
        "converged_sample": f"{nb} seeded pixels vs the {pool.kind} FP64 chi^2",
        "cpu_pixels_per_s": nb / ref_dt,
        "param_err_vs_truth_median_p99": param_errors(res_l, par_true),
        "ref_param_err_vs_truth_median_p99": param_errors(ref_res[ref_res[:, 9] > 0],
                                                          par_true[idx][ref_res[:, 9] > 0]),
        "profile_stream_gb_per_s": npix * (4 * w["nl"] * 8 + 80) / learned_s / 1e9,
        "wall_s": time.perf_counter() - t_start})
    return label, out


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
    cores = host_cores()
    nb = min(npix, sample_size(args, cores))

    # ---- the sample pixels, built on the host (rank 0; same as the reference arm's)
    pool = None
    idx = sprof = None
    if rank == 0:
        pool = CpuPool(name, cores, (nb + cores - 1) // cores, widen)
        idx, sprof = sample_profiles(pool, name, npix, nb, seed)

    # ---- synthetic map resident in HBM: seeded draws -> GPU FP64 synthesis + noise
    par_true, prof = gpu_map(torch, me_b200, name, npix, seed, local)
    if rank == 0:
        prof[torch.from_numpy(idx).cuda()] = torch.from_numpy(sprof).cuda()
        torch.cuda.synchronize()
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
    for pl in (plan, plain):
        if args.svd_registers >= 0:
            pl.svd_registers = args.svd_registers
        if args.kernel_variant >= 0:
            pl.kernel_variant = args.kernel_variant

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
            if args.svd_registers >= 0:
                plain.svd_registers = args.svd_registers
            if args.kernel_variant >= 0:
                plain.kernel_variant = args.kernel_variant
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
        sprof32 = prof[sel.cuda()].contiguous()
        out32 = torch.zeros((ns, 10), dtype=torch.float64, device="cuda")
        out64 = torch.zeros((ns, 10), dtype=torch.float64, device="cuda")
        ctl64 = me_maps.control_text(name, precision="FP64", seed=seed, widen_bounds=widen)
        with me_b200.Plan(me_b200.parse_config_text(ctl), lam, device=local) as p32, \
                me_b200.Plan(me_b200.parse_config_text(ctl64), lam, device=local) as p64:
            p32.invert_device(sprof32.data_ptr(), ns, out32.data_ptr(), 0, stream.cuda_stream)
            p64.invert_device(sprof32.data_ptr(), ns, out64.data_ptr(), 0, stream.cuda_stream)
        torch.cuda.synchronize()
        a, b = out32.cpu().numpy(), out64.cpu().numpy()
        v = b[:, 9] > 0
        ratio = a[v, 9] / b[v, 9]
        fp_cmp = {"pixels": int(ns), "param_err_median_p99": param_errors(a[v], b[v]),
                  "chi2_ratio_q01_q50_q99": [float(np.quantile(ratio, q)) for q in (0.01, 0.5, 0.99)],
                  "chi2_within_1.05": float(np.mean(ratio <= 1.05))}

    # ---- the plain algorithm in FP64 on the GPU, on the sample alone (parity)
    res_fp64_sample = None
    if rank == 0 and args.parity:
        ctl64 = me_maps.control_text(name, precision="FP64", seed=seed, widen_bounds=widen)
        d_s = torch.from_numpy(sprof).cuda()
        o64 = torch.zeros((nb, 10), dtype=torch.float64, device="cuda")
        with me_b200.Plan(me_b200.parse_config_text(ctl64), lam, device=local) as p64:
            p64.invert_device(d_s.data_ptr(), nb, o64.data_ptr(), 0, stream.cuda_stream)
        torch.cuda.synchronize()
        res_fp64_sample = o64.cpu().numpy()

    # ---- end to end through the host entry point (pinned host buffers)
    e2e = None
    if args.e2e_steps > 0:
        h_prof = torch.empty((npix, 4, nl), dtype=torch.float64, pin_memory=True)
        h_prof.copy_(prof)
        h_prof_np = h_prof.numpy()
        h_res = torch.empty((npix, 10), dtype=torch.float64, pin_memory=True)
        h_res_np = h_res.numpy()
        for _ in range(args.e2e_warmup):  # first-call set-up of the streamed copy
            plan.invert(h_prof_np, out=h_res_np)
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            _, st_e2e = plan.invert(h_prof_np, out=h_res_np)
        e2e_s = me_ranks.max_over_ranks((time.perf_counter() - t0) / args.e2e_steps, dist, "cuda")
        e2e = {"seconds": e2e_s, "h2d_ms": st_e2e["h2d_ms"], "d2h_ms": st_e2e["d2h_ms"],
               "steps": args.e2e_steps, "warmup": args.e2e_warmup}
        del h_prof, h_prof_np, h_res, h_res_np

    res_np = res.cpu().numpy()
    res_plain_np = res_plain.cpu().numpy()
    out = {}
    if rank == 0:
        # ---- CPU leg: the reference core on the sample, timed on the host
        # cores (cpu_baseline); its chi^2 decides which of the GPU's pixels
        # count as converged (chi^2 <= 1.05 x the reference's)
        pool.invert(sprof[:cores])  # every worker set up
        ref_res, base_dt = pool.invert(sprof, REF_SEED)
        spread = {}
        if args.parity:
            ref_b, _ = pool.invert(sprof, REF_SEED_B)
            ref_u, _ = pool.invert(sprof, REF_SEED, perturb=True)
            v = ref_res[:, 9] > 0
            spread = {"other_restart_seed": {"err": param_errors(ref_b[v], ref_res[v]),
                                             "chi2": chi2_agreement(ref_b, ref_res)},
                      "one_ulp_input": {"err": param_errors(ref_u[v], ref_res[v]),
                                        "chi2": chi2_agreement(ref_u, ref_res)}}
        valid = ref_res[:, 9] > 0
        learned_s = res_np[idx]
        conv = chi2_agreement(learned_s, ref_res)
        conv_plain = chi2_agreement(res_plain_np[idx], ref_res) if plain_s else None
        parity = None
        if args.parity:
            arms = {"plain_fp32": res_plain_np[idx] if plain_s else None,
                    "plain_fp64": res_fp64_sample}
            parity = {"tolerance": TOLERANCE,
                      "rule": "median <= max(tol, 1.1 x ref spread median) and p99 <= max(tol, "
                              "1.25 x ref spread p99); chi2 within 1.05 share >= ref spread "
                              "share - 0.02; ref spread = the reference against itself with "
                              "another restart seed and with a one-ulp input change, same "
                              "pixels",
                      "ref_self_spread": spread,
                      "arms": {k: parity_vs_reference(r, ref_res, spread)
                               for k, r in arms.items() if r is not None}}
            # the learned start is judged by chi^2 and truth recovery: it
            # finds lower minima than the reference's restarts on most pixels
            miss = valid & (learned_s[:, 9] > 1.05 * ref_res[:, 9])
            b_miss = valid & (ref_b[:, 9] > 1.05 * ref_res[:, 9])
            parity["arms"]["learned"] = {
                "chi2": conv,
                "misses": int(miss.sum()),
                "misses_where_ref_other_seed_also_misses": int((miss & b_miss).sum()),
                "misses_within_1.05_of_ref_other_seed": int(
                    (miss & (learned_s[:, 9] <= 1.05 * ref_b[:, 9])).sum()),
                "truth_recovery": truth_recovery(learned_s, ref_res, par_true[idx]),
                "err_vs_ref_median_p99": param_errors(learned_s[valid], ref_res[valid])}
            parity["arms"]["learned"]["all_pass"] = bool(
                conv["within_1.05"] >= spread["other_restart_seed"]["chi2"]["within_1.05"] - 0.02
                and all(p["pass"] for p in parity["arms"]["learned"]["truth_recovery"].values()))
            parity["all_pass"] = bool(all(a["all_pass"] for a in parity["arms"].values()))
        fc = json.load(open(os.path.join(ROOT, "tests", "golden", "flop_counts.json")))[name]
        peak = fp32_peak_tflops(torch)
        peak64 = fp64_peak_tflops(torch)
        kr = kernel_rooflines(prof_stats, fc, nl, peak, peak64)
        top = max(kr, key=lambda k: kr[k]["ms"])
        alg_step = sum(event_flops(fc, nl, last["jacobians"], last["trials"]).values())
        out = {"conv": conv, "conv_plain": conv_plain, "parity": parity,
               "cpu_value": nb / base_dt, "base_kind": pool.kind, "kernels": kr, "top": top,
               "alg_step": alg_step, "step_tflops": alg_step / (kernel_ms / 1e3) / 1e12,
               "clk": clk.summary(), "peak": peak, "peak64": peak64,
               "err_vs_ref": param_errors(learned_s[valid], ref_res[valid]),
               "err_vs_truth": param_errors(res_np, par_true),
               "err_vs_truth_ref": param_errors(ref_res[valid], par_true[idx][valid])}
        pool.close()

    # ---- the other configurations (one GPU only; after the headline)
    others = {}
    if rank == 0 and world == 1 and args.other_workloads:
        t_other = time.perf_counter()
        del res, res_plain
        torch.cuda.empty_cache()
        for key in [k.strip() for k in args.other_workloads.split(",") if k.strip()]:
            if time.perf_counter() - t_other > args.other_budget_s:
                others[key] = {"skipped": f"wall-time budget of {args.other_budget_s} s spent"}
                continue
            try:
                label, o = other_workload(torch, me_b200, args, key, stream, cores, init)
                others[label] = o
            except Exception as exc:  # report, do not lose the headline line
                others[key] = {"error": f"{type(exc).__name__}: {exc}"}

    if dist:
        dist.barrier()
    if rank == 0:
        pix_per_s = npix * world / step_s
        frac = out["conv"]["within_1.05"]
        value = pix_per_s * frac
        plain_cfg = None
        plain_conv = None
        if plain_s:
            plain_raw = npix * world / plain_s
            plain_conv = plain_raw * out["conv_plain"]["within_1.05"]
            plain_cfg = {"converged_pixels_per_s": plain_conv,
                         "raw_pixels_per_s": plain_raw, "ms_per_step": plain_s * 1e3,
                         "converged_fraction": out["conv_plain"]["within_1.05"],
                         "chi2_ratio_q01_q50_q99": out["conv_plain"]["ratio_q01_q50_q99"],
                         "runs_per_pixel": plain_last["runs"] / max(1, plain_last["valid"]),
                         "steps": plain_steps, "warmup": 1}
        learned_vs_plain = value / plain_conv if plain_conv else None
        parity = out["parity"]
        config = arm_config(name, widen, npix, nb)
        config.update({
            "converged_fraction": frac,
            "raw_pixels_per_s": pix_per_s,
            "plain_converged_pixels_per_s": plain_conv,
            "learned_vs_plain": learned_vs_plain,
            "parity_all_pass": parity["all_pass"] if parity else None,
            "ref_seed_to_seed_within_1.05": (parity["ref_self_spread"]["other_restart_seed"]
                                             ["chi2"]["within_1.05"] if parity else None),
            "precision": args.precision,
            "parallelism": f"pixel shards x{world}",
            "l2": "inputs larger than L2 (2 GB of profiles per GPU)",
            "fallback_rate": 1.0 - last["learned_done"] / max(1, last["valid"]),
            "runs_per_pixel": last["runs"] / max(1, last["valid"]),
            "init_ms_per_step": init_ms,
            "init": "learned (MLP 240-256-256-256-10 GELU), then the reference's "
                    "restarts for pixels above chisq_criteria",
            "train": {"samples": args.train_samples, "epochs": args.train_epochs,
                      "batch": 4096, "lr": 1e-3, "seconds": train_s,
                      "final_loss": init.final_loss},
            "converged_sample": f"{nb} seeded pixels vs the {out['base_kind']} FP64 chi^2",
            "chi2_ratio_q01_q50_q99": out["conv"]["ratio_q01_q50_q99"],
            "ended_after_learned_start": last["learned_done"] / max(1, last["valid"]),
            "profile_stream": {
                "bytes_per_pixel": 4 * nl * 8 + 10 * 8,
                "gb_per_s": npix * (4 * nl * 8 + 10 * 8) / step_s / 1e9,
                "note": "profiles read once and results written once per step "
                        "(HBM), far below the measured HBM bandwidth: the path is "
                        "compute bound"},
            "initialiser_gemm": mlp_cmp,
            "autotuned": {"learned": tuned, "plain": tuned_plain},
            "histograms": {"learned": work_histograms(counts_learned),
                           "plain": work_histograms(counts_plain)},
            "fp32_vs_fp64_plain": fp_cmp,
            "plain_lm": plain_cfg,
            "param_err_vs_fp64_ref_median_p99": out["err_vs_ref"],
            "param_err_vs_truth_median_p99": out["err_vs_truth"],
            "ref_param_err_vs_truth_median_p99": out["err_vs_truth_ref"]})
        # the SVD solve computes in FP64: its roofline is the FP64 rate
        top_is64 = out["top"] == "svd_kernel" and bool(out["peak64"])
        top_bound = "fp64" if top_is64 else "fp32"
        top_peak = out["peak64"] if top_is64 else out["peak"]
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_s * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32+f64 (MLP bf16)" if args.precision == "FP32" else "f64 (MLP bf16)",
            "data": "synthetic (seeded draws of the workload's parameter distributions, "
                    "GPU FP64 synthesis + Gaussian noise; the sample pixels synthesised by "
                    "the reference core on the host)",
            "config": config,
            "plain_converged_pixels_per_s": plain_conv,
            "learned_vs_plain": learned_vs_plain,
            "parity_all_pass": parity["all_pass"] if parity else None,
            "gpu_launches": int(sum(s["launches"] for s in stats)),
            "e2e": None, "clocks": out["clk"],
            "roofline": {"bound": top_bound, "kernel": out["top"],
                         "achieved": out["kernels"][out["top"]]["tflops"],
                         "peak": top_peak, "unit": "TFLOP/s",
                         "frac": out["kernels"][out["top"]]["tflops"] / top_peak,
                         "traffic": None,
                         "note": "dominant kernel by device time in a profiled step (CUDA "
                                 "events around every launch): algorithmic FLOPs of the "
                                 "reference algorithm for the events it ran (counted with a "
                                 "counting scalar type) / its time; peak = the rate of the "
                                 "kernel's arithmetic measured in this run: FP32 FFMA (cuBLAS "
                                 "SGEMM, TF32 off) for the synthesis kernels, FP64 (cuBLAS "
                                 "DGEMM) for the SVD solve (MEASURED_PEAKS.json has neither); "
                                 "every kernel against both in 'kernels'",
                         "fp64_peak": out["peak64"],
                         "kernels": out["kernels"],
                         "step_algorithmic_tflops": out["step_tflops"],
                         "algorithmic_flop_per_step": out["alg_step"]},
            "cpu_baseline": {"value": out["cpu_value"], "unit": UNIT, "cores": cores,
                             "kind": out["base_kind"],
                             "sample": f"{nb} seeded pixels of the map, "
                                       f"{cores} processes of the reference core"},
            "parity": parity,
            "other_workloads": others or None,
            "stats": {k: last[k] for k in ("valid", "runs", "iterations", "trials", "accepted",
                                           "jacobians", "redo_pixels", "launches",
                                           "learned_done")},
        }
        if e2e:
            line["e2e"] = {"value": npix * world / e2e["seconds"] * frac, "unit": UNIT,
                           "h2d_bytes_per_step": npix * 4 * nl * 8,
                           "d2h_bytes_per_step": npix * 10 * 8,
                           "h2d_ms": e2e["h2d_ms"], "d2h_ms": e2e["d2h_ms"],
                           "steps": e2e["steps"], "warmup": e2e["warmup"],
                           "host_buffers": "page-locked (profiles streamed in chunks)"}
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
        return _gemm_peak(torch, torch.float32)
    finally:
        torch.backends.cuda.matmul.allow_tf32 = old


def fp64_peak_tflops(torch):
    """FP64 throughput of this GPU: cuBLAS DGEMM."""
    return _gemm_peak(torch, torch.float64)


def _gemm_peak(torch, dtype):
    n = 8192
    a = torch.randn(n, n, device="cuda", dtype=dtype)
    b = torch.randn(n, n, device="cuda", dtype=dtype)
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
    del a, b
    return best


if __name__ == "__main__":
    sys.exit(main())
