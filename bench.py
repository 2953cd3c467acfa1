#!/usr/bin/env python
"""Throughput of ProFit's likelihood-and-gradient on B200.

Metric: LL+grad evaluations/s of the bulge + disk + point-source model
(400x400 image, 51x51 Moffat PSF, brute-force convolution, 17-parameter
gradient) with the FP32 path and its hand-written adjoint.  One step = one
sampler proposal: write the 17 parameters, evaluate logL and d(logL)/d(theta),
read them back.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Reported on one JSON line (rank 0):
  value      device-side throughput: K / sum of the per-step device time of
             the evaluation pipeline (CUDA events on the library's stream),
             inputs (data, sigma, PSF) resident in HBM
  e2e        the same metric through the public C ABI call with host buffers:
             parameters in, logL + gradient out, per-step host<->device copies
             inside the timed region (host clock around each synchronous call,
             after a device synchronize; maximum over ranks)
  roofline   the dominant kernel (forward brute-force convolution) against the
             measured FP32 FMA peak of this GPU
  cpu_baseline  the reference's own libprofit C++ (compiled in place, OpenMP on
             all host cores) computing logL + central finite differences
  plain_fp64_fd  this library's plain FP64 form with finite differences, the
             denominator of the FP32-adjoint speed-up target

With --impl reference, rank 0 times the reference CPU implementation on the
same workload and metric; other ranks exit.  With N > 1 every rank runs an
independent replica (the path does not shard across GPUs): value is the
aggregate, timed as the maximum over ranks.
"""
from __future__ import annotations

import argparse
import ctypes
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

METRIC = "LL+grad evals/s, 1 B200: FP32 adjoint vs FP64 plain @rel err≤1e-5"
UNIT = "evals/s"
L2_FLUSH_BYTES = 256 << 20


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--sampler-n", type=int, default=4096,
                    help="proposals per call of the sampler-batch line (smaller for profiling runs)")
    ap.add_argument("--catalogue-n", type=int, default=10000,
                    help="galaxies of the uneven-catalogue line (0 skips it)")
    ap.add_argument("--no-large-field", action="store_true", help="skip the 2000x2000 large-field line")
    return ap.parse_args()


def workload():
    from profit_b200 import workloads as W
    return W.bulge_disk_ps()


def config_dict(wl, n_gpus):
    return {
        "workload": "bulge_disk_ps: 400x400 image, Sersic bulge (nser logU[2,8]) + exponential disk + "
                    "unconvolved Moffat point source, 51x51 Moffat PSF (fwhm 3, con 2.5), brute-force "
                    "convolver, sigma map U[0.5,2], 17-parameter gradient",
        "proposals": "each step a new sampler proposal: params = init + N(0, 0.02|init|)",
        "image": [wl["width"], wl["height"]],
        "psf": list(wl["psf"].shape),
        "n_params": len(wl["grad"]),
        "l2": "flushed by a 256 MiB device write between timed steps (working set ~30 MB < L2)",
        "parallelism": f"replicas x{n_gpus}" if n_gpus > 1 else "single GPU",
    }


# ---------------------------------------------------------------------------
# clocks
# ---------------------------------------------------------------------------

class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.QUERY,
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "samples": len(sm), "reasons": sorted(reasons)}


# ---------------------------------------------------------------------------
# CPU reference (libprofit compiled in place) timing
# ---------------------------------------------------------------------------

def fastest_reference_build(wl, threads, reps=3):
    """The build of the compiled reference that evaluates the workload's model
    fastest on this host, among those it can run (the -O3 -march=x86-64-v4 /
    v3 speed builds and the parity build); one warm-up and `reps` timed
    evaluations each.  Returns (build, {build: seconds per evaluation})."""
    from profit_b200 import workloads as W
    from oracle.pyoracle import RefModel, runnable_reference_builds
    times = {}
    for b in runnable_reference_builds():
        m = W.configure(RefModel(wl["width"], wl["height"], build=b), wl)
        m.set_omp_threads(threads)
        m.set_convolver("brute", threads)
        m.evaluate()
        t0 = time.perf_counter()
        for _ in range(reps):
            m.evaluate()
        times[b] = (time.perf_counter() - t0) / reps
    best = min(times, key=times.get)
    return best, times


def reference_ll_grad(wl, params, image, sigma, threads, n_grad=None, rel_step=1e-7, build="parity"):
    """logL + central FD gradient with the reference's own C++; returns (ll, grad, n_model_evals)."""
    from oracle.pyoracle import RefModel, loglike_norm

    def ll_at(overrides):
        m = RefModel(wl["width"], wl["height"], build=build)
        m.set_magzero(wl["magzero"])
        m.set_psf(wl["psf"])
        m.set_omp_threads(threads)
        m.set_convolver("brute", threads)
        for i, (name, p) in enumerate(params):
            q = dict(p)
            q.update(overrides.get(i, {}))
            m.add_profile(name, **q)
        img, _ = m.evaluate()
        return loglike_norm(image, sigma, img)

    refs = wl["grad"] if n_grad is None else wl["grad"][:n_grad]
    ll0 = ll_at({})
    g = []
    for (pi, k) in refs:
        v = params[pi][1][k]
        h = rel_step * max(abs(v), 1.0)
        g.append((ll_at({pi: {k: v + h}}) - ll_at({pi: {k: v - h}})) / (2 * h))
    return ll0, np.array(g), 1 + 2 * len(refs)


def cpu_baseline(wl, image, sigma, budget_s=15.0):
    """Reference CPU LL+grad evals/s on a bounded sample (rank 0, N=1)."""
    from profit_b200 import workloads as W
    threads = os.cpu_count() or 1
    build, _ = fastest_reference_build(wl, threads)
    t0 = time.perf_counter()
    n_full = 0
    evals = 0
    while True:
        prop = W.perturbed(wl, seed=10_000 + n_full, scale=0.02)
        _, _, ne = reference_ll_grad(wl, prop["profiles"], image, sigma, threads, build=build)
        evals += ne
        n_full += 1
        if time.perf_counter() - t0 > budget_s or n_full >= 20:
            break
    dt = time.perf_counter() - t0
    return {"value": n_full / dt, "unit": UNIT, "cores": threads, "kind": "reference",
            "sample": f"{n_full} LL+grad evaluations ({evals} libprofit model evaluations, central FD over "
                      f"{len(wl['grad'])} parameters) of the same workload, OpenMP {threads} threads, "
                      f"{dt:.1f} s wall, libprofit built {build_flags(build)}"}


def build_flags(build):
    return {"parity": "-O3 -mavx -ffp-contract=off (parity build)",
            "x86-64-v3": "-O3 -march=x86-64-v3 (AVX2+FMA speed build)",
            "x86-64-v4": "-O3 -march=x86-64-v4 (AVX-512 speed build)"}[build]


# ---------------------------------------------------------------------------
# main (B200 arm)
# ---------------------------------------------------------------------------

def max_over_ranks(values, dist=None, device="cpu"):
    """Element-wise maximum over ranks of a list of floats (timed regions are
    reported as the slowest rank's).  With no process group, the values."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return list(values)
    import torch
    t = torch.tensor(list(values), dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


def aggregate_rate(steps, seconds, world):
    """Whole-job throughput of `world` replicas that each ran `steps` steps,
    the slowest taking `seconds`."""
    return world * steps / seconds


def init_dist():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def main_b200(args):
    import torch
    import torch.distributed as dist
    from datetime import timedelta

    world, rank, local = init_dist()
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))

    from profit_b200 import PF_FP32, PF_FP64, Model, _capi
    from profit_b200 import workloads as W

    wl = workload()
    truth_model = W.configure(Model(wl["width"], wl["height"]), wl)
    truth, _ = truth_model.evaluate()
    image, sigma = W.make_data(wl, truth)
    truth_model.close()

    refs = wl["grad"]
    proposals = [W.perturbed(wl, seed=s, scale=0.02) for s in range(args.warmup + args.steps)]
    pvals = [np.array([p["profiles"][i][1][k] for (i, k) in refs]) for p in proposals]

    m = W.configure(Model(wl["width"], wl["height"], precision=PF_FP32), W.perturbed(wl, seed=0, scale=0.02))
    m.set_data(image, sigma)
    L = _capi.lib()
    arr, keep = Model._refs(refs)
    ll = ctypes.c_double()
    grad = np.zeros(len(refs))
    gptr = grad.ctypes.data_as(_capi._dp)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")

    # accuracy of the FP32 adjoint against the plain FP64 form (FD), outside timing
    m.set_parameters(refs, pvals[0])
    m.set_precision(PF_FP64)
    ll_fd, g_fd = m.loglike_grad_fd(refs, rel_step=1e-7)
    _, g_fd6 = m.loglike_grad_fd(refs, rel_step=1e-6)
    m.set_precision(PF_FP32)
    ll_ad, g_ad = m.loglike_grad(refs)
    # FD carries its own error (roundoff of logL over the step, truncation):
    # per component the closer of the two steps is the reference
    g_err = np.minimum(np.abs(g_ad - g_fd), np.abs(g_ad - g_fd6))
    g_rel = g_err / np.abs(g_fd)
    worst = int(np.argmax(g_rel))
    accuracy = {"vs": "plain FP64 form, central FD at rel steps 1e-7 and 1e-6 (the closer per component), "
                      "first proposal, one FP32 evaluation (its cells are added atomically in no fixed order, "
                      "so the worst component moves by a few 1e-6 from one evaluation to the next)",
                "loglike_rel_err": abs(ll_ad - ll_fd) / abs(ll_fd),
                "grad_max_rel_err": float(g_rel.max()), "grad_median_rel_err": float(np.median(g_rel)),
                "grad_worst_component": {"profile": int(refs[worst][0]), "parameter": refs[worst][1],
                                         "abs_over_max_abs_grad": float(abs(g_fd[worst]) / np.max(np.abs(g_fd)))},
                "grad_norm_rel_err": float(np.linalg.norm(g_ad - g_fd) / np.linalg.norm(g_fd)),
                "grad_err_over_max_grad": float(np.max(g_err) / np.max(np.abs(g_fd))),
                "fd_step_spread_max_rel": float(np.max(np.abs(g_fd - g_fd6) / np.abs(g_fd)))}

    # plain FP64 + FD timing (the speed-up target's denominator), a few steps
    m.set_precision(PF_FP64)
    fd_times = []
    for s in range(3 + 5):
        m.set_parameters(refs, pvals[s % len(pvals)])
        m.loglike_grad_fd(refs, rel_step=1e-7)
        if s >= 3:
            fd_times.append(m.last_timings()[0])
    m.set_precision(PF_FP32)
    fp64_fd_value = 1e3 / statistics.mean(fd_times)

    # ctypes argument objects built once (a C caller passes plain pointers;
    # building them per call costs the Python harness ~4 us)
    vptrs = [v.ctypes.data_as(_capi._dp) for v in pvals]
    llref = ctypes.byref(ll)
    nrefs = len(refs)

    # one proposal per call: its 17 values in, logL and the gradient out
    def step(s):
        st = L.pf_model_loglike_grad_batch(m._h, arr, nrefs, 1, vptrs[s], llref, gptr)
        if st != 0:
            raise RuntimeError(L.pf_last_error().decode())

    # the same through libprofit's call pattern: set the parameters, evaluate
    def step_set_parameters(s):
        L.pf_model_set_parameters(m._h, arr, nrefs, vptrs[s])
        st = L.pf_model_loglike_grad(m._h, arr, nrefs, llref, gptr)
        if st != 0:
            raise RuntimeError(L.pf_last_error().decode())

    for s in range(args.warmup):
        step(s)
    torch.cuda.synchronize()

    clocks = ClockSampler(local)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    torch.cuda.nvtx.range_push("timed")
    launches0 = L.pf_kernel_launches()
    dev_ms, e2e_ms, conv_ms, tim = [], [], [], (ctypes.c_float * 4)()
    for s in range(args.warmup, args.warmup + args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        # the call is synchronous: it returns with logL and the gradient in
        # host memory, so the host clock around it is the end-to-end time
        t0 = time.perf_counter()
        step(s)
        e2e_ms.append(1e3 * (time.perf_counter() - t0))
        L.pf_model_last_timings(m._h, tim, 4)
        dev_ms.append(tim[0])
    torch.cuda.synchronize()
    launches = L.pf_kernel_launches() - launches0
    torch.cuda.nvtx.range_pop()
    clk = clocks.stop()
    if world > 1:
        dist.barrier()

    # The forward convolution's own time (the roofline) needs events around
    # it inside the recorded pipeline, which cost each replay a few
    # microseconds: a second timed pass of the same steps with them on.
    L.pf_model_set_phase_timing(m._h, 1)
    for s in range(args.warmup):
        step(s)
    phase_dev_ms = []
    for s in range(args.warmup, args.warmup + args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        step(s)
        torch.cuda.synchronize()
        L.pf_model_last_timings(m._h, tim, 4)
        conv_ms.append(tim[2])
        phase_dev_ms.append(tim[0])
    L.pf_model_set_phase_timing(m._h, 0)
    # end to end through set_parameters + loglike_grad
    for s in range(args.warmup):
        step_set_parameters(s)
    e2e_sp_ms = []
    for s in range(args.warmup, args.warmup + args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        step_set_parameters(s)
        e2e_sp_ms.append(1e3 * (time.perf_counter() - t0))
    e2e_sp_total = max_over_ranks([sum(e2e_sp_ms) / 1e3], dist if world > 1 else None, device="cuda")[0]

    dev_total, e2e_total = max_over_ranks([sum(dev_ms) / 1e3, sum(e2e_ms) / 1e3],
                                          dist if world > 1 else None, device="cuda")

    # roofline of the forward convolution (the dominant kernel)
    P = wl["psf"].shape[0]
    n_out = wl["width"] * wl["height"]
    flop = 2.0 * P * P * n_out
    conv_s = statistics.mean(conv_ms) / 1e3
    peaks = measured_fp32_peak()
    roof = {"kernel": "k_conv3_tile (forward brute-force convolution, packed FP32 FMA, autotuned tile)",
            "bound": "fp32",
            "achieved": flop / conv_s / 1e12, "peak": peaks, "unit": "TFLOP/s",
            "frac": (flop / conv_s / 1e12) / peaks if peaks else None,
            "traffic": recorded_traffic(),
            "algorithmic": f"2*P^2*W*H = {flop:.3e} FLOP per launch (P={P}, W*H={n_out})",
            "peak_source": "measured on this GPU: dependent FP32 FMA chains, plain and packed (FFMA2), the higher "
                           "of the two, libpf_peaks.so, best of 5 (burst); the convolution is FP32-pipe bound, so "
                           "neither the HBM nor the bf16 tensor peak applies",
            "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one forward launch "
                              "(profiles/conv_fwd_bulge_disk_ps.txt)",
            "timing": "CUDA events around the forward convolution inside the recorded pipeline, over a second "
                      f"timed pass of the same {args.steps} steps with those phase events on "
                      f"({statistics.mean(phase_dev_ms):.4f} ms per step there; the headline pass records no "
                      "events inside the pipeline)"}

    render = render_rate(wl, image, sigma, refs, pvals)
    conv_choice = convolver_choice_rate(torch, flush, wl, image, sigma, refs, pvals)
    sampler = sampler_batch_rate(args, torch, flush, n=args.sampler_n)
    catalogue = catalogue_rate(args, torch, flush, n=args.catalogue_n) if args.catalogue_n > 0 else None
    large = None if args.no_large_field else large_field_rate(args, torch, flush)

    out = None
    if rank == 0:
        per_step_in = 8 * len(refs) + 16 * len(refs)  # values + parameter references
        out = {
            "metric": METRIC, "value": aggregate_rate(args.steps, dev_total, world), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dev_total / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic: seeded PCG64 images/sigma/PSF of the configuration's shapes (no public dataset)",
            "config": config_dict(wl, world),
            "e2e": {"value": aggregate_rate(args.steps, e2e_total, world), "unit": UNIT,
                    "h2d_bytes_per_step": 8 * len(refs), "d2h_bytes_per_step": 8 * (1 + len(refs)),
                    "path": "pf_model_loglike_grad_batch with one proposal (C ABI, host buffers: the 17 values "
                            "in, logL and 17 gradient components out)",
                    "ms_per_step": 1e3 * e2e_total / args.steps,
                    "set_parameters_path": {"value": aggregate_rate(args.steps, e2e_sp_total, world), "unit": UNIT,
                                            "path": "pf_model_set_parameters + pf_model_loglike_grad",
                                            "ms_per_step": 1e3 * e2e_sp_total / args.steps}},
            "roofline": roof,
            "gpu_launches": int(launches),
            "clocks": clk,
            # auxiliary lines first, the headline's accuracy and render work last
            "sampler_batch": sampler,
            "catalogue_batch": catalogue,
            "large_field": large,
            "convolver_choice": conv_choice,
            "render": render,
            "plain_fp64_fd": {"value": fp64_fd_value, "unit": UNIT,
                              "speedup_fp32_adjoint": (world * args.steps / dev_total) / fp64_fd_value},
            "accuracy": accuracy,
        }
    m.close()
    if world > 1:
        dist.destroy_process_group()
    if rank == 0:
        if not args.no_cpu_baseline and world == 1:
            out["cpu_baseline"] = cpu_baseline(wl, image, sigma)
        print(json.dumps(out), flush=True)


# Algorithmic cost of one libprofit profile evaluation (evaluate_at) in the
# FP32 form, counted from the profile formulas with box = 0 (render32.cu:
# sersic_tan, moffat_tan, eval_val, tan_to_j): FP32 arithmetic in FLOP (a
# multiply or add 1, a fused multiply-add 2) and transcendental operations
# (exp, log, sqrt, reciprocal: one XU operation each; the FMA-pipe polish
# inside those functions is implementation, not counted).  A "tangent"
# evaluation is the value plus every parameter tangent and its accumulation
# into the nine tangent sums (coordinates 6 FLOP, accumulation 21 FLOP); a
# "test" evaluation is libprofit's second point of a sub-pixel that may still
# recurse (value only, plus the acceptance test).
RENDER_COST = {  # kind: {"tangent": (FLOP, XU), "test": (FLOP, XU)}
    "sersic": {"tangent": (62, 7), "test": (12, 3)},
    "moffat": {"tangent": (59, 8), "test": (11, 3)},
}


def render_work(wl, counts_per_level, max_rec=2):
    """(FLOP, XU ops) of one evaluation of the workload's radial profiles:
    direct pixels and sub-points of the last level are tangent evaluations;
    at a level below max_recursions (2) each sub-point is a tangent and a test
    evaluation (libprofit counts both).  The Sersic centre cusp recurses past
    level 2 at a handful of cells; those are counted as tangent evaluations."""
    flop = xu = 0.0
    for (kind, params), per in zip(wl["profiles"], counts_per_level):
        cost = RENDER_COST.get(kind)
        if cost is None or params.get("box", 0.0) != 0.0 or not per:
            continue
        tf, tx = cost["tangent"]
        sf, sx = cost["test"]
        flop += per[0] * tf
        xu += per[0] * tx
        for lvl, n in enumerate(per[1:]):
            if lvl < max_rec:
                flop += n / 2 * (tf + sf)
                xu += n / 2 * (tx + sx)
            else:
                flop += n * tf
                xu += n * tx
    return flop, xu


def render_rate(wl, image, sigma, refs, pvals, steps=20):
    """Render work of the headline evaluation, outside the timed region:
    libprofit's evaluate_at calls for the first proposal (direct pixels plus
    subsampling points, counted by the plain FP64 form's debug counters, whose
    decisions are the reference's pixel for pixel), over the render phase of
    the FP32 LL+grad pipeline (CUDA events around the pixel and level kernels,
    median over proposals; each evaluation there also forms the profile's
    parameter tangents).  The roofline: the FP32 FLOP and transcendental (XU)
    operations those evaluations need (RENDER_COST) at the measured FP32 FMA
    and XU peaks of this GPU; the slower pipe sets the time.  The render is
    compute bound and its working set is in L2 either way, so no flush here."""
    from profit_b200 import PF_FP32, Model
    from profit_b200 import workloads as W
    try:
        m = W.configure(Model(wl["width"], wl["height"]), wl)
        m.set_parameters(refs, pvals[0])
        m.set_debug(True)
        m.evaluate()
        counts = [m.evaluation_counts(i) for i in range(len(wl["profiles"]))]
        m.set_debug(False)
        m.set_precision(PF_FP32)
        m.set_data(image, sigma)
        m.set_phase_timing(True)  # the render's own events inside the replayed pipeline
        ts = []
        for s in range(3 + steps):
            m.set_parameters(refs, pvals[s % len(pvals)])
            m.loglike_grad(refs)
            if s >= 3:
                ts.append(m.last_timings()[1])
        m.close()
    except Exception as e:  # an auxiliary figure: report, never lose the bench line
        return {"error": str(e)}
    n_eval = int(sum(c[0] for c in counts))
    render_ms = statistics.median(ts)
    flop, xu = render_work(wl, [c[1] for c in counts])
    fp32 = measured_peak(0)   # plain FP32 FMA, TFLOP/s (the render's arithmetic is not packed)
    xu_peak = measured_peak(3)  # Tops/s
    t = render_ms / 1e3
    out = {"evaluations": n_eval, "per_profile": [int(c[0]) for c in counts],
           "per_level": [c[1] for c in counts], "render_ms": render_ms,
           "evaluations_per_s": n_eval / t,
           "definition": "evaluate_at calls of the first proposal (plain FP64 debug counters) over the "
                         f"FP32 render phase (value + parameter tangents per evaluation), median of {steps} "
                         "proposals"}
    if fp32 and xu_peak:
        t_fma, t_xu = flop / (fp32 * 1e12), xu / (xu_peak * 1e12)
        out["roofline"] = {
            "flop": flop, "xu_ops": xu, "fp32_tflops": flop / t / 1e12, "xu_tops": xu / t / 1e12,
            "peak_fp32_tflops": fp32, "peak_xu_tops": xu_peak, "bound": "xu" if t_xu > t_fma else "fp32",
            "frac": max(t_fma, t_xu) / t,
            "cost": "RENDER_COST per evaluation (FLOP, XU) from the profile formulas; peaks measured on this GPU "
                    "(libpf_peaks.so: FP32 FMA chains, fast-exponential chains)"}
    return out


def convolver_choice_rate(torch, flush, wl, image, sigma, refs, pvals, steps=30):
    """The headline workload with the convolver profitSetupData would pick
    when benchmarking (pf_model_benchmark_convolvers: "brute" and "fft" timed
    on the model, the faster kept), timed like the headline: device time of
    the pipeline and the C-ABI call with host buffers, L2 flushed between
    steps."""
    from profit_b200 import PF_FP32, Model, _capi
    from profit_b200 import workloads as W
    m = W.configure(Model(wl["width"], wl["height"], precision=PF_FP32), W.perturbed(wl, seed=0, scale=0.02))
    m.set_data(image, sigma)
    best, ms = m.benchmark_convolvers(nbench=10)
    L = _capi.lib()
    arr, keep = Model._refs(refs)
    ll = ctypes.c_double()
    grad = np.zeros(len(refs))
    gptr = grad.ctypes.data_as(_capi._dp)
    tim = (ctypes.c_float * 4)()
    vptrs = [v.ctypes.data_as(_capi._dp) for v in pvals]
    llref = ctypes.byref(ll)
    dev, e2e = [], []
    torch.cuda.nvtx.range_push("convolver_choice")
    for s in range(steps + 3):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        if L.pf_model_loglike_grad_batch(m._h, arr, len(refs), 1, vptrs[s % len(pvals)], llref, gptr) != 0:
            raise RuntimeError(L.pf_last_error().decode())
        t1 = time.perf_counter()
        if s >= 3:
            e2e.append(t1 - t0)
            L.pf_model_last_timings(m._h, tim, 4)
            dev.append(tim[0] / 1e3)
    torch.cuda.nvtx.range_pop()
    m.close()
    return {"workload": "the headline workload with the benchmark-chosen convolver",
            "benchmark": {"chosen": best, "mean_device_ms": ms, "nbench": 10},
            "value": len(dev) / sum(dev), "unit": UNIT,
            "e2e": {"value": len(e2e) / sum(e2e), "unit": UNIT}}


def sampler_batch_rate(args, torch, flush, n=4096, calls=3):
    """4096 proposals of the single-Sersic model (200x200, 31x31 PSF) per
    call, logL + 8-parameter adjoint gradient; compared with the plain FP64
    form and FD on the same model.  Reported beside the headline metric."""
    from profit_b200 import PF_FP32, PF_FP64, Model
    from profit_b200 import workloads as W
    wl, vals = W.sampler_batch(n)
    refs = wl["grad"]
    m = W.configure(Model(wl["width"], wl["height"]), wl)
    truth, _ = m.evaluate()
    image, sigma = W.make_data(wl, truth)
    m.set_data(image, sigma)
    fd = []
    for s in range(4):
        m.set_parameters(refs, vals[s])
        m.loglike_grad_fd(refs, rel_step=1e-7)
        if s >= 1:
            fd.append(m.last_timings()[0])
    fd_rate = 1e3 / statistics.mean(fd)
    m.set_precision(PF_FP32)
    m.loglike_grad_batch(refs, vals)  # warm-up: tuning, queue sizing, graph capture
    times = []
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.nvtx.range_push("sampler")
    for _ in range(calls):
        flush.zero_()
        torch.cuda.synchronize()
        ev0.record()
        ll, g = m.loglike_grad_batch(refs, vals)
        ev1.record()
        ev1.synchronize()
        times.append(ev0.elapsed_time(ev1) / 1e3)
    torch.cuda.nvtx.range_pop()
    # the same batch with the FFT convolver (the configuration names brute
    # force; reported beside it, as the benchmark-chosen convolver would be)
    m.set_convolver("fft")
    m.loglike_grad_batch(refs, vals)
    fft_times = []
    for _ in range(calls):
        flush.zero_()
        torch.cuda.synchronize()
        ev0.record()
        m.loglike_grad_batch(refs, vals)
        ev1.record()
        ev1.synchronize()
        fft_times.append(ev0.elapsed_time(ev1) / 1e3)
    m.close()
    rate = n / statistics.mean(times)
    return {"workload": "single Sersic 200x200, 31x31 Gaussian PSF, brute force, 8-parameter gradient; "
                        f"{n} proposals init + N(0, 0.05|init|) per call through pf_model_loglike_grad_batch "
                        "(host parameters in, logL + gradients out)",
            "value": rate, "unit": UNIT, "ms_per_call": 1e3 * statistics.mean(times),
            "fft_convolver": {"value": n / statistics.mean(fft_times), "unit": UNIT,
                              "ms_per_call": 1e3 * statistics.mean(fft_times)},
            "plain_fp64_fd_value": fd_rate, "speedup_vs_plain_fp64_fd": rate / fd_rate,
            "finite_fraction": float(np.isfinite(ll).mean())}


def large_field_rate(args, torch, flush, calls=3):
    """2000x2000 field of 200 Sersic components (mag U[14,22], nser logU[0.5,8],
    re logU[1,60]), 101x101 Moffat PSF, FFT convolver; logL + gradient of all
    1600 parameters per evaluation (FP32 adjoint, recomputing form).  The plain
    FP64 form with FD would take 2*1600+1 model evaluations: it is reported as
    that many times one timed FP64 evaluation."""
    from profit_b200 import PF_FP32, Model
    from profit_b200 import workloads as W
    wl = W.large_field()
    m = W.configure(Model(wl["width"], wl["height"]), wl)
    truth, _ = m.evaluate()
    image, sigma = W.make_data(wl, truth)
    m.set_data(image, sigma)
    m.loglike()
    t64 = []
    for _ in range(2):
        m.loglike()
        t64.append(m.last_timings()[0] / 1e3)
    m.close()
    w2 = W.perturbed(wl, seed=1, scale=0.01)
    refs = w2["grad"]
    mm = W.configure(Model(wl["width"], wl["height"], precision=PF_FP32), w2)
    mm.set_data(image, sigma)
    mm.set_phase_timing(True)  # render / convolution / likelihood+adjoint split
    mm.loglike_grad(refs)  # warm-up: FFT plans, queue sizing, graph capture
    dev, wall, phases = [], [], []
    torch.cuda.nvtx.range_push("large_field")
    for _ in range(calls):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ll, g = mm.loglike_grad(refs)
        wall.append(time.perf_counter() - t0)
        t = mm.last_timings()
        dev.append(t[0] / 1e3)
        phases.append(list(t))
    torch.cuda.nvtx.range_pop()
    mm.close()
    fd_s = (2 * len(refs) + 1) * statistics.mean(t64)
    ph = np.mean(np.array(phases), axis=0)
    return {"workload": "large field: 2000x2000, 200 Sersic components, 101x101 Moffat PSF, FFT convolver, "
                        "logL + gradient of all 1600 parameters (FP32 adjoint)",
            "value": 1.0 / statistics.mean(dev), "unit": "LL+grad evals/s", "seconds_per_eval": statistics.mean(dev),
            "wall_seconds_per_eval": statistics.mean(wall), "n_params": len(refs),
            "phases_ms": {"render": float(ph[1]), "convolution": float(ph[2]), "likelihood_and_adjoint": float(ph[3])},
            "plain_fp64_eval_seconds": statistics.mean(t64),
            "plain_fp64_fd_value": 1.0 / fd_s,
            "plain_fp64_fd_note": f"{2 * len(refs) + 1} plain FP64 evaluations at the measured time of one",
            "speedup_vs_plain_fp64_fd": fd_s / statistics.mean(dev),
            "finite": bool(np.isfinite(ll) and np.all(np.isfinite(g)))}


def catalogue_rate(args, torch, flush, n=10000, calls=2, fd_sample=6):
    """Uneven catalogue: n galaxies, side ~ logU[32, 512], odd PSF sides in
    [15, 65], 1-3 components of the six radial kinds, logL + full gradient per
    galaxy through pf_catalogue_loglike_grad.  The data are N(0, 1) noise with
    sigma = 1 (the timing does not depend on the data values).  The plain
    FP64 form with FD gradients is timed on the first fd_sample galaxies."""
    from profit_b200 import PF_FP64, Model
    from profit_b200 import workloads as W
    from profit_b200.catalogue import Catalogue, grad_names
    gals = W.catalogue(n)
    r = np.random.Generator(np.random.PCG64([W.SEED, 93]))
    cat = Catalogue(magzero=gals[0]["magzero"])
    npix = 0
    for g in gals:
        side = g["side"]
        npix += side * side
        cat.add_galaxy(r.normal(size=(side, side)), np.ones((side, side)), g["psf"], g["profiles"])
    _, ngrad = cat.size()
    t0 = time.perf_counter()
    cat.loglike_grad()  # warm-up: uploads, bucketing, convolution tuning
    first_s = time.perf_counter() - t0
    dev, wall = [], []
    torch.cuda.nvtx.range_push("catalogue")
    for _ in range(calls):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ll, _ = cat.loglike_grad()
        wall.append(time.perf_counter() - t0)
        dev.append(cat.last_time_ms() / 1e3)
    torch.cuda.nvtx.range_pop()
    fft_chunks, chunks = cat.convolvers()
    cat.close()
    # plain FP64 + FD on a sample of the same galaxies
    fd_t, fd_n = 0.0, 0
    for g in gals[:fd_sample]:
        side = g["side"]
        m = Model(side, side)
        m.set_magzero(g["magzero"])
        m.set_psf(g["psf"])
        for kind, params in g["profiles"]:
            m.add_profile(kind, convolve=True, **params)
        m.set_data(r.normal(size=(side, side)), np.ones((side, side)))
        refs = [(i, k) for i, (kind, _) in enumerate(g["profiles"]) for k in grad_names(kind)]
        m.set_precision(PF_FP64)
        m.loglike_grad_fd(refs, rel_step=1e-7)
        t0 = time.perf_counter()
        m.loglike_grad_fd(refs, rel_step=1e-7)
        fd_t += time.perf_counter() - t0
        fd_n += 1
        m.close()
    rate = n / statistics.mean(dev)
    fd_rate = fd_n / fd_t if fd_t > 0 else None
    return {"workload": f"uneven catalogue: {n} galaxies, side logU[32,512], odd PSF side in [15,65] (Gaussian or "
                        "Moffat), 1-3 components from sersic/coresersic/moffat/ferrer/king/brokenexp, logL + full "
                        "gradient per galaxy (pf_catalogue_loglike_grad); data N(0,1), sigma 1",
            "value": rate, "unit": "galaxy LL+grad evals/s", "seconds_per_catalogue": statistics.mean(dev),
            "wall_seconds_per_catalogue": statistics.mean(wall), "first_call_seconds": first_s,
            "pixels": npix, "gradient_components": ngrad,
            "batches": {"total": chunks, "fft_convolved": fft_chunks,
                        "choice": "per batch, brute force or FP64 FFTs, the faster timed at the first call"},
            "plain_fp64_fd_value": fd_rate, "plain_fp64_fd_sample": f"first {fd_n} galaxies, host wall clock",
            "speedup_vs_plain_fp64_fd": (rate / fd_rate) if fd_rate else None,
            "finite_fraction": float(np.isfinite(ll).mean())}


_PEAKS = {}


def measured_peak(kind):
    """Peak of this GPU from libpf_peaks.so (best of 5): 0 FP32 FMA, 1 FP64
    FMA, 2 packed FP32 FMA (TFLOP/s), 3 transcendental XU operations
    (Tops/s); None if the probe is unavailable."""
    if kind not in _PEAKS:
        path = os.path.join(ROOT, "profit_b200", "lib", "libpf_peaks.so")
        try:
            lib = ctypes.CDLL(path)
            lib.pf_peak_fma_tflops.restype = ctypes.c_double
            lib.pf_peak_fma_tflops.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int]
            v = lib.pf_peak_fma_tflops(kind, 4096, 5)
            _PEAKS[kind] = v if v > 0 else None
        except OSError:
            _PEAKS[kind] = None
    return _PEAKS[kind]


def measured_fp32_peak():
    """The FP32 ceiling of the convolution: plain FMA and packed FP32-pair
    FMA, whichever is higher."""
    a, b = measured_peak(0), measured_peak(2)
    vals = [v for v in (a, b) if v]
    return max(vals) if vals else None


def recorded_traffic():
    """DRAM bytes per forward-convolution launch from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "conv_fwd_bulge_disk_ps.txt")
    try:
        for line in open(path):
            if line.startswith("traffic_bytes_per_launch:"):
                return float(line.split(":", 1)[1])
    except OSError:
        pass
    return None


# ---------------------------------------------------------------------------
# reference arm
# ---------------------------------------------------------------------------

def main_reference(args):
    world, rank, local = init_dist()
    if rank != 0:
        return
    from profit_b200 import workloads as W
    from oracle.pyoracle import RefModel
    wl = workload()
    threads = os.cpu_count() or 1
    build, build_times = fastest_reference_build(wl, threads)
    # data from the reference itself at the truth
    m = W.configure(RefModel(wl["width"], wl["height"], build=build), wl)
    m.set_omp_threads(threads)
    m.set_convolver("brute", threads)
    truth, _ = m.evaluate()
    image, sigma = W.make_data(wl, truth)
    n_all = len(wl["grad"])
    # per-step sample: logL + FD over n_grad parameters, sized to ~2 min total
    t0 = time.perf_counter()
    reference_ll_grad(wl, W.perturbed(wl, seed=0, scale=0.02)["profiles"], image, sigma, threads, n_grad=1,
                      build=build)
    per_eval = (time.perf_counter() - t0) / 3
    budget = 120.0
    total_steps = args.warmup + args.steps
    n_grad = int(max(1, min(n_all, ((budget / total_steps) / per_eval - 1) / 2)))
    times = []
    for s in range(total_steps):
        prop = W.perturbed(wl, seed=s, scale=0.02)
        t = time.perf_counter()
        _, _, ne = reference_ll_grad(wl, prop["profiles"], image, sigma, threads, n_grad=n_grad, build=build)
        dt = time.perf_counter() - t
        if s >= args.warmup:
            times.append(dt * (1 + 2 * n_all) / ne)   # scaled to a full LL+grad
    per_full = statistics.mean(times)
    value = 1.0 / per_full
    sample = (f"each step: logL + central FD over {n_grad} of {n_all} parameters "
              f"({1 + 2 * n_grad} libprofit evaluations), time scaled by {1 + 2 * n_all}/{1 + 2 * n_grad} "
              f"to a full LL+grad; OpenMP {threads} threads, brute-force convolver; libprofit built "
              f"{build_flags(build)}, the fastest on this host of "
              + ", ".join(f"{b} {1e3 * t:.1f} ms" for b, t in build_times.items()) + " per model evaluation")
    out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": 1e3 * per_full, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "impl": "reference",
           "data": "synthetic: seeded PCG64 images/sigma/PSF of the configuration's shapes (no public dataset)",
           "config": config_dict(wl, 1),
           "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference", "sample": sample},
           "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    a = parse_args()
    if a.impl == "reference":
        main_reference(a)
    else:
        main_b200(a)
