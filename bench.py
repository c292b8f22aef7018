"""Benchmark of the spectral relaxation step (pfc-relax's hot path) on B200.

Workload (default): the two-component lateral heterostructure at 4096 x 4096
(U = 2, conserved dynamics, dt = 0.25, epsilon_01 smoothed-density coupling,
4% lattice mismatch), seeded synthetic initial state of alternating 512-wide
stripes plus noise. A step is one semi-implicit (ETD1) step of all fields:
x-pass (c2r, nonlinear term, r2c along x) and y-pass (FFT along y, coupling
and update, inverse FFT along y). The working set (spectral state + mixed
workspace, 268 MB in FP32) is larger than L2 (126 MB), so no L2 flush is
needed between timed steps.

    python bench.py [--gpus N --steps K --warmup W] [--precision fp32|fp64]
    python bench.py --impl reference   # the reference solver's CPU step

Multi-GPU: one process per GPU (torchrun), each rank relaxes its own replica
(independent seeds, no collective in the data path): weak scaling. The time is
the max over ranks of the device-timed region.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from pfc_b200 import lib, nfile, synth  # noqa: E402
from pfc_b200 import params as P  # noqa: E402

METRIC = "steps/s & time-to-relaxed at 4096² 2-comp, FP32/warm-start vs plain FP64 on 1 B200"
PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM = 6650.0


def workload(N: int, rank: int):
    """Parameters, box and initial fields of the heterostructure workload."""
    pd = P.hetero_2c(0.04)
    dx = dy = 0.7
    a0 = 7.2552
    f = synth.stripes2(N, N, dx, dy, 512 if N >= 2048 else max(N // 8, 8), (0.3, -0.3), (0.3, 0.3),
                       (a0, a0 * 1.04), 0.02, 1000 + rank)
    return pd, dx, dy, f


def reduce_max(x: float, dist=None, device="cpu") -> float:
    """Max of x over the ranks of the process group (x itself without one)."""
    if dist is None:
        return x
    import torch

    t = torch.tensor([x], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(steps: int, seconds_max: float, world: int) -> float:
    """Whole-job steps/s of `world` independent replicas that each took `steps`
    steps, timed as the slowest rank (weak scaling)."""
    return steps * world / seconds_max


def hbm_peak():
    try:
        with open(PEAKS) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM, "fallback"


class Clocks:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.out = None

    def __enter__(self):
        try:
            self.out = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.out, stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.out.flush()
        rows = []
        with open(self.out.name) as fh:
            for line in fh:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 8:
                    rows.append(parts)
        os.unlink(self.out.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        reasons = sorted({names[i] for r in rows for i in range(4) if r[4 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def traffic_from_profiles(kernel: str, workload_name: str):
    """DRAM bytes per launch from the committed ncu summary, if one exists for this workload."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(p) as fh:
            d = json.load(fh)
        return d.get(workload_name, {}).get(kernel)
    except Exception:
        return None


def cpu_baseline(N: int, U: int, rank: int, steps: int, warmup: int = 1, case=None):
    """The reference solver's step (demos/honey/pfc-relax.c over the project FFT
    shim, all host threads) timed on a bounded sample of the same workload:
    `warmup` untimed steps, then `steps` timed ones. case = (parameter dict,
    dx, dy, fields, dt, c) replaces the heterostructure workload."""
    exe = os.path.join(ROOT, "oracle", "_ref", "pfc-relax-bench")
    if not os.path.exists(exe):
        return None
    if case is None:
        pd, dx, dy, f = workload(N, rank)
        dt, c = 0.25, 1.0
    else:
        pd, dx, dy, f, dt, c = case
    with tempfile.TemporaryDirectory() as d:
        ins = ["in%d.n" % u for u in range(U)]
        for u in range(U):
            nfile.write_n_header_only(os.path.join(d, ins[u]), N, N, dx, dy)
        nfile.write_input(os.path.join(d, "x.in"), ins, ["o%d" % u for u in range(U)], Tprint=10 ** 9,
                          Twrite=10 ** 9, params=pd, c=c, tend=10 ** 6, dx=dx, dy=dy, dt=dt)
        np.ascontiguousarray(f, dtype="<f8").tofile(os.path.join(d, "fields.bin"))
        env = dict(os.environ)
        threads = os.cpu_count() or 1
        env["OMP_NUM_THREADS"] = str(threads)
        r = subprocess.run([exe, "x.in", "fields.bin", str(warmup), str(steps)], cwd=d, capture_output=True,
                           text=True, env=env, timeout=900)
        if r.returncode != 0:
            return {"error": r.stderr[-300:]}
        res = json.loads(r.stdout.strip().splitlines()[-1])
    return {"value": res["steps"] / res["seconds"], "unit": "steps/s", "cores": res["threads"],
            "kind": "reference",
            "sample": "%d steps of %dx%d U=%d after %d warm-up steps; reference step() over the project FFT shim "
                      "(not FFTW), %d OpenMP threads in the FFT, pointwise loops single-threaded"
                      % (res["steps"], N, N, U, warmup, res["threads"])}


def config_cases():
    """The single-field configurations beside the headline: C1 (512^2 honeycomb
    from noise, dt = 1) and C2 (2048^2 32-grain polycrystal, dt = 1), both
    with dx = dy = pi/4; (name, N, parameter dict, dx, fields, dt, c)."""
    pd = P.honeycomb_1c(-0.25)
    dx = math.pi / 4
    return [("c1_honeycomb_512", 512, pd, dx, synth.noise_state(512, 512, 0.25, 0.05, 0)[None], 1.0, 1.0),
            ("c2_polycrystal_2048", 2048, pd, dx, synth.polycrystal(2048, 2048, dx, dx, 32, 0.25, -0.4, 0.01, 0)[None],
             1.0, 1.0)]


def configs_record(steps: int, warmup: int, cpu: bool) -> dict:
    """Steps/s of C1 and C2 on the GPU in both precisions (CUDA events on the
    handle's stream), and the reference's CPU step on bounded samples."""
    import torch

    out = {}
    for name, N, pd, dx, f0, dt, c in config_cases():
        params = P.make_params(pd, c, dt)
        rec = {"grid": [N, N], "U": 1}
        for prec in ("fp32", "fp64"):
            with lib.Relaxation(params, N, N, dx, dx, prec) as r:
                r.upload(f0)
                r.step(warmup)
                st = torch.cuda.ExternalStream(r.stream)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                torch.cuda.synchronize()
                e0.record(st)
                r.step(steps)
                e1.record(st)
                torch.cuda.synchronize()
                rec[prec + "_steps_per_s"] = steps * 1000.0 / e0.elapsed_time(e1)
        if cpu:
            k = 20 if N <= 512 else 5
            cb = cpu_baseline(N, 1, 0, k, 1, case=(pd, dx, dx, f0, dt, c))
            if cb and "error" not in cb:
                rec["reference_cpu_steps_per_s"] = cb["value"]
                rec["reference_cpu_sample"] = cb["sample"]
        out[name] = rec
    return out


def batch_problems(seed: int = 7, n: int = 96):
    """Heterogeneous batch: sizes uniform over {256, 384, 512, 768, 1024, 1536}^2,
    U in {1, 2}, seeded states; 8 problems are box-size scalings 0.98-1.02 of one
    state (the trial sizes of a box optimisation)."""
    sizes = (256, 384, 512, 768, 1024, 1536)
    u = synth.uniform(seed, 2 * n, stream=9)
    p1 = P.make_params(P.honeycomb_1c(-0.25), 1.0, 1.0)
    p2 = P.make_params(P.hetero_2c(0.04), 1.0, 0.25)
    out = []
    for i in range(n - 8):
        N = sizes[int(u[2 * i] * len(sizes))]
        U = 1 + int(u[2 * i + 1] * 2)
        if U == 1:
            out.append((p1, N, N, math.pi / 4, math.pi / 4, synth.noise_state(N, N, 0.25, 0.05, seed * 1000 + i)[None]))
        else:
            f = synth.stripes2(N, N, 0.7, 0.7, max(N // 8, 8), (0.3, -0.3), (0.3, 0.3), (7.2552, 7.2552 * 1.04), 0.02,
                               seed * 1000 + i)
            out.append((p2, N, N, 0.7, 0.7, f))
    base = synth.noise_state(512, 512, 0.25, 0.05, seed * 1000 + 999)[None]
    for k in range(8):
        sc = 0.98 + 0.04 * k / 7
        out.append((p1, 512, 512, math.pi / 4 * sc, math.pi / 4 * sc, base))
    return out


def batch_record(steps: int, warmup: int) -> dict:
    """Config C4: aggregate grid-point updates/s of the batched launch (two
    kernels per step for each class of problems of one size and field count,
    the classes side by side, steps captured in one CUDA graph) against the
    same problems relaxed one after another through their own handles. Both
    timed with CUDA events on their streams around `steps` steps after
    `warmup` untimed ones."""
    import torch

    probs = batch_problems()
    upd = sum(p[0].U * p[1] * p[2] for p in probs)
    res = {}
    with lib.Batch([p[:5] for p in probs], "fp32", autotune=True) as b:
        for prob, p in zip(b.problems, probs):
            prob.upload(p[5])
        b.step(warmup)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        st = torch.cuda.ExternalStream(b.stream)
        e0.record(st)
        b.step(steps)
        e1.record(st)
        torch.cuda.synchronize()
        dt = e0.elapsed_time(e1) * 1e-3
        res["batched"] = {"updates_per_s": upd * steps / dt, "ms_per_step": dt / steps * 1e3,
                          "kernel_launches_per_step": b.launches(1)[0], "graph_launches_per_call": 1}
        rs = [lib.Relaxation(*p[:5], "fp32") for p in probs]
    for r, p in zip(rs, probs):
        r.autotune(5)
        r.upload(p[5])
        r.step(warmup)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for r in rs:
        r.step(steps)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    res["sequential"] = {"updates_per_s": upd * steps / dt, "ms_per_step": dt / steps * 1e3,
                         "kernel_launches_per_step": 2 * len(probs),
                         "timing": "wall clock around the 96 handles' calls, one after another"}
    for r in rs:
        r.close()
    res.update(problems=len(probs), points_x_fields_per_step=upd, steps=steps, warmup=warmup,
               speedup_vs_sequential=res["batched"]["updates_per_s"] / res["sequential"]["updates_per_s"],
               unit="grid-point updates/s")
    return res


def run_batch(args):
    """--batch: the C4 line on its own."""
    res = batch_record(args.steps, args.warmup)
    line = {"metric": "batched relaxation, aggregate grid-point updates/s (96 problems, sizes 256-1536, U 1-2)",
            "value": res["batched"]["updates_per_s"], "unit": "grid-point updates/s", "higher_is_better": True,
            "steps": args.steps, "warmup": args.warmup, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "batch96_mixed", "problems": res["problems"],
                       "points_x_fields_per_step": res["points_x_fields_per_step"]},
            "batched": res["batched"], "sequential": res["sequential"],
            "speedup_vs_sequential": res["speedup_vs_sequential"]}
    print(json.dumps(line))


def run_reference(args, rank, world):
    """--impl reference: the reference's CPU implementation of the step."""
    if rank != 0:
        return
    N, U = args.size, 2
    # the same step and warm-up counts as the GPU arm, bounded so that the run
    # stays within about a minute of host time at 4096^2
    steps = max(1, min(args.steps, args.ref_max_steps))
    warm = max(1, min(args.warmup, 10))
    per = []
    for _ in range(max(1, args.reps)):
        cb = cpu_baseline(N, U, rank, steps, warm)
        if cb is None or "error" in cb:
            print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/pfc-relax-bench missing or failed: %s"
                              % (cb or {}).get("error", "not built")}))
            return
        per.append(cb)
    v = statistics.median(c["value"] for c in per)
    cb = per[0]
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "steps/s", "n_gpus": world,
            "steps": steps, "warmup": warm, "ms_per_step": 1000.0 / v, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "hetero2c_%dx%d" % (N, N), "U": U, "grid": [N, N], "dt": 0.25, "dynamics": "conserved",
                       "precision": "fp64 (the reference's only precision)", "parallelism": "one process",
                       "l2": "inputs larger than L2"},
            "cpu_baseline": {"value": v, "unit": "steps/s", "cores": cb["cores"], "kind": "reference",
                             "sample": cb["sample"]},
            "e2e": {"value": v, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def accuracy_profile(params, N, dx, dy, f0, marks=(10, 100, 300)):
    """FP32 against FP64 from the same initial state at fixed step counts:
    relative difference of <f> and max |psi_fp32 - psi_fp64| over the grid."""
    out = []
    with lib.Relaxation(params, N, N, dx, dy, "fp32") as a, lib.Relaxation(params, N, N, dx, dy, "fp64") as b:
        a.upload(f0)
        b.upload(f0)
        done = 0
        for m in marks:
            a.step(m - done)
            b.step(m - done)
            done = m
            fa, fb = a.evaluate()[0], b.evaluate()[0]
            da = float(np.abs(a.download() - b.download()).max())
            out.append({"steps": m, "rel_dF": abs(fa - fb) / abs(fb), "max_dpsi": da})
    return out


def run_ttr(args):
    """Time to relaxed on the 4096^2 two-field workload: steps until the mean
    free energy changes by less than 1e-9 per step over a 100-step window, with
    the box optimised every 100 steps (the heterostructure configuration's box
    optimisation), and the wall time of the whole run (every step, evaluation
    and optimisation, and for the warm start the network's tiled application).
    Arms from the same initial state: the plain FP64 iteration (the reference
    precision), the same from the initial state moved by one ulp (the control:
    how far two FP64 runs end apart), the plain FP32 iteration, and FP32 with the
    learned warm start (the network's input step of plain steps, the network,
    then the plain finish). Creating the network and loading its weights is
    reported apart, as set-up."""
    lib.set_device(0)
    N = args.size
    reps = []
    for _ in range(max(1, args.ttr_reps)):
        reps.append(ttr_arms(N, args.ttr_max_steps, args.ttr_topt, args.ttr_warm_at))
    arms = ttr_median(reps)
    first_warm = [k for k in arms if k.startswith("warm_fp32")][0]
    line = {"metric": "time to relaxed (|d<f>|/step < 1e-9), %dx%d two-field heterostructure" % (N, N),
            "value": arms[first_warm]["seconds"], "unit": "s", "higher_is_better": False,
            "dtype": "f32", "data": "synthetic", "n_gpus": 1,
            "config": {"workload": "hetero2c_%dx%d" % (N, N), "criterion": "|<f>(t) - <f>(t-100)| / 100 < 1e-9",
                       "evaluate_every": 100, "box_optimisation_every": args.ttr_topt, "repeats": len(reps)},
            "arms": arms, "repeats": reps if len(reps) > 1 else None}
    print(json.dumps(line))


def ttr_median(reps):
    """Per arm, the repeat with the median time (all fields of that repeat)."""
    if len(reps) == 1:
        return reps[0]
    out = {}
    for name in reps[0]:
        runs = sorted((r[name] for r in reps), key=lambda a: a["seconds"])
        out[name] = dict(runs[len(runs) // 2], seconds_all=[a["seconds"] for a in runs])
    return out


TTR_TOL = 1e-9
TTR_EVERY = 100


def ttr_arms(N: int, max_steps: int, Topt: int = 100, warm_at=None) -> dict:
    """The time-to-relaxed arms (see run_ttr) on the N x N workload. With
    warm_at, only warm-started FP32 arms, the network applied after each of
    those numbers of plain steps (the plain FP64 arm runs too, as the
    reference end state)."""
    import torch

    from pfc_b200 import fno

    pd, dx, dy, f0 = workload(N, 0)
    params = P.make_params(pd, 1.0, 0.25)
    # the control: every initial value moved up by one unit in the last place
    f0_ulp = np.nextafter(f0, np.inf)
    arms = {}
    plan = (("plain_fp64", "fp64", False, f0), ("control_fp64_1ulp", "fp64", False, f0_ulp),
            ("plain_fp32", "fp32", False, f0), ("warm_fp32", "fp32", True, f0))
    if warm_at:
        plan = (("plain_fp64", "fp64", False, f0),) + tuple(("warm_fp32_at_%d" % t, "fp32", t, f0) for t in warm_at)
    for name, prec, warm, state in plan:
        r = lib.Relaxation(params, N, N, dx, dy, prec)
        r.upload(state)
        rec = {}
        net = None
        if warm is not False:
            t0 = time.perf_counter()
            meta = fno.weights_meta()
            net = fno.Network(meta["tile"], 32)
            net.set_params(fno.load_weights())
            torch.cuda.synchronize()
            rec["setup_s"] = time.perf_counter() - t0
            rec["weights"] = {k: meta[k] for k in ("tile", "input_step", "horizon", "pairs", "epochs", "val_mse",
                                                   "identity_mse") if k in meta}
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        pre = 0
        d = 1e-4
        if warm is not False:
            # the network's input is the state after its input step of plain FP32 steps
            pre = int(meta.get("input_step", 0)) if warm is True else int(warm)
            for t in range(0, pre, TTR_EVERY):
                r.step(TTR_EVERY)
                if Topt > 0 and (t + TTR_EVERY) % Topt == 0:
                    d = r.optimize(1, 1, d)
            t1 = time.perf_counter()
            r.warmstart(net)
            torch.cuda.synchronize()
            rec["network_s"] = time.perf_counter() - t1
            rec["f_after_network"] = r.evaluate()[0]
        steps, fave, _ = r.relax_until(TTR_TOL, TTR_EVERY, max_steps, Topt=Topt, d=d)
        rec.update(seconds=time.perf_counter() - t0, steps=None if steps is None else steps + pre, fave=fave,
                   relaxed=steps is not None, plain_steps_before_network=pre, box=list(r.box()))
        arms[name] = rec
        r.close()
        if net:
            net.close()
    f64 = arms["plain_fp64"]
    for rec in arms.values():
        rec["rel_dF_vs_plain_fp64"] = abs(rec["fave"] - f64["fave"]) / abs(f64["fave"])
        rec["rel_dbox_vs_plain_fp64"] = max(abs(a - b) / b for a, b in zip(rec["box"], f64["box"]))
        rec["speedup_vs_plain_fp64"] = f64["seconds"] / rec["seconds"]
    return arms


def run_fno_train(B: int, iters: int):
    """One training iteration of the warm-start network (loss and gradients,
    then an Adam step) on B random 512^2 two-field tiles, after two untimed
    iterations; CUDA-synchronised wall time."""
    import torch

    from pfc_b200 import fno

    with fno.Network(512, B) as net:
        net.set_params(fno.init_params(0))
        g = torch.Generator(device="cuda").manual_seed(0)
        x = torch.randn((B, 2, 512, 512), device="cuda", dtype=torch.float32, generator=g) * 0.3
        t = x + 0.01 * torch.randn(x.shape, device="cuda", dtype=torch.float32, generator=g)
        torch.cuda.synchronize()
        for _ in range(2):
            net.loss_grad(x.data_ptr(), t.data_ptr(), B)
            net.adam_step(1e-4)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(iters):
            net.loss_grad(x.data_ptr(), t.data_ptr(), B)
            net.adam_step(1e-4)
        torch.cuda.synchronize()
        dt = (time.perf_counter() - t0) / iters
    print(json.dumps({"metric": "warm-start network training iteration (512^2 tiles)", "value": dt * 1e3,
                      "unit": "ms", "higher_is_better": False, "tiles": B, "iters": iters,
                      "ms_per_tile": dt * 1e3 / B, "data": "synthetic"}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    ap.add_argument("--size", type=int, default=4096)
    ap.add_argument("--cpu-steps", type=int, default=6, help="reference steps in the CPU sample of the GPU arm")
    ap.add_argument("--ref-max-steps", type=int, default=60, help="cap on the steps of --impl reference")
    ap.add_argument("--reps", type=int, default=1)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64 comparison run")
    ap.add_argument("--no-cufft", action="store_true", help="skip the cuFFT reference timing")
    ap.add_argument("--batch", action="store_true", help="the batched workload (96 mixed problems) instead")
    ap.add_argument("--no-batch", action="store_true", help="leave the batched workload out of the default line")
    ap.add_argument("--no-configs", action="store_true", help="leave the C1/C2 timings out of the default line")
    ap.add_argument("--batch-steps", type=int, default=200, help="timed steps of the batch record")
    ap.add_argument("--ttr", action="store_true", help="time to relaxed: plain FP64, plain FP32, warm-started FP32")
    ap.add_argument("--ttr-max-steps", type=int, default=80000)
    ap.add_argument("--ttr-topt", type=int, default=100, help="box optimisation period of the time-to-relaxed arms")
    ap.add_argument("--ttr-reps", type=int, default=1, help="repeats of the time-to-relaxed arms (median reported)")
    ap.add_argument("--ttr-warm-at", type=int, nargs="+", default=None, metavar="T0",
                    help="with --ttr: only warm-started arms, the network applied after T0 plain steps")
    ap.add_argument("--no-ttr", action="store_true", help="leave the time-to-relaxed arms out of the default line")
    ap.add_argument("--fno-train", type=int, default=0, metavar="B",
                    help="time one warm-start network training iteration on B tiles of 512^2 instead")
    ap.add_argument("--fno-iters", type=int, default=10)
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.batch:
        lib.set_device(local)
        run_batch(args)
        return
    if args.fno_train:
        lib.set_device(local)
        run_fno_train(args.fno_train, args.fno_iters)
        return
    if args.ttr:
        if rank == 0:
            run_ttr(args)
        return
    if args.warmup < 3:
        args.warmup = 3

    import torch

    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    lib.set_device(local)
    torch.cuda.init()

    N, U = args.size, 2
    pd, dx, dy, f0 = workload(N, rank)
    params = P.make_params(pd, 1.0, 0.25)
    Hspec = (N // 2 + 1) * N

    def timed_steps(r: lib.Relaxation, K: int):
        stream = torch.cuda.ExternalStream(r.stream)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        l0 = r.launches
        e0.record(stream)
        r.step(K)
        e1.record(stream)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        ms = reduce_max(e0.elapsed_time(e1), dist, "cuda")
        return ms, r.launches - l0

    results = {}
    precisions = [args.precision] + ([] if args.no_fp64 or args.precision == "fp64" else ["fp64"])
    for prec in precisions:
        r = lib.Relaxation(params, N, N, dx, dy, prec)
        r.upload(f0)
        r.step(args.warmup)
        with Clocks(local) as clk:
            ms, nl = timed_steps(r, args.steps)
        clocks = clk.summary()
        # per-kernel durations (events on the library stream), separate run
        r.set_profiling(True)
        r.step(min(args.steps, 100))
        prof = r.profile()
        r.set_profiling(False)
        fave, nave = r.evaluate()
        results[prec] = dict(ms=ms, launches=nl, clocks=clocks, prof=prof, fave=fave, nave=list(nave), r=r)

    main_p = args.precision
    res = results[main_p]
    ms = res["ms"]
    steps_per_s = aggregate_rate(args.steps, ms * 1e-3, world)
    eb = 4 if main_p == "fp32" else 8
    # algorithmic bytes (complex elements of 2*eb bytes): y-pass reads work and
    # spec, writes spec and work (4 per point); x-pass reads and writes work (2)
    bytes_y = 4 * 2 * eb * U * Hspec
    bytes_x = 2 * 2 * eb * U * Hspec
    prof = res["prof"]
    kx_ms = prof["xpass"][0] / max(prof["xpass"][1], 1)
    ky_ms = prof["ypass"][0] / max(prof["ypass"][1], 1)
    # dominant kernel: the one with the longer time per step
    dom, dom_ms, dom_bytes = ("ypass", ky_ms, bytes_y) if ky_ms >= kx_ms else ("xpass", kx_ms, bytes_x)
    peak, peak_kind = hbm_peak()
    achieved = dom_bytes / (dom_ms * 1e-3) / 1e9
    wl_name = "hetero2c_%dx%d_%s" % (N, N, main_p)

    # end to end through the C ABI with host buffers: upload from pinned host
    # memory, the K steps, the printed energy (device -> host), download
    r = res["r"]
    host_in = torch.from_numpy(np.ascontiguousarray(f0)).pin_memory()
    host_out = torch.empty((U, N, N), dtype=torch.float64).pin_memory()
    hin = host_in.numpy()
    hout = host_out.numpy()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    r.upload(hin)
    r.step(args.steps)
    r.evaluate()
    r.download(hout)
    torch.cuda.synchronize()
    e2e_s = reduce_max(time.perf_counter() - t0, dist, "cuda")
    e2e = {"value": aggregate_rate(args.steps, e2e_s, world), "unit": "steps/s",
           "h2d_bytes_per_step": int(hin.nbytes / args.steps),
           "d2h_bytes_per_step": int((hout.nbytes + 8 * (1 + U)) / args.steps),
           "note": "one relaxation call sequence per run: upload, %d steps, evaluate, download" % args.steps}

    # cuFFT beside the step, as a reference point only: the FFT work of one step
    # (forward r2c and inverse c2r of all U fields) through torch.fft
    cufft = None
    if rank == 0 and not args.no_cufft:
        x = torch.randn((U, N, N), device="cuda", dtype=torch.float32 if main_p == "fp32" else torch.float64)
        for _ in range(3):
            y = torch.fft.irfft2(torch.fft.rfft2(x), s=(N, N))
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(20):
            y = torch.fft.irfft2(torch.fft.rfft2(x), s=(N, N))
        e1.record()
        torch.cuda.synchronize()
        cufft = {"ms_r2c_plus_c2r": e0.elapsed_time(e1) / 20, "what": "torch.fft rfft2 + irfft2 of the U fields (cuFFT)"}
        del x, y

    acc = None
    if rank == 0 and not args.no_fp64 and main_p == "fp32":
        acc = accuracy_profile(params, N, dx, dy, f0)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(N, U, rank, args.cpu_steps)

    line = {
        "metric": METRIC, "value": steps_per_s, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32" if main_p == "fp32" else "f64", "data": "synthetic",
        "config": {"workload": "hetero2c_%dx%d" % (N, N), "U": U, "grid": [N, N], "dt": 0.25, "dynamics": "conserved",
                   "precision": main_p + " FFT/pointwise, fp64 reductions and k=0 mode",
                   "parallelism": "replicas x%d" % world, "l2": "inputs larger than L2 (268 MB working set)"},
        "gpu_launches": res["launches"],
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind,
                     "algorithmic_bytes_per_launch": dom_bytes, "ms_per_launch": dom_ms,
                     "traffic": traffic_from_profiles(dom, wl_name),
                     "step_frac": (bytes_x + bytes_y) / (ms / args.steps * 1e-3) / 1e9 / peak},
        "kernels_ms": {"xpass": kx_ms, "ypass": ky_ms},
        "clocks": res["clocks"],
        "e2e": e2e,
        "energy": {"fave": res["fave"], "nave": res["nave"]},
    }
    if "fp64" in results and main_p != "fp64":
        r64 = results["fp64"]
        line["fp64"] = {"steps_per_s": args.steps * 1000.0 / r64["ms"] * world, "ms_per_step": r64["ms"] / args.steps,
                        "fave": r64["fave"], "rel_dF_vs_fp32": abs(res["fave"] - r64["fave"]) / abs(r64["fave"])}
    if acc:
        line["accuracy_fp32_vs_fp64"] = acc
    if rank == 0 and world == 1 and not args.no_configs and main_p == "fp32":
        line["configs"] = configs_record(max(args.steps, 50), max(3, args.warmup), not args.no_cpu)
    if rank == 0 and world == 1 and not args.no_batch and main_p == "fp32":
        line["batch"] = batch_record(args.batch_steps, max(3, args.warmup))
    if rank == 0 and world == 1 and not args.no_ttr and main_p == "fp32":
        for v in results.values():
            v["r"].close()
        results = {}
        line["time_to_relaxed"] = {"criterion": "|<f>(t) - <f>(t-100)| / 100 < 1e-9, <f> every 100 steps",
                                   "box_optimisation_every": args.ttr_topt,
                                   "unit": "s (wall, whole run)",
                                   "arms": ttr_arms(N, args.ttr_max_steps, args.ttr_topt)}
    if cpu:
        line["cpu_baseline"] = cpu
    if cufft:
        line["cufft_reference"] = cufft
    if rank == 0:
        print(json.dumps(line))
    for v in results.values():
        v["r"].close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
