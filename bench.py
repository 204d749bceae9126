#!/usr/bin/env python
"""Gradient evaluations per second of the clinical field (forward dose + plan loss + adjoint).

Workload: water, 128^3 voxels of 2 mm, 41x41 spots at 2.5 mm x 40 layers (67,240 pencil
beams), ranges 60-160 mm, SOBP-like float32 weights (seed 1); loss L = sum m (D - P)^2
with a 60 mm target cube at 110 mm depth and a 20 mm shell; gradients wrt all weights
and the 40 per-layer range shifts.  One step = one gradient evaluation.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU (torchrun, one rank per GPU): every rank evaluates its own copy of the field
(independent gradient evaluations, e.g. robust scenarios): weak scaling, no collective
on the data path; the job time is the max over ranks.
"""
from __future__ import annotations

import argparse
import ctypes
import importlib
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "fwd+adjoint dose-gradient evals/s, 67,240 spots/128\u00b3 voxels vs plain fwd @\u22641e-6"
UNIT = "grad_evals/s"
CREDITED_NOTE = ("credited FLOPs = 2*sum over (layer,slice) pairs with IDD != 0 of "
                 "(nsx*nsy*ny + nx*nsx*ny), forward and W-adjoint each")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default=None,
                    help="fp32 | fp16x3 | tf32x3 | bf16x3 | tf32 | bf16; the clinical workload "
                    "defaults to fp16x3 (tcgen05, <= 1e-6 of max against FP64)")
    ap.add_argument("--cpu-budget-s", type=float, default=20.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-side-legs", action="store_true",
                    help="skip the plain-forward, same-box GPU baseline, robust and precision "
                    "legs of the default line")
    ap.add_argument("--workload", default="clinical",
                    choices=["clinical", "robust", "precision", "optimize", "gamma", "luts",
                             "hetero"],
                    help="clinical: the headline gradient workload; robust: 4 fields x 25 "
                    "scenarios batched; precision: forward error vs FP64 per precision mode; "
                    "optimize: on-device plan-optimisation iterations; gamma: gamma index; "
                    "luts: depth-table builds; hetero: dose in a slab phantom (WED)")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def workload_arrays():
    pb = importlib.import_module("gpu-proton-dose-engine_b200")
    wl = pb.workloads.build_workload(2)
    return pb, wl


def credited_flops(wl, active_pairs):
    nsx, nsy = wl["n_sx"], wl["n_sy"]
    g = wl["grid"]
    per_pair = 2 * (nsx * nsy * g["ny"] + g["nx"] * nsx * g["ny"])
    return per_pair * active_pairs


class ClockSampler:
    """nvidia-smi clock / throttle-reason samples (every 50 ms) while the GPU runs the
    benchmark: from the first warm-up step to the end of the end-to-end leg, so that a
    short timed region still has samples under load."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
            return
        # nvidia-smi takes a moment to start: wait (<= 10 s) for its first sample so that the
        # timed region, which can be well under a second, is covered
        t0 = time.time()
        while time.time() - t0 < 10.0 and self.proc.poll() is None:
            if os.path.getsize(self.path) > 0:
                break
            time.sleep(0.05)

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def blas_threads() -> int:
    """Threads of the BLAS pool NumPy's float64 work ran on (all host cores if unknown)."""
    try:
        from threadpoolctl import threadpool_info
        n = [i.get("num_threads") or 0 for i in threadpool_info() if i.get("user_api") == "blas"]
        if n and max(n) > 0:
            return int(max(n))
    except Exception:
        pass
    return os.cpu_count() or 1


def read_traffic(kernel):
    """Per-launch DRAM bytes of ``kernel`` from the committed ncu summary, if present."""
    path = os.path.join(REPO, "profiles", "traffic_per_launch.txt")
    if not os.path.exists(path):
        return None
    for line in open(path):
        parts = line.split()
        if len(parts) >= 2 and parts[0] == kernel:
            try:
                return float(parts[1])
            except ValueError:
                return None
    return None


def peaks():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return d, "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


# --------------------------------------------------------------------------- CPU port
def cpu_port_grad_eval(wl, tables, torch):
    """One gradient evaluation with the oracle's torch CPU port of the reference engine
    (engines.py:256-274) in float64, autograd for dL/dW and dL/d(idd, sigma), chained
    with the range-derivative tables for dL/dR."""
    from oracle import engine_ref as er
    g = wl["grid"]
    xv = g["ox"] + np.arange(g["nx"]) * g["dx"]
    yv = g["oy"] + np.arange(g["ny"]) * g["dy"]
    xs = (np.arange(wl["n_sx"]) - (wl["n_sx"] - 1) / 2.0) * wl["spot_pitch"]
    ys = (np.arange(wl["n_sy"]) - (wl["n_sy"] - 1) / 2.0) * wl["spot_pitch"]
    w = torch.tensor(wl["weights"], dtype=torch.float64, requires_grad=True)
    idd = torch.tensor(tables["idd"], requires_grad=True)
    sig = torch.tensor(tables["sigma"], requires_grad=True)
    d = er.separable_torch(xv, yv, xs, ys, w, idd, sig)
    loss = er.masked_quadratic_loss(d, tables["mask"], tables["presc"])
    loss.backward()
    gr = (idd.grad * tables["didd"]).sum(1) + (sig.grad * tables["dsig"]).sum(1)
    return {"loss": float(loss), "dose": d.detach(), "grad_w": w.grad, "grad_range": gr}


def cpu_tables(wl):
    from oracle import physics_ref as pr
    import torch
    g = wl["grid"]
    z = g["oz"] + np.arange(g["nz"]) * g["dz"]
    en = pr.layer_energies(wl["n_layers"], wl["r_min"], wl["r_max"])
    idd, sig = pr.layer_luts(z, en)
    h = 0.005
    ip, sp = pr.layer_luts(z, en, range_shift=np.full(len(en), h))
    im, sm = pr.layer_luts(z, en, range_shift=np.full(len(en), -h))
    return {"idd": idd, "sigma": sig, "didd": torch.tensor((ip - im) / (2 * h)),
            "dsig": torch.tensor((sp - sm) / (2 * h)),
            "mask": torch.tensor(wl["mask"], dtype=torch.float64),
            "presc": torch.tensor(wl["presc"], dtype=torch.float64)}


def run_cpu_port(wl, budget_s, max_evals=None, warmup=1):
    import torch
    tables = cpu_tables(wl)
    for _ in range(warmup):
        cpu_port_grad_eval(wl, tables, torch)
    n, t0, last = 0, time.perf_counter(), None
    while True:
        last = cpu_port_grad_eval(wl, tables, torch)
        n += 1
        el = time.perf_counter() - t0
        if (max_evals is not None and n >= max_evals) or (max_evals is None and el >= budget_s):
            break
    return n / el, n, el, torch.get_num_threads(), last


# --------------------------------------------------------------------------- reference arm
def reference_arm(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    pb, wl = workload_arrays()
    import torch
    tables = cpu_tables(wl)
    t0 = time.perf_counter()
    cpu_port_grad_eval(wl, tables, torch)          # first warm-up, also sizes the sample
    t_eval = time.perf_counter() - t0
    steps = max(1, min(args.steps, int(120.0 / max(t_eval, 1e-3))))
    W = max(3, min(args.warmup, 5))                # warm-up evaluations, the first included
    rate, n, el, cores, _ = run_cpu_port(wl, budget_s=0.0, max_evals=steps, warmup=W - 1)
    line = {"impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus,
            "steps": n, "warmup": W, "ms_per_step": 1e3 * el / n,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": wl["name"], "grid": [128, 128, 128], "spots": 67240,
                       "layers": 40, "engine": "torch CPU port of engines.torch_separable "
                       "(per_layer=True) + autograd, float64"},
            "cpu_baseline": {"value": rate, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": f"{n} full gradient evaluations"},
            "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# --------------------------------------------------------------------------- side workloads
def _timed(torch, dev, fn, steps, flush):
    """Mean ms of ``fn`` over ``steps`` calls, CUDA events around each call, L2 flushed
    (256 MiB write) before each one, outside the events."""
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(steps)]
    torch.cuda.synchronize(dev)
    for k in range(steps):
        flush.zero_()
        ev[k][0].record()
        fn()
        ev[k][1].record()
    torch.cuda.synchronize(dev)
    return sum(a.elapsed_time(b) for a, b in ev) / steps


def robust_bench(args):
    """4 uneven fields x 25 setup/range scenarios (100 doses on 128^3) per step.

    Three legs, each timed with L2 flushed between steps: a loop of one plain FP32
    ``pbd_forward`` per job (the per-scenario baseline), the batched forward of every job
    in one persistent launch replayed from a CUDA graph, and the loss gradient of every
    job (``pbd_loss_grad_batch``: one forward and one adjoint launch for all jobs) replayed
    from a CUDA graph."""
    import torch
    pb = importlib.import_module("gpu-proton-dose-engine_b200")
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    prec = args.precision or "fp16x3"
    fields = pb.workloads.robust_fields()
    scen = pb.workloads.robust_scenarios()
    probs = pb.robust.robust_problems(fields)
    sb = pb.robust.ScenarioBatch(probs, scen, precision=prec, device=dev, with_grad=True)
    g = fields[0]["grid"]
    m_np, p_np = pb.workloads.target_loss_arrays(g)
    m = torch.as_tensor(m_np, device=dev)
    p = torch.as_tensor(p_np, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    lib = pb._lib
    K, W = args.steps, max(args.warmup, 3)
    clocks = ClockSampler(0)
    clocks.start()
    for _ in range(W):
        sb.loop_forward("fp32")
    t_loop = _timed(torch, dev, lambda: sb.loop_forward("fp32"), K, flush)
    sb.capture()
    for _ in range(W):
        sb.replay()
    n0 = lib.launch_count()
    t_batch = _timed(torch, dev, sb.replay, K, flush)
    sb.capture_loss_grad(m, p)
    for _ in range(W):
        sb.replay_loss_grad()
    t_grad = _timed(torch, dev, sb.replay_loss_grad, K, flush)
    clk = clocks.stop()
    # graph replays do not pass through the host launch counter: count one replay's kernels
    n1 = lib.launch_count()
    sb.run()
    torch.cuda.synchronize(dev)
    per_batch = lib.launch_count() - n1
    sb.loss_grad_all(m, p)
    torch.cuda.synchronize(dev)
    per_grad = lib.launch_count() - n1 - per_batch
    del n0
    worst = 0.0
    sb.loop_forward("fp32")
    sb.run()
    torch.cuda.synchronize(dev)
    for a, b in zip(sb.doses, sb._loop_doses):
        worst = max(worst, float((a.double() - b.double()).abs().max() / b.double().abs().max()))
    n = sb.n_jobs
    line = {"workload": "robust", "metric": "robust scenario doses/s, 4 fields x 25 scenarios "
            "on 128^3", "value": n * 1e3 / t_batch, "unit": "doses/s", "n_gpus": 1, "steps": K,
            "warmup": W, "ms_per_step": t_batch, "higher_is_better": True, "dtype": prec,
            "data": "synthetic",
            "config": {"workload": "4 fields (21x21x16, 33x33x28, 41x41x40, 51x41x48 spots x "
                       "layers) x 25 scenarios, 128^3 voxels of 2 mm", "jobs": n,
                       "precision": prec, "l2": "flushed between steps"},
            "legs_ms": {"fp32_loop_per_job_forward": t_loop, "batched_forward_graph": t_batch,
                        "batched_loss_grad_graph": t_grad},
            "speedup_batched_vs_fp32_loop": t_loop / t_batch,
            "grad_evals_per_s": n * 1e3 / t_grad,
            "gpu_launches_per_replay": {"batched_forward": per_batch, "loss_grad": per_grad},
            "batched_vs_fp32_loop_max_rel": worst, "clocks": clk}
    print(json.dumps(line), flush=True)
    return 0


def optimize_bench(args):
    """Plan optimisation on the device, every iteration one CUDA-graph replay, L2 flushed
    between iterations (outside the events):

      nominal  projected Adam on the 67,240 spot weights of the 128^3 / 41x41x40 field
               (masked quadratic loss of the 60 mm target cube)
      range    the same plus the 40 per-layer range shifts (tables rebuilt every iteration)
      robust   min-max over 4 fields x 25 scenarios: 100 loss gradients, 4 combinations
               and 4 Adam updates per iteration"""
    import torch
    pb, wl = workload_arrays()
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    prec = args.precision or "fp16x3"
    K, W = args.steps, max(args.warmup, 3)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    prob = pb.model.problem_from_workload(wl)
    m = torch.as_tensor(wl["mask"], device=dev)
    p = torch.as_tensor(wl["presc"], device=dev)
    Adam = pb.optimize.Adam
    clocks = ClockSampler(0)
    clocks.start()
    legs = {}

    def leg(name, opt, steps):
        opt.step(W)
        ms = _timed(torch, dev, lambda: opt.step(1), steps, flush)
        h = opt.history()
        h = h if h.ndim == 1 else h.sum(0)
        legs[name] = {"ms_per_iteration": ms, "iterations_per_s": 1e3 / ms, "iterations": steps,
                      "loss_first": float(h[0]), "loss_last": float(h[-1])}

    n_it = W + K + 1
    plan = pb.engines.DosePlan(prob, tables="device", precision=prec, device=dev)
    leg("nominal", pb.optimize.PlanOptimizer(plan, m, p, adam=Adam(lr=0.01), max_iter=n_it), K)
    plan_r = pb.engines.DosePlan(prob, tables="device", precision=prec, device=dev)
    leg("range", pb.optimize.PlanOptimizer(plan_r, m, p, adam=Adam(lr=0.01),
                                           range_adam=Adam(lr=0.01, lo=-0.5, hi=0.5),
                                           max_iter=n_it), K)
    del plan, plan_r
    fields = pb.workloads.robust_fields()
    sb = pb.robust.ScenarioBatch(pb.robust.robust_problems(fields),
                                 pb.workloads.robust_scenarios(), precision=prec, device=dev,
                                 with_grad=True)
    mr_np, pr_np = pb.workloads.target_loss_arrays(fields[0]["grid"])
    mr = torch.as_tensor(mr_np, device=dev)
    pr_ = torch.as_tensor(pr_np, device=dev)
    kr = max(3, min(K, 20))
    leg("robust_minmax", pb.optimize.RobustOptimizer(sb, mr, pr_, objective="max",
                                                      adam=Adam(lr=0.01), max_iter=W + kr + 1),
        kr)
    clk = clocks.stop()
    nom = legs["nominal"]
    line = {"workload": "optimize", "metric": "plan-optimisation iterations/s (projected Adam "
            "on 67,240 spot weights, 128^3 / 41x41x40)", "value": nom["iterations_per_s"],
            "unit": "iterations/s", "n_gpus": 1, "steps": K, "warmup": W,
            "ms_per_step": nom["ms_per_iteration"], "higher_is_better": True, "dtype": prec,
            "data": "synthetic",
            "config": {"workload": "128^3 / 41x41x40 masked quadratic loss; robust: 4 fields x "
                       "25 scenarios", "precision": prec,
                       "l2": "flushed between iterations (256 MiB write, outside the events)"},
            "legs": legs, "clocks": clk}
    print(json.dumps(line), flush=True)
    return 0


def gamma_bench(args):
    """Gamma index of two doses of the clinical field (128^3, 2 mm; the evaluation has the
    spot lattice moved 1 mm in x and 1 % more weight) at 3 %/3 mm and 2 %/2 mm, and of two
    doses of the 200 x 200 x 256 field of 1 mm voxels at 3 %/3 mm (123 search offsets).  One
    ``GammaPlan.run`` per step (map, mask, statistics and percentiles) replayed from a CUDA
    graph (the eager call's time, host launch work included, is reported beside it), L2
    flushed between steps; the oracle's float64 NumPy gamma index on the host is the CPU
    baseline."""
    import torch
    pb = importlib.import_module("gpu-proton-dose-engine_b200")
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    K, W = args.steps, max(args.warmup, 3)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    clocks = ClockSampler(0)
    clocks.start()
    legs = {}
    pairs = {}
    for cfg in (1, 4):
        wl = pb.workloads.build_workload(cfg)
        prob = pb.model.problem_from_workload(wl)
        plan = pb.engines.DosePlan(prob, tables="device", precision="tf32x3", device=dev)
        ref = plan.forward()
        prob.lattice.x0 += 0.1
        plan2 = pb.engines.DosePlan(prob, tables="device", precision="tf32x3", device=dev)
        ev = plan2.forward(plan2.w * 1.01)
        g = wl["grid"]
        pairs[cfg] = (ref, ev, (g["dz"], g["dy"], g["dx"]))
    cases = [("clinical_3mm_3pct", 1, 3.0, 3.0), ("clinical_2mm_2pct", 1, 2.0, 2.0),
             ("fine_1mm_grid_3mm_3pct", 4, 3.0, 3.0)]
    for name, cfg, dp, dta in cases:
        ref, ev, sp = pairs[cfg]
        spec = pb.gamma.gamma_spec(sp, dose_crit_pct=dp, dta_mm=dta)
        gp = pb.gamma.GammaPlan(ref.shape, spec, device=dev)
        for _ in range(W):
            gp.run(ref, ev)
        ms_eager = _timed(torch, dev, lambda: gp.run(ref, ev), K, flush)
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph):
            gp.run(ref, ev)
        for _ in range(W):
            graph.replay()
        ms = _timed(torch, dev, graph.replay, K, flush)
        st = gp.stats()
        n_vox = ref.numel()
        legs[name] = {"ms": ms, "analyses_per_s": 1e3 / ms, "ms_eager_call": ms_eager,
                      "voxels": n_vox, "voxels_per_s": n_vox * 1e3 / ms,
                      "offsets": st.n_dta_offsets, "pass_rate": st.pass_rate,
                      "gamma_p95": st.gamma_p95, "n_eval": st.n_eval}
    clk = clocks.stop()
    cpu = None
    if not args.no_cpu_baseline:
        from oracle import gamma_ref
        ref, ev, sp = pairs[1]
        r64, e64 = ref.double().cpu().numpy(), ev.double().cpu().numpy()
        t0 = time.perf_counter()
        n = 0
        while n < 3 and (n == 0 or time.perf_counter() - t0 < args.cpu_budget_s):
            gamma_ref.gamma_index(r64, e64, spacing=sp)
            n += 1
        el = time.perf_counter() - t0
        cpu = {"value": n / el, "unit": "analyses/s", "cores": 1, "kind": "port",
               "sample": f"{n} full 128^3 gamma analyses at 3 %/3 mm (NumPy float64)"}
    head = legs["clinical_3mm_3pct"]
    line = {"workload": "gamma", "metric": "gamma analyses/s, 128^3 dose pair at 3 %/3 mm",
            "value": head["analyses_per_s"], "unit": "analyses/s", "n_gpus": 1, "steps": K,
            "warmup": W, "ms_per_step": head["ms"], "higher_is_better": True, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": "gamma index of TF32x3 doses: clinical 128^3 field vs the "
                       "same with the lattice moved 1 mm and +1 % weight; 200x200x256 1 mm "
                       "field likewise", "l2": "flushed between steps"},
            "legs": legs, "cpu_baseline": cpu, "clocks": clk}
    print(json.dumps(line), flush=True)
    return 0


def luts_bench(args):
    """Depth tables of the clinical field (40 layers, 128 depths of 2 mm) built on the device
    by one ``pbd_build_luts`` call -- the per-layer host loop of the reference's model.py
    moved to the device -- replayed from a CUDA graph, L2 flushed between steps: the nominal
    tables alone, and with the +-5 um range variants that give dIDD/dR and dsigma/dR.  The
    CPU baseline is the oracle's NumPy restatement of the reference's loop (one host core)."""
    import torch
    pb, wl = workload_arrays()
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    K, W = args.steps, max(args.warmup, 3)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    g = wl["grid"]
    prob = pb.model.problem_from_workload(wl)
    en = prob.lattice.energies
    legs = {}
    clocks = ClockSampler(0)
    clocks.start()
    for name, fd in (("nominal", 0.0), ("with_range_derivatives", 0.005)):
        tb = pb.physics.TableBuilder(g["nz"], g["oz"], g["dz"], en, fd_step=fd, device=dev)
        tb.build()
        torch.cuda.synchronize(dev)
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph):
            tb.build()
        for _ in range(W):
            graph.replay()
        ms = _timed(torch, dev, graph.replay, K, flush)
        legs[name] = {"ms": ms, "builds_per_s": 1e3 / ms}
    clk = clocks.stop()
    cpu = None
    if not args.no_cpu_baseline:
        from oracle import physics_ref as pr
        z = g["oz"] + np.arange(g["nz"]) * g["dz"]
        e_np = np.asarray(en, dtype=np.float64)
        t0 = time.perf_counter()
        n = 0
        while n < 3 and (n == 0 or time.perf_counter() - t0 < args.cpu_budget_s):
            pr.layer_luts(z, e_np)
            n += 1
        el = time.perf_counter() - t0
        cpu = {"value": n / el, "unit": "builds/s", "cores": 1, "kind": "port",
               "sample": f"{n} nominal 40-layer builds (NumPy float64)"}
    head = legs["nominal"]
    line = {"workload": "luts", "metric": "depth-table builds/s, 40 layers x 128 depths",
            "value": head["builds_per_s"], "unit": "builds/s", "n_gpus": 1, "steps": K,
            "warmup": W, "ms_per_step": head["ms"], "higher_is_better": True, "dtype": "f64",
            "data": "synthetic", "config": {"workload": "clinical field tables (IDD, sigma), "
                                            "40 layers, 60-160 mm ranges, 128 depths of 2 mm",
                                            "l2": "flushed between steps"},
            "legs": legs, "cpu_baseline": cpu, "clocks": clk}
    print(json.dumps(line), flush=True)
    return 0


def hetero_bench(args):
    """The clinical field (128^3, 41x41x40) in a slab phantom -- bone (1.6) from 3 to 5 cm,
    lung (0.25) from 7 to 10 cm on one side: the WED ray trace and the heterogeneous forward
    (activity table, every layer's lateral map from one tensor-core forward launch, then the
    depth doses at the WED) from the plan's depth curves, built once per plan like the homogeneous
    plan's tables and timed as their own leg (wed_curves), each replayed from a CUDA graph, L2
    flushed between steps; the homogeneous forward of the same field beside them, and dL/dW
    of the heterogeneous dose for a dL/dD (one single-layer adjoint per layer).  CPU
    baseline: the oracle's float64 heterogeneous dose."""
    import torch
    pb, wl = workload_arrays()
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    prec = args.precision or "tf32x3"
    K, W = args.steps, max(args.warmup, 3)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    prob = pb.model.problem_from_workload(wl)
    g = prob.grid
    zc = g.oz + np.arange(g.nz) * g.dz
    rho_np = np.ones((g.nz, g.ny, g.nx), dtype=np.float32)
    rho_np[(zc >= 3.0) & (zc < 5.0)] = 1.6
    rho_np[(zc >= 7.0) & (zc < 10.0), :, : g.nx // 2] = 0.25
    rho = torch.as_tensor(rho_np, device=dev)
    wed = torch.empty((g.nz, g.ny, g.nx), dtype=torch.float64, device=dev)
    plan = pb.hetero.WedPlan(prob, precision=prec, device=dev)
    homog = pb.engines.DosePlan(prob, tables="device", precision=prec, device=dev)
    out = torch.empty((g.nz, g.ny, g.nx), dtype=torch.float32, device=dev)
    out_h = torch.empty_like(out)
    gdose = torch.as_tensor(np.random.default_rng(3).standard_normal((g.nz, g.ny, g.nx)),
                            dtype=torch.float32, device=dev)
    clocks = ClockSampler(0)
    clocks.start()

    def trace():
        wed.copy_(pb.hetero.wed_raytrace(rho, g, device=dev))

    def curves():
        pb._lib.call("pbd_build_wed_curves", ctypes.byref(plan.spec), len(prob.lattice.energies),
                     pb._lib.ptr(plan.energies), None, pb._lib.ptr(plan.curves),
                     plan.curves.numel(), pb._lib.stream_handle(dev))

    legs = {}
    for name, fn in (("wed_raytrace", lambda: pb.hetero.wed_raytrace(rho, g, device=dev)),
                     ("wed_curves", curves),
                     ("heterogeneous_forward", lambda: plan.forward(wed, out=out)),
                     ("heterogeneous_adjoint", lambda: plan.adjoint(gdose, wed)),
                     ("heterogeneous_adjoint_with_range",
                      lambda: plan.adjoint(gdose, wed, with_range=True)),
                     ("homogeneous_forward", lambda: homog.forward(out=out_h))):
        trace()
        fn()
        torch.cuda.synchronize(dev)
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph):
            fn()
        for _ in range(W):
            graph.replay()
        legs[name] = {"ms": _timed(torch, dev, graph.replay, K, flush)}
    clk = clocks.stop()
    trace()
    plan.forward(wed, out=out)
    torch.cuda.synchronize(dev)
    cpu = None
    if not args.no_cpu_baseline:
        from oracle import hetero_ref, physics_ref as pr
        t0 = time.perf_counter()
        wr = hetero_ref.wed_ref(rho_np, g.oz, g.dz)
        sig = pr.layer_luts(zc, prob.lattice.energies)[1]
        ref = hetero_ref.dose_ref(g.x, g.y, prob.lattice.spot_x, prob.lattice.spot_y,
                                  prob.lattice.ensure_weights(), prob.lattice.energies, sig, wr)
        el = time.perf_counter() - t0
        d = out.double().cpu().numpy()
        legs["max_rel_err_vs_fp64"] = float(np.max(np.abs(d - ref)) / np.max(np.abs(ref)))
        cpu = {"value": 1.0 / el, "unit": "doses/s", "cores": blas_threads(), "kind": "port",
               "sample": "1 heterogeneous 128^3 dose (NumPy / torch float64, incl. the tables)"}
    head = legs["heterogeneous_forward"]
    line = {"workload": "hetero", "metric": "heterogeneous-medium doses/s, 128^3 / 41x41x40",
            "value": 1e3 / head["ms"], "unit": "doses/s", "n_gpus": 1, "steps": K, "warmup": W,
            "ms_per_step": head["ms"], "higher_is_better": True, "dtype": prec,
            "data": "synthetic", "config": {"workload": "clinical field, bone and lung slabs",
                                            "l2": "flushed between steps"},
            "legs": legs, "cpu_baseline": cpu, "clocks": clk}
    print(json.dumps(line), flush=True)
    return 0


def precision_bench(args):
    """Forward of the 200x200x256 / 61x61x60 field in every precision mode: time per call
    (L2 flushed between calls) and error against the FP64 oracle on the host."""
    import torch
    from oracle import engine_ref as er
    pb = importlib.import_module("gpu-proton-dose-engine_b200")
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    wl = pb.workloads.build_workload(4)
    prob = pb.model.problem_from_workload(wl)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    K, W = args.steps, max(args.warmup, 3)
    base = pb.engines.DosePlan(prob, tables="device", precision="fp32", device=dev)
    idd = base.idd.cpu().numpy()
    sig = base.sigma.cpu().numpy()
    g, L = prob.grid, prob.lattice
    t0 = time.perf_counter()
    ref = er.separable_torch(g.x, g.y, L.spot_x, L.spot_y, wl["weights"], idd, sig,
                              layer_chunk=2).numpy()
    t_ref = time.perf_counter() - t0
    active = base.active_pairs()
    flop = 2 * active * (L.n_sx * L.n_sy * g.ny + g.nx * L.n_sx * g.ny)
    clocks = ClockSampler(0)
    clocks.start()
    modes = {}
    for mode in ("fp32", "fp16x3", "tf32x3", "bf16x3", "tf32", "bf16"):
        plan = base if mode == "fp32" else pb.engines.DosePlan(prob, tables="device",
                                                                precision=mode, device=dev)
        plan.idd, plan.sigma = base.idd, base.sigma
        out = torch.empty(plan.shape, dtype=torch.float32, device=dev)
        for _ in range(W):
            plan.forward(out=out)
        ms = _timed(torch, dev, lambda: plan.forward(out=out), K, flush)
        err = pb.engines.relative_error(out, ref)
        modes[mode] = {"ms": ms, "tflops_credited": flop / (ms * 1e-3) / 1e12,
                       "max_rel_err": err["max_rel_err_global"],
                       "rms_rel_err": err["rms_rel_global"]}
    clk = clocks.stop()
    line = {"workload": "precision", "metric": "forward ms and error vs FP64 oracle per precision "
            "mode", "unit": "ms", "higher_is_better": False, "n_gpus": 1, "steps": K, "warmup": W,
            "data": "synthetic",
            "config": {"workload": wl["name"], "grid": [g.nx, g.ny, g.nz], "spots": L.n_spots,
                       "layers": L.n_layers, "active_pairs": active, "credited_flop": flop,
                       "l2": "flushed between calls",
                       "oracle": f"torch CPU float64 port, {t_ref:.1f} s"},
            "modes": modes, "clocks": clk}
    print(json.dumps(line), flush=True)
    return 0


# --------------------------------------------------------------------------- same-box GPU baseline
def reference_bmm_dose(torch, xv, yv, xs, ys, w, idd, sig):
    """The reference's per-layer batched-matmul dose (engines.py:256-274, layer_chunk=None)
    restated for this GPU: every (layer, slice) Gaussian materialised in HBM, two cuBLAS
    batched matmuls and the sum over layers, in the dtype of ``w`` (float32 = the reference's
    CUDA default; TF32 off, as with allow_tf32=False).  Differentiable (autograd)."""
    nl, nz = idd.shape
    nx, ny, nsx, nsy = xv.numel(), yv.numel(), xs.numel(), ys.numel()
    dx2 = (xv.view(1, 1, -1, 1) - xs.view(1, 1, 1, -1)) ** 2
    dy2 = (yv.view(1, 1, -1, 1) - ys.view(1, 1, 1, -1)) ** 2
    s4 = sig.clamp_min(1e-9).reshape(nl, nz, 1, 1)
    norm = (1.0 / np.sqrt(2.0 * np.pi)) / s4
    gx = (norm * torch.exp(-dx2 / (2.0 * s4 ** 2))).reshape(nl * nz, nx, nsx)
    gy = (norm * torch.exp(-dy2 / (2.0 * s4 ** 2))).reshape(nl * nz, ny, nsy)
    amp = (idd[:, :, None, None] * w[:, None, :, :]).reshape(nl * nz, nsy, nsx)
    t = torch.bmm(amp.transpose(1, 2), gy.transpose(1, 2))
    dl = torch.bmm(gx, t)
    return dl.reshape(nl, nz, nx, ny).sum(0).transpose(1, 2)


def gpu_baseline_leg(torch, dev, pb, wl, plan, flush, steps, ours_fwd_ms, ours_grad_ms, d64):
    """The reference's own CUDA path (its torch_separable: cuBLAS FP32 bmm) timed on this
    B200 in the same process: forward ms, and forward + autograd gradient (dL/dW, dL/dIDD,
    dL/dsigma, chained to dL/dR) evaluations/s, each with its error against the FP64 dose."""
    g = wl["grid"]
    f32 = torch.float32
    xv = torch.as_tensor(g["ox"] + np.arange(g["nx"]) * g["dx"], dtype=f32, device=dev)
    yv = torch.as_tensor(g["oy"] + np.arange(g["ny"]) * g["dy"], dtype=f32, device=dev)
    xs = torch.as_tensor((np.arange(wl["n_sx"]) - (wl["n_sx"] - 1) / 2.0) * wl["spot_pitch"],
                         dtype=f32, device=dev)
    ys = torch.as_tensor((np.arange(wl["n_sy"]) - (wl["n_sy"] - 1) / 2.0) * wl["spot_pitch"],
                         dtype=f32, device=dev)
    idd = plan.idd.to(f32)
    sig = plan.sigma.to(f32)
    didd = plan.didd.to(f32)
    dsig = plan.dsig.to(f32)
    w = plan.w.clone()
    m = torch.as_tensor(wl["mask"], device=dev)
    p = torch.as_tensor(wl["presc"], device=dev)
    old = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        def fwd():
            return reference_bmm_dose(torch, xv, yv, xs, ys, w, idd, sig)

        def grad():
            wq = w.detach().requires_grad_(True)
            iq = idd.detach().requires_grad_(True)
            sq = sig.detach().requires_grad_(True)
            d = reference_bmm_dose(torch, xv, yv, xs, ys, wq, iq, sq)
            r = d - p
            loss = (m * r * r).sum()
            loss.backward()
            gr = (iq.grad * didd).sum(1) + (sq.grad * dsig).sum(1)
            return d, wq.grad, gr
        for _ in range(3):
            fwd()
            grad()
        t_fwd = _timed(torch, dev, fwd, steps, flush)
        t_grad = _timed(torch, dev, grad, steps, flush)
        d = fwd()
        err = float((d.double() - d64).abs().max() / d64.abs().max())
    finally:
        torch.backends.cuda.matmul.allow_tf32 = old
    return {"what": "the reference's torch_separable algorithm (engines.py:256-274: Gaussians "
                    "materialised, two cuBLAS FP32 bmm, sum over layers) restated in bench.py "
                    "and timed on this GPU; gradient by torch autograd",
            "kind": "port", "dtype": "fp32",
            "fwd_ms": t_fwd, "dose_fields_per_s": 1e3 / t_fwd,
            "grad_ms": t_grad, "grad_evals_per_s": 1e3 / t_grad,
            "fwd_max_rel_err_vs_fp64": err,
            "speedup_fwd": t_fwd / ours_fwd_ms, "speedup_grad": t_grad / ours_grad_ms,
            "l2": "flushed between steps"}


def robust_leg(torch, dev, pb, flush, steps, warmup):
    """The 4-field x 25-scenario batch (100 doses of 128^3): the batched forward (FP16x3) in
    one persistent launch replayed from a CUDA graph, against loops of one pbd_forward per job
    in plain FP32 and in FP16x3, and the batched loss gradient of all 100 jobs."""
    fields = pb.workloads.robust_fields()
    scen = pb.workloads.robust_scenarios()
    probs = pb.robust.robust_problems(fields)
    sb = pb.robust.ScenarioBatch(probs, scen, precision="fp16x3", device=dev, with_grad=True)
    m_np, p_np = pb.workloads.target_loss_arrays(fields[0]["grid"])
    m = torch.as_tensor(m_np, device=dev)
    p = torch.as_tensor(p_np, device=dev)
    for _ in range(warmup):
        sb.loop_forward("fp32")
    t_fp32 = _timed(torch, dev, lambda: sb.loop_forward("fp32"), steps, flush)
    for _ in range(warmup):
        sb.loop_forward("fp16x3")
    t_tc = _timed(torch, dev, lambda: sb.loop_forward("fp16x3"), steps, flush)
    loop_doses = [d.clone() for d in sb._loop_doses]
    sb.capture()
    for _ in range(warmup):
        sb.replay()
    t_batch = _timed(torch, dev, sb.replay, steps, flush)
    sb.capture_loss_grad(m, p)
    for _ in range(warmup):
        sb.replay_loss_grad()
    t_grad = _timed(torch, dev, sb.replay_loss_grad, steps, flush)
    torch.cuda.synchronize(dev)
    worst = max(float((a.double() - b.double()).abs().max() / b.double().abs().max())
                for a, b in zip(sb.doses, loop_doses))
    n = sb.n_jobs
    return {"workload": "4 fields (21x21x16, 33x33x28, 41x41x40, 51x41x48 spots x layers) x 25 "
                        "scenarios (setup shifts +-3 mm, range x0.965/1.035, 4 corners), 128^3",
            "jobs": n, "batched_forward_ms": t_batch, "doses_per_s": n * 1e3 / t_batch,
            "precision": "fp16x3 (batch and second loop)",
            "loop_fp32_forward_ms": t_fp32, "loop_fp16x3_forward_ms": t_tc,
            "speedup_vs_fp32_loop": t_fp32 / t_batch, "speedup_vs_fp16x3_loop": t_tc / t_batch,
            "batched_loss_grad_ms": t_grad, "grad_evals_per_s": n * 1e3 / t_grad,
            "batched_vs_fp16x3_loop_max_rel": worst, "l2": "flushed between steps"}


def precision_leg(torch, dev, pb, flush, steps, warmup):
    """The 200x200x256 / 61x61x60 field (223,260 beams) in every precision mode: ms per
    forward and max |D - D64| / max D64 against the FP64 kernel's dose (pbd_forward_f64,
    itself within 1e-12 of the float64 oracle in the tests)."""
    wl = pb.workloads.build_workload(4)
    prob = pb.model.problem_from_workload(wl)
    base = pb.engines.DosePlan(prob, tables="device", precision="fp32", device=dev)
    d64 = base.forward_f64()
    for _ in range(warmup):
        base.forward_f64(out=d64)
    t64 = _timed(torch, dev, lambda: base.forward_f64(out=d64), steps, flush)
    g, L = prob.grid, prob.lattice
    active = base.active_pairs()
    flop = 2 * active * (L.n_sx * L.n_sy * g.ny + g.nx * L.n_sx * g.ny)
    ref_max = float(d64.abs().max())
    modes = {"fp64": {"ms": t64, "tflops_credited": flop / (t64 * 1e-3) / 1e12,
                      "max_rel_err": 0.0}}
    for mode in ("fp32", "fp16x3", "tf32x3", "bf16x3", "tf32", "bf16"):
        plan = base if mode == "fp32" else pb.engines.DosePlan(prob, tables="device",
                                                                precision=mode, device=dev)
        plan.idd, plan.sigma = base.idd, base.sigma
        out = torch.empty(plan.shape, dtype=torch.float32, device=dev)
        for _ in range(warmup):
            plan.forward(out=out)
        ms = _timed(torch, dev, lambda: plan.forward(out=out), steps, flush)
        diff = (out.double() - d64).abs()
        modes[mode] = {"ms": ms, "tflops_credited": flop / (ms * 1e-3) / 1e12,
                       "max_rel_err": float(diff.max()) / ref_max,
                       "rms_rel_err": float(diff.pow(2).mean().sqrt()) / ref_max}
    return {"workload": wl["name"], "active_pairs": active, "credited_flop": flop,
            "reference": "pbd_forward_f64 (FP64 on the CUDA cores)", "modes": modes,
            "l2": "flushed between calls"}


# --------------------------------------------------------------------------- our arm
def main():
    args = parse()
    if args.impl == "reference":
        return reference_arm(args)
    if args.workload == "robust":
        return robust_bench(args)
    if args.workload == "precision":
        return precision_bench(args)
    if args.workload == "optimize":
        return optimize_bench(args)
    if args.workload == "gamma":
        return gamma_bench(args)
    if args.workload == "luts":
        return luts_bench(args)
    if args.workload == "hetero":
        return hetero_bench(args)
    import torch
    import torch.distributed as dist

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120),
                                device_id=dev)
    pb, wl = workload_arrays()
    lib = pb._lib
    prec = args.precision or "fp16x3"
    prob = pb.model.problem_from_workload(wl)
    plan = pb.engines.DosePlan(prob, tables="device", precision=prec, device=dev)
    active = plan.active_pairs()
    flops_eval = 2 * credited_flops(wl, active)
    m = torch.as_tensor(wl["mask"], device=dev)
    p = torch.as_tensor(wl["presc"], device=dev)
    out = plan.alloc_outputs()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)   # > 126 MB L2

    def barrier():
        if world > 1:
            dist.barrier(device_ids=[local])

    clocks = ClockSampler(local)
    clocks.start()
    for _ in range(max(args.warmup, 3)):
        plan.loss_grad(m, p, outputs=out)
    torch.cuda.synchronize(dev)

    K = args.steps

    def timed(fn):
        """Total ms of K calls of fn, CUDA events around each call, L2 flushed (256 MiB
        write) before each one outside the events; max over ranks."""
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(K)]
        barrier()
        torch.cuda.synchronize(dev)
        for k in range(K):
            flush.zero_()
            ev[k][0].record()
            fn()
            ev[k][1].record()
        torch.cuda.synchronize(dev)
        barrier()
        t = sum(a.elapsed_time(b) for a, b in ev)
        if world > 1:
            tt = torch.tensor([t], device=dev, dtype=torch.float64)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            t = float(tt.item())
        return t

    # ---- device-resident, eager calls (per-kernel event profile, launch count) ----
    n0 = lib.launch_count()
    lib.profile_begin()
    t_eager = timed(lambda: plan.loss_grad(m, p, outputs=out))
    prof = lib.profile_end()
    launches_per_eval = (lib.launch_count() - n0) / K

    # ---- device-resident, the same call replayed from a CUDA graph (headline) ----
    g_dev = pb.engines.LossGradGraph(plan, m, p)
    for _ in range(max(args.warmup, 3)):
        g_dev.replay()
    t_ms = timed(g_dev.replay)
    value = world * K / (t_ms * 1e-3)
    launches = int(round(launches_per_eval * K))

    # ---- end to end through the public API, host buffers (pinned) ----
    # grad_w, grad_range and loss in one packed buffer on each side: one download per step
    w_host = torch.tensor(wl["weights"], dtype=torch.float32).pin_memory()
    host_res = plan.alloc_host_results()
    out_p = plan.alloc_outputs(packed=True)

    def eager_e2e():
        plan.loss_grad(m, p, w=w_host, outputs=out_p)
        host_res["packed"].copy_(out_p["packed"], non_blocking=True)

    t2_eager = timed(eager_e2e)
    g_e2e = pb.engines.LossGradGraph(plan, m, p, host_w=w_host, host_out=host_res)
    for _ in range(max(args.warmup, 3)):
        g_e2e.replay()
    t2 = timed(g_e2e.replay)

    # ---- the plain forward (no loss) replayed from a CUDA graph: dose fields/s ----
    dose_out = torch.empty(plan.shape, dtype=torch.float32, device=dev)
    plan.forward(out=dose_out)
    torch.cuda.synchronize(dev)
    g_fwd = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g_fwd):
        plan.forward(out=dose_out)
    for _ in range(max(args.warmup, 3)):
        g_fwd.replay()
    t_fwd = timed(g_fwd.replay)

    side = {}
    if not args.no_side_legs and world == 1:
        Ks, Ws = max(3, min(K, 20)), 3
        d64 = plan.forward_f64()
        side["gpu_baseline"] = gpu_baseline_leg(torch, dev, pb, wl, plan, flush, Ks,
                                                t_fwd / K, t_ms / K, d64)
        del d64
        side["robust"] = robust_leg(torch, dev, pb, flush, 5, Ws)
        side["precision"] = precision_leg(torch, dev, pb, flush, 5, Ws)
    clk = clocks.stop()
    e2e = world * K / (t2 * 1e-3)
    h2d = w_host.numel() * 4
    d2h = host_res["packed"].numel()   # the packed span: grad_w, grad_range, loss and padding

    # ---- roofline of the dominant kernel ----
    pk, pk_src = peaks()
    dom = "adjoint" if prof["adj_ms"] >= prof["fwd_ms"] else "forward"
    dom_ms = (prof["adj_ms"] / max(prof["n_adj"], 1)) if dom == "adjoint" else \
        (prof["fwd_ms"] / max(prof["n_fwd"], 1))
    per_launch_flop = flops_eval / 2.0
    achieved = per_launch_flop / (dom_ms * 1e-3) / 1e12
    # a ~0.1 ms kernel timed on its own: the burst figure
    peak = float(pk.get("bf16_tflops", 1590.0))
    if dom == "adjoint":
        kname = "adj_simt_kernel" if prec == "fp32" else "adj_tc_kernel"
    else:
        kname = {"fp32": "fwd_simt_kernel", "fp16x3": "fwd_tc16_kernel"}.get(prec, "fwd_tc_kernel")
    # the split forms' own ceiling: TF32 runs at half the BF16 rate, three products per MAC
    # (BF16x3: the BF16 rate, three products); credited FLOPs count one product
    split_ceiling = {"fp16x3": peak / 3.0, "tf32x3": peak / 6.0, "bf16x3": peak / 3.0,
                     "tf32": peak / 2.0, "bf16": peak}.get(prec if dom == "forward" else "bf16x3")
    roof = {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
            "frac": achieved / peak, "traffic": read_traffic(kname), "kernel": kname,
            "kernel_ms_per_launch": dom_ms, "flop_per_launch": per_launch_flop,
            "peak_source": ("measured bf16 dense burst (MEASURED_PEAKS.json)" if pk_src == "measured"
                            else "fallback bf16 dense burst 1590 TFLOP/s"),
            "split_ceiling_tflops": split_ceiling,
            "frac_of_split_ceiling": (achieved / split_ceiling) if split_ceiling else None,
            "note": CREDITED_NOTE + "; split_ceiling = the peak at the mode's operand rate "
                    "divided by its products per MAC",
            "fwd_ms_per_launch": prof["fwd_ms"] / max(prof["n_fwd"], 1),
            "adj_ms_per_launch": prof["adj_ms"] / max(prof["n_adj"], 1)}

    adj_mode = {"fp16x3": "bf16x3", "tf32x3": "bf16x3", "tf32": "bf16x3", "bf16x3": "bf16x3",
                "bf16": "bf16", "fp32": "fp32"}[prec]
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K,
            "warmup": max(args.warmup, 3), "ms_per_step": t_ms / K, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": f"{prec} fwd / {adj_mode} adj",
            "data": "synthetic",
            "config": {"workload": wl["name"], "grid": [128, 128, 128], "spots": 67240,
                       "layers": 40, "active_pairs": active, "precision": prec,
                       "credited_flop_per_eval": flops_eval,
                       "l2": "flushed between steps (256 MiB write, outside the events)",
                       "parallelism": f"{world} independent evaluations (one per rank)"},
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "how": "DosePlan loss gradient replayed from a "
                    "CUDA graph that uploads the weights and downloads dL/dW, dL/dR and L "
                    "(one packed copy)"},
            "eager": {"value": world * K / (t_eager * 1e-3),
                      "e2e": world * K / (t2_eager * 1e-3),
                      "how": "one DosePlan.loss_grad call per step (host work per call)"},
            "dose_fields_per_s": world * K / (t_fwd * 1e-3),
            "fwd_ms_per_step": t_fwd / K,
            "grad_over_fwd": t_ms / t_fwd,
            "gpu_launches": launches, "roofline": roof, "clocks": clk}
    line.update(side)

    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, n, el, cores, ref = run_cpu_port(wl, args.cpu_budget_s)
        line["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": cores, "kind": "port",
                                "sample": f"{n} full gradient evaluations in {el:.1f} s "
                                          "(torch CPU float64 port + autograd)"}
        torch.cuda.synchronize(dev)
        o = plan.loss_grad(m, p, outputs=out)
        torch.cuda.synchronize(dev)
        dref = ref["dose"].numpy()
        gwr = ref["grad_w"].numpy()
        grr = ref["grad_range"].numpy()
        line["accuracy_vs_fp64"] = {
            "dose_max_rel": float(np.max(np.abs(o["dose"].cpu().numpy() - dref)) / np.max(np.abs(dref))),
            "grad_w_max_rel": float(np.max(np.abs(o["grad_w"].cpu().numpy() - gwr)) / np.max(np.abs(gwr))),
            "grad_range_max_rel": float(np.max(np.abs(o["grad_range"].cpu().numpy() - grr))
                                        / np.max(np.abs(grr)))}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
