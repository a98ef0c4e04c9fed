"""Benchmark of the TMz FDTD hot path: one forward solve plus one
reference-mode gradient solve per step, in Gcell-steps/s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload config2] [--shots S] [--nt NT] [--tuning JSON]

Workload (default): the batched multi-shot gradient case -- a 400x300
physical model padded by 20 CPML cells per side (compute grid 440x340),
dx = 0.025 m, 64 shots, nt = 4000, 200 MHz Ricker, 100 receivers, layered
eps_r/sigma model generated from a fixed seed (synthetic data, no dataset).
The full Ez history (nt x 64 x 440 x 340 float32, 153 GB) stays resident in
HBM between the forward and the adjoint.

A step is compute()'s forward (traces + history) followed by the
reference-mode adjoint (imaging sums, L2-normalised): the path
GPRFWI.forward / GPRFWI.backward of the reference (src/compute.py:877-942)
with tv=False.  Gcell-steps/s fwd+adjoint = nx * ny * shots * nt / step time:
one unit per cell-step solved forward and back (the throughput definition
of the reference's epoch timings, cells x shots x steps / epoch time).

  value      device-resident inputs, CUDA events on the solve stream
  e2e        through the public compute() API: er/se/mr and the residual
             copied from pinned host memory, traces and both gradients
             copied back, every step
  roofline   the dominant kernel (the adjoint step kernel): algorithmic bytes
             per launch / its mean launch time, against the measured HBM
             copy bandwidth
  cpu_baseline  the CPU oracle (a C++/OpenMP restatement of the reference's
             update equations) on a bounded sample of the same workload

--impl reference prints the reference arm: the reference's update
equations on the host cores (the reference has no CPU code of its own; its
kernels are CUDA only), through the same CPU restatement, on a bounded sample.

Under torchrun (N > 1) every rank solves its own 64-shot batch (weak
scaling) and the unnormalised imaging sums are summed across ranks with one
NCCL all-reduce before the normalisation, as a multi-GPU gradient needs.
"""
from __future__ import annotations

import argparse
import importlib
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np
import torch

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
PKG = "fast-gpr-fwi_b200"

METRIC = "Gcell-steps/s fwd+adjoint"
UNIT = "Gcell-steps/s"

# DRAM bytes per shot-cell-step of each step kernel, from one ncu capture on the 440 x 340 grid with 64 shots
# (read + write); a kernel with no capture reports null traffic
# DRAM bytes (read + write) per launch of a step from one ncu capture of the
# 64-shot 440x340 workload, per shot and cell; a split step adds its two
# kernels (boundary lane march + interior kernel)
NCU_BYTES_PER_SHOT_CELL_STEP = {
    "fg::k_fwd + fg::k_fwd_slab + fg::k_fwd_core": (7.8e6 + 41.2e6 + 8.4e6 + 89.5e6 + 64.0e6) / (64 * 440 * 340),
    "fg::k_fwd + fg::k_fwd_core": (54.3e6 + 14.7e6 + 89.8e6 + 63.9e6) / (64 * 440 * 340),
    "fg::k_adj + fg::k_adj_core": (79.9e6 + 15.4e6 + 119.6e6 + 50.4e6) / (64 * 440 * 340),
    "fg::k_fwd (": 259.6e6 / (64 * 440 * 340), "fg::k_adj_pipe": 281.5e6 / (64 * 440 * 340),
    "fg::k_adj (": 293.9e6 / (64 * 440 * 340)}


def _fg():
    return importlib.import_module(PKG)


def parse():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="config2")
    ap.add_argument("--shots", type=int, default=None)
    ap.add_argument("--nt", type=int, default=None)
    ap.add_argument("--tuning", default=None, help="JSON dict of fg_tuning fields")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="target CPU sample length")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving leg")
    ap.add_argument("--no-config3", action="store_true", help="skip the config-3 multiscale inversion leg")
    ap.add_argument("--aux", action="store_true",
                    help="time only the TV and FIR kernels at config-3 sizes (one JSON line, not the headline)")
    return ap.parse_args()


def workload(args):
    fg = _fg()
    gen = fg.workloads.CONFIGS[args.workload]
    kw = {}
    if args.workload == "config2":
        if args.shots:
            kw["shots"] = args.shots
        if args.nt:
            kw["nt"] = args.nt
    wl = gen(**kw)
    if args.workload != "config2":
        if args.shots:
            wl.shots = args.shots
        if args.nt:
            wl.nt = args.nt
    return wl


# ---------------------------------------------------------------------------
# byte model (algorithmic bytes; FP32 TMz)
# ---------------------------------------------------------------------------

def strip_cells(nx, ny, th):
    """Cells inside at least one CPML slab (x strips + y strips)."""
    if th <= 0:
        return 0
    return 2 * th * ny + 2 * th * nx


def kernel_name(tuning, direction, split=False):
    """The step kernel a default (or given) launch shape runs, for the report
    (split: the interior tiles run in a kernel of their own beside it)."""
    t = tuning or {}
    if split:
        if direction == "forward" and t.get("slab", 0) != -1:
            return ("fg::k_fwd + fg::k_fwd_slab + fg::k_fwd_core (lane march on the tiles with events or in two "
                    "slabs, slab kernel on the CPML slabs, interior kernel, forward step)")
        d = "fwd" if direction == "forward" else "adj"
        return "fg::k_%s + fg::k_%s_core (lane march on the boundary tiles beside the interior kernel, %s step)" % (
            d, d, direction)
    if direction == "forward":
        k = t.get("kernel", 1)
    else:
        ak = t.get("adj_kernel", 0)
        k = (t.get("kernel", 1) if t else 1) if ak == 0 else (0 if ak == 1 else 1)
    pair = t.get("lanes") == 3
    if k == 0:
        return "fg::k_%s_pipe (tensor-map tile pipeline, %s step)" % ("fwd" if direction == "forward" else "adj",
                                                                      direction)
    return "fg::k_%s%s (lane march%s, %s step)" % ("fwd" if direction == "forward" else "adj", "2" if pair else "",
                                                  ", shot pairs" if pair else "", direction)


def algorithmic_bytes(nx, ny, shots, th):
    """Per launch of the forward / adjoint step kernel.

    forward: Ez/Hx/Hy read + write (24 B per shot-cell), Ca/Cb (8 B per cell,
    shared by the shots), two CPML auxiliaries read + write per strip cell
    (16 B per shot-strip-cell), the Ez history write (4 B per shot-cell).
    adjoint: the same plus the history read instead of its write, and the
    two imaging accumulators read + write (16 B per cell).
    """
    N = nx * ny
    P = strip_cells(nx, ny, th)
    fwd = 24 * shots * N + 8 * N + 16 * shots * P + 4 * shots * N
    adj = 24 * shots * N + 8 * N + 16 * shots * P + 4 * shots * N + 16 * N
    return fwd, adj


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ---------------------------------------------------------------------------
# clocks sampling during the timed region
# ---------------------------------------------------------------------------

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self._t = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self._t = threading.Thread(target=self._read, daemon=True)
        self._t.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        if self._t is not None:
            self._t.join(timeout=2)
        sm, mx, reasons = [], 0.0, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = max(mx, float(parts[2]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
# distributed plumbing
# ---------------------------------------------------------------------------

def dist_init(n_gpus):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        torch.cuda.set_device(local)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                             device_id=torch.device("cuda", local))
    return rank, local, world


def barrier(world):
    if world > 1:
        torch.distributed.barrier()


def max_over_ranks(x: float, world: int, dev) -> float:
    if world <= 1:
        return x
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------

def run_ours(args, rank, local, world):
    fg = _fg()
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    wl = workload(args)
    tuning = json.loads(args.tuning) if args.tuning else None
    kw = wl.kwargs(dev, tv=False)
    er_d = torch.tensor(wl.er, device=dev)
    se_d = torch.tensor(wl.se, device=dev)
    mr_d = torch.tensor(wl.mr, device=dev)
    setup = fg.grid.build_setup(dev, kw["dx"], kw["ny"], kw["nx"], kw["nz"], kw["time_windows"], kw["source"],
                                kw["source_location"], kw["source_step"], kw["receiver_location"],
                                kw["receiver_step"], kw["pmlthick"], kw["source_apmlitudes"], kw["step"],
                                torch.clamp(kw["er"], min=1), kw["mr"], kw["nsrc"], kw["nrx"], kw["dt"], None,
                                None, kw["Fixedreceiver"], None, None)
    nx, ny, S, nt = setup.nx, setup.ny, setup.shots, setup.nt
    solve = fg.Solve(dev, setup, tuning=tuning, tv=False)
    plan = solve.plan
    nrx = plan.nrx
    stream = torch.cuda.current_stream(dev)
    gen = torch.Generator(device=dev)
    gen.manual_seed(1234 + rank)
    resid = torch.randn((S, nt, nrx), device=dev, generator=gen, dtype=torch.float32) * 1e-3
    traces = torch.empty((S, nt, nrx), dtype=torch.float32, device=dev)
    hist = plan.new_hist()
    ge = torch.empty((nx, ny), dtype=torch.float32, device=dev)
    gs = torch.empty((nx, ny), dtype=torch.float32, device=dev)

    def one_step(ev=None):
        if ev is not None:
            ev[0].record(stream)
        plan.forward(er_d, se_d, mr_d, traces, hist)
        if ev is not None:
            ev[1].record(stream)
        if world > 1:
            plan.adjoint_reference(er_d, se_d, mr_d, hist, resid, ge, gs, normalize=False)
            fg.shots.combine_gradients(ge, gs)
        else:
            plan.adjoint_reference(er_d, se_d, mr_d, hist, resid, ge, gs, normalize=True)
        if ev is not None:
            ev[2].record(stream)

    for _ in range(args.warmup):
        one_step()
    torch.cuda.synchronize(dev)
    plan.device_check()

    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(args.steps)]
    clocks = ClockSampler(local)
    clocks.start()
    barrier(world)
    torch.cuda.synchronize(dev)
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for k in range(args.steps):
        one_step(evs[k])
    t1.record(stream)
    torch.cuda.synchronize(dev)
    barrier(world)
    clk = clocks.stop()
    ms_total = t0.elapsed_time(t1)
    fwd_ms = [e[0].elapsed_time(e[1]) for e in evs]
    adj_ms = [e[1].elapsed_time(e[2]) for e in evs]
    plan.device_check()
    ms_total = max_over_ranks(ms_total, world, dev)
    ms_step = ms_total / args.steps
    cell_steps = nx * ny * S * nt
    value = world * cell_steps / (ms_step * 1e-3) / 1e9

    # roofline of the dominant kernel (adjoint step kernel, nt-1 launches per adjoint)
    fwd_b, adj_b = algorithmic_bytes(nx, ny, S, setup.th)
    peak, peak_kind = measured_peaks()
    fwd_launch_ms = float(np.median(fwd_ms)) / nt
    adj_launch_ms = float(np.median(adj_ms)) / (nt - 1)
    dom = "adjoint" if np.median(adj_ms) >= np.median(fwd_ms) else "forward"
    bytes_launch = adj_b if dom == "adjoint" else fwd_b
    launch_ms = adj_launch_ms if dom == "adjoint" else fwd_launch_ms
    achieved = bytes_launch / (launch_ms * 1e-3) / 1e9
    # the interior split of the lane march (shot lanes, no stages, not
    # persistent, nx * ny * groups >= 12,000)
    t = tuning or {}
    shot = t.get("lanes", 1 if S >= 8 else 2) == 1
    work = nx * ny * ((S + 31) // 32)
    split = (shot and t.get("interior", 0) != -1 and not t.get("stages") and t.get("kernel", 1) == 1
             and (t.get("interior", 0) > 0 or (work >= 12000 and t.get("persistent", 0) != 1)))
    kname = kernel_name(tuning, dom, split)
    # this library's kernels per fwd + adj step: the forward's (general, slab,
    # interior) per time step, the adjoint's (general, interior; slab when
    # asked for or below 120,000 cells x groups) per iteration, two
    # coefficient kernels, the imaging tail and three gradient reductions
    slab = t.get("slab", 0)
    fwd_k = (3 if slab != -1 else 2) if split else 1
    adj_k = (3 if slab > 0 or (slab == 0 and work < 120000) else 2) if split else 1
    launches_per_step = fwd_k * nt + adj_k * (nt - 1) + 6
    ncu = next((v for k, v in NCU_BYTES_PER_SHOT_CELL_STEP.items() if kname.startswith(k)), None)
    roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "peak_source": peak_kind,
                "traffic": None if ncu is None else int(ncu * S * nx * ny),
                "kernel": kname,
                "algorithmic_bytes_per_launch": int(bytes_launch), "launch_ms": round(launch_ms, 5)}
    other = {"forward": {"launch_ms": round(fwd_launch_ms, 5), "algorithmic_bytes_per_launch": int(fwd_b),
                         "achieved_gbs": round(fwd_b / (fwd_launch_ms * 1e-3) / 1e9, 1),
                         "phase_ms": round(float(np.median(fwd_ms)), 3)},
             "adjoint": {"launch_ms": round(adj_launch_ms, 5), "algorithmic_bytes_per_launch": int(adj_b),
                         "achieved_gbs": round(adj_b / (adj_launch_ms * 1e-3) / 1e9, 1),
                         "phase_ms": round(float(np.median(adj_ms)), 3)}}
    # the same step captured once in a CUDA graph and replayed (the method of
    # the batched-gradient workload): every launch of the fwd + adj step in one
    # graph, programmatic dependencies included
    graph = None
    if world == 1 and not args.no_e2e:
        side = torch.cuda.Stream(dev)
        side.wait_stream(stream)
        with torch.cuda.stream(side):
            one_step()
        stream.wait_stream(side)
        torch.cuda.synchronize(dev)
        t_cap = time.perf_counter()
        cg = torch.cuda.CUDAGraph()
        with torch.cuda.graph(cg):
            one_step()
        t_cap = time.perf_counter() - t_cap
        cg.replay()
        torch.cuda.synchronize(dev)
        g0 = torch.cuda.Event(enable_timing=True)
        g1 = torch.cuda.Event(enable_timing=True)
        g0.record(stream)
        for _ in range(2):
            cg.replay()
        g1.record(stream)
        torch.cuda.synchronize(dev)
        plan.device_check()
        gms = g0.elapsed_time(g1) / 2
        graph = {"value": round(cell_steps / (gms * 1e-3) / 1e9, 3), "unit": UNIT, "ms_per_step": round(gms, 3),
                 "replays": 2, "capture_s": round(t_cap, 2),
                 "launches_per_step": int(launches_per_step)}
        del cg
    del hist, traces
    torch.cuda.empty_cache()

    e2e = None
    if not args.no_e2e:
        e2e = run_e2e(args, fg, wl, dev, rank, world)

    per_shot = None
    if rank == 0 and world == 1 and not args.no_e2e:
        per_shot = run_per_shot(args, fg, wl, dev)

    small = ckpt = cfg3 = batch = None
    if rank == 0 and world == 1 and not args.no_e2e:
        small = run_small_configs(fg, dev)
        batch = run_batch_uneven(fg, dev)
        ckpt = run_checkpointed(args, fg, wl, dev, tuning)
        if not args.no_config3:
            cfg3 = run_config3(fg, dev)

    serving = None
    if rank == 0 and world == 1 and not args.no_serve:
        serving = run_serving(fg, dev)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(wl, setup, args.cpu_seconds)

    fp64 = None
    if rank == 0 and world == 1 and not args.no_cpu:
        fp64 = fp64_error(fg, wl, dev, tuning)

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_step, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "%s: %dx%d compute grid (incl. 2x%d CPML), dx=%g m, %d shots, nt=%d, "
                                   "%d receivers, %.0f MHz Ricker, fwd + reference-mode adjoint, tv=False"
                                   % (wl.name, nx, ny, setup.th, setup.dx, S, nt, nrx, wl.freq / 1e6),
                       "shots_per_gpu": S, "nx": nx, "ny": ny, "nt": nt,
                       "history_gb": round(plan.hist_floats * 4 / 1e9, 1),
                       "l2": "inputs larger than L2 (state %.0f MB read + written per step, history %.0f GB)"
                             % (24 * S * nx * ny / 1e6, plan.hist_floats * 4 / 1e9),
                       "tuning": tuning or "default",
                       "parallelism": "replicas: shots per GPU, one all-reduce of the imaging sums" if world > 1
                       else "single GPU"},
            "gpu_launches": int(args.steps * launches_per_step),
            "roofline": roofline,
            "kernels": other,
            "clocks": clk,
            "e2e": e2e,
            "graph_replay": graph,
            "per_shot_path": per_shot,
            "small_configs": small,
            "batch_uneven": batch,
            "checkpointed": ckpt,
            "config3": cfg3,
            "serving": serving,
            "cpu_baseline": cpu,
            "fp64_err": fp64,
        }
        print(json.dumps(line), flush=True)


def run_e2e(args, fg, wl, dev, rank, world):
    """The same metric through compute() with host buffers, copies inside the timing."""
    pin = lambda a: torch.tensor(np.ascontiguousarray(a)[:, :, None]).pin_memory()
    er_h, se_h, mr_h = pin(wl.er), pin(wl.se), pin(wl.mr)
    S, nt, nrx = wl.shots, wl.nt, wl.nrx
    rng = np.random.default_rng(99 + rank)
    resid_h = torch.tensor(rng.standard_normal((S, nt, nrx)).astype(np.float32) * 1e-3).pin_memory()
    tr_h = torch.empty((S, nt, nrx), dtype=torch.float32).pin_memory()
    ge_h = torch.empty(er_h.shape, dtype=torch.float32).pin_memory()
    gs_h = torch.empty(se_h.shape, dtype=torch.float32).pin_memory()
    stream = torch.cuda.current_stream(dev)
    tuning = json.loads(args.tuning) if args.tuning else None

    def step():
        er = er_h.to(dev, non_blocking=True).requires_grad_(True)
        se = se_h.to(dev, non_blocking=True).requires_grad_(True)
        mr = mr_h.to(dev, non_blocking=True)
        g = resid_h.to(dev, non_blocking=True)
        kw = wl.kwargs(dev, er=er, se=se, mr=mr, tv=False, tuning=tuning)
        traces, _ = fg.compute(**kw)
        traces.backward(g)
        tr_h.copy_(traces.detach(), non_blocking=True)
        ge_h.copy_(er.grad, non_blocking=True)
        gs_h.copy_(se.grad, non_blocking=True)

    for _ in range(max(1, args.warmup)):
        step()
    torch.cuda.synchronize(dev)
    barrier(world)
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for _ in range(args.steps):
        step()
    t1.record(stream)
    torch.cuda.synchronize(dev)
    ms = max_over_ranks(t0.elapsed_time(t1), world, dev) / args.steps
    torch.cuda.empty_cache()
    cells = wl.nx * wl.ny * S * nt
    h2d = 3 * er_h.numel() * 4 + resid_h.numel() * 4
    d2h = tr_h.numel() * 4 + ge_h.numel() * 4 + gs_h.numel() * 4
    return {"value": round(world * cells / (ms * 1e-3) / 1e9, 3), "unit": UNIT, "ms_per_step": round(ms, 3),
            "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
            "api": "compute(..., tv=False) + traces.backward(resid)"}


def run_per_shot(args, fg, wl, dev, shots=4):
    """The plain per-shot drop-in path: compute() with step=1, one call (and
    one backward) per shot, inputs resident on the device, for the first
    `shots` shots of the workload; same metric as the batched solve."""
    er = torch.as_tensor(np.ascontiguousarray(wl.er)[:, :, None], device=dev).requires_grad_(True)
    se = torch.as_tensor(np.ascontiguousarray(wl.se)[:, :, None], device=dev).requires_grad_(True)
    mr = torch.as_tensor(np.ascontiguousarray(wl.mr)[:, :, None], device=dev)
    loc = torch.tensor(wl.source_location, dtype=torch.float32)
    dsrc = torch.tensor(wl.source_step, dtype=torch.float32)
    rloc = torch.tensor(wl.receiver_location, dtype=torch.float32)
    drx = torch.tensor(wl.receiver_step, dtype=torch.float32)
    gen = torch.Generator(device=dev)
    gen.manual_seed(4321)
    resid = torch.randn((1, wl.nt, wl.nrx), device=dev, generator=gen) * 1e-3

    def one(s):
        kw = wl.kwargs(dev, er=er, se=se, mr=mr, tv=False, step=1, source_location=loc + s * dsrc,
                       receiver_location=rloc if wl.fixed_receiver else rloc + s * drx)
        traces, _ = fg.compute(**kw)
        traces.backward(resid)

    one(0)
    torch.cuda.synchronize(dev)
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record()
    for s in range(shots):
        one(s)
    t1.record()
    torch.cuda.synchronize(dev)
    ms = t0.elapsed_time(t1)
    torch.cuda.empty_cache()
    return {"value": round(wl.nx * wl.ny * shots * wl.nt / (ms * 1e-3) / 1e9, 3), "unit": UNIT,
            "shots": shots, "ms_per_shot": round(ms / shots, 3),
            "api": "compute(..., step=1, tv=False) + traces.backward(resid), looped over shots"}


def run_batch_uneven(fg, dev, n_models=8, seed=2024, reps=2):
    """Many small models of uneven size: 8 seeded models (grids 100x60 to
    256x256 plus a 20-cell CPML, 8-32 shots, nt 800-1600, layered), each a
    forward + reference-mode adjoint, solved (a) one after another with the
    default launch shapes and (b) all in one persistent launch per direction
    (fg_forward_batch / fg_adjoint_reference_batch, plans with persistent = 1).
    Same metric, the pair counted once; inputs resident on the device."""
    nat = importlib.import_module(PKG + "._native")
    wmod = fg.workloads
    rng = np.random.default_rng(seed)
    models = []
    for _ in range(n_models):
        nx_, ny_ = int(rng.integers(100, 257)), int(rng.integers(60, 257))
        shots, nt = int(rng.integers(8, 33)), int(rng.integers(800, 1601))
        er, se = wmod._layered_model(rng, nx_, ny_, 0.025)
        er = wmod._pad(er, wmod.PAD).astype(np.float32)
        se = wmod._pad(se, wmod.PAD).astype(np.float32)
        p, lx, ly = wmod.PAD * 0.025, nx_ * 0.025, ny_ * 0.025
        models.append(wmod.Workload("batch", nx_ + 40, ny_ + 40, 0.025, shots, nt, 2e8, er, se, np.ones_like(er),
                                    source_location=[p + 0.05 * lx, p + 0.1 * ly, 0.0],
                                    source_step=[0.9 * lx / shots, 0.0, 0.0],
                                    receiver_location=[p + 0.05 * lx, p + 0.9 * ly, 0.0],
                                    receiver_step=[0.9 * lx / 16, 0.0, 0.0], nrx=16, fixed_receiver=True))
    cells = sum(w.nx * w.ny * w.shots * w.nt for w in models)
    out = {"models": n_models, "cell_steps": int(cells)}
    for mode, tuning in (("one_after_another", None), ("one_persistent_launch", {"lanes": 1, "persistent": 1})):
        solves, mats, bufs = [], [], []
        for w in models:
            setup = _setup_of(fg, w, dev)
            s = fg.Solve(dev, setup, tuning=tuning, tv=False)
            m = tuple(torch.tensor(a, device=dev) for a in (w.er, w.se, w.mr))
            tr = torch.empty((setup.shots, setup.nt, s.plan.nrx), device=dev)
            bufs.append((tr, s.plan.new_hist(), torch.randn(tr.shape, device=dev) * 1e-3,
                         torch.empty((setup.nx, setup.ny), device=dev), torch.empty((setup.nx, setup.ny), device=dev)))
            solves.append(s)
            mats.append(m)
        plans = [s.plan for s in solves]

        def step():
            if mode == "one_after_another":
                for p, m, b in zip(plans, mats, bufs):
                    p.forward(m[0], m[1], m[2], b[0], b[1])
                    p.adjoint_reference(m[0], m[1], m[2], b[1], b[2], b[3], b[4])
            else:
                cols = lambda k: [m[k] for m in mats]
                nat.forward_batch(plans, cols(0), cols(1), cols(2), [b[0] for b in bufs], [b[1] for b in bufs])
                nat.adjoint_reference_batch(plans, cols(0), cols(1), cols(2), [b[1] for b in bufs],
                                            [b[2] for b in bufs], [b[3] for b in bufs], [b[4] for b in bufs])

        step()
        torch.cuda.synchronize(dev)
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record()
        for _ in range(reps):
            step()
        t1.record()
        torch.cuda.synchronize(dev)
        for p in plans:
            p.device_check()
        ms = t0.elapsed_time(t1) / reps
        out[mode] = {"value": round(cells / (ms * 1e-3) / 1e9, 3), "unit": UNIT, "ms_per_step": round(ms, 2)}
        del solves, plans, bufs, mats
        torch.cuda.empty_cache()
    return out


def run_small_configs(fg, dev, reps=3):
    """The benchmark's two smaller configurations, each as one forward +
    reference-mode adjoint per step with inputs resident on the device and
    the default launch shapes: config 0 (140x100, 1 shot, nt 1200) and
    config 1 (240x160, 13 shots, nt 3000); same metric as the headline."""
    out = {}
    for wl in (fg.workloads.config0(), fg.workloads.config1()):
        kw = wl.kwargs(dev, tv=False)
        setup = fg.grid.build_setup(dev, kw["dx"], kw["ny"], kw["nx"], kw["nz"], kw["time_windows"], kw["source"],
                                    kw["source_location"], kw["source_step"], kw["receiver_location"],
                                    kw["receiver_step"], kw["pmlthick"], kw["source_apmlitudes"], kw["step"],
                                    torch.clamp(kw["er"], min=1), kw["mr"], kw["nsrc"], kw["nrx"], kw["dt"], None,
                                    None, kw["Fixedreceiver"], None, None)
        solve = fg.Solve(dev, setup, tv=False)
        plan = solve.plan
        er, se, mr = (torch.tensor(a, device=dev) for a in (wl.er, wl.se, wl.mr))
        S, nt = setup.shots, setup.nt
        traces = torch.empty((S, nt, plan.nrx), device=dev)
        hist = plan.new_hist()
        gen = torch.Generator(device=dev)
        gen.manual_seed(77)
        resid = torch.randn(traces.shape, device=dev, generator=gen) * 1e-3
        ge = torch.empty((setup.nx, setup.ny), device=dev)
        gs = torch.empty_like(ge)

        def step():
            plan.forward(er, se, mr, traces, hist)
            plan.adjoint_reference(er, se, mr, hist, resid, ge, gs)

        for _ in range(3):
            step()
        torch.cuda.synchronize(dev)
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record()
        for _ in range(reps):
            step()
        t1.record()
        torch.cuda.synchronize(dev)
        plan.device_check()
        ms = t0.elapsed_time(t1) / reps
        out[wl.name] = {"value": round(setup.nx * setup.ny * S * nt / (ms * 1e-3) / 1e9, 3), "unit": UNIT,
                        "ms_per_step": round(ms, 3), "grid": [setup.nx, setup.ny], "shots": S, "nt": nt,
                        "lanes": "shot lanes" if S >= 8 else "column lanes", "steps": reps, "warmup": 3}
        del hist, traces, solve, plan
        torch.cuda.empty_cache()
    return out


def _setup_of(fg, wl, dev, er=None):
    kw = wl.kwargs(dev, tv=False)
    er = torch.clamp(kw["er"] if er is None else er, min=1)
    return fg.grid.build_setup(dev, kw["dx"], kw["ny"], kw["nx"], kw["nz"], kw["time_windows"], kw["source"],
                               kw["source_location"], kw["source_step"], kw["receiver_location"],
                               kw["receiver_step"], kw["pmlthick"], kw["source_apmlitudes"], kw["step"], er,
                               kw["mr"], kw["nsrc"], kw["nrx"], kw["dt"], None, None, kw["Fixedreceiver"], None,
                               None)


def run_checkpointed(args, fg, wl, dev, tuning, steps=2):
    """The headline workload with checkpoint='auto': the solver state every K
    steps (K the autotuner's: the fastest checkpointed gradient that fits in
    80% of the free memory) instead of the whole Ez history; the adjoint
    recomputes each history segment (one more forward solve per step).  Same
    metric, inputs resident on the device."""
    autotune = importlib.import_module(PKG + ".autotune")
    setup = _setup_of(fg, wl, dev)
    t_tune = time.perf_counter()
    solve = fg.Solve(dev, setup, tuning=tuning, tv=False, checkpoint="auto")
    t_tune = time.perf_counter() - t_tune
    plan, k = solve.plan, solve.interval
    er, se, mr = (torch.tensor(a, device=dev) for a in (wl.er, wl.se, wl.mr))
    S, nt = setup.shots, setup.nt
    traces = torch.empty((S, nt, plan.nrx), device=dev)
    gen = torch.Generator(device=dev)
    gen.manual_seed(1234)
    resid = torch.randn(traces.shape, device=dev, generator=gen) * 1e-3
    ge = torch.empty((setup.nx, setup.ny), device=dev)
    gs = torch.empty_like(ge)
    ck = plan.new_checkpoints(k)
    seg = plan.new_segment(k)

    def step():
        plan.forward_checkpointed(er, se, mr, traces, ck, k)
        plan.adjoint_reference_checkpointed(er, se, mr, ck, k, seg, resid, ge, gs)

    step()
    torch.cuda.synchronize(dev)
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record()
    for _ in range(steps):
        step()
    t1.record()
    torch.cuda.synchronize(dev)
    plan.device_check()
    ms = t0.elapsed_time(t1) / steps
    mem = autotune.checkpoint_memory(plan, k)
    del ck, seg, traces, solve, plan
    torch.cuda.empty_cache()
    return {"value": round(setup.nx * setup.ny * S * nt / (ms * 1e-3) / 1e9, 3), "unit": UNIT,
            "ms_per_step": round(ms, 3), "interval": k, "steps": steps, "warmup": 1,
            "checkpoints_plus_segment_gb": round(mem / 1e9, 2),
            "full_history_gb": round(4 * setup.nx * setup.ny * S * nt / 1e9, 1),
            "autotune_s": round(t_tune, 1),
            "api": "Solve(checkpoint='auto'): fg_forward_checkpointed + fg_adjoint_reference_checkpointed"}


def run_config3(fg, dev, epochs_per_stage=2):
    """Config 3 end to end: 840x540 (800x500 + 2x20 CPML), 30 shots, nt 6000,
    the three-stage multiscale inversion of the reference's example (observed
    traces low-passed at 50, 100 and 200 MHz by apply_filter, compute()'s
    freq set to the stage's), TV weight 1e-3, two epochs per stage (the
    workload names 20; every epoch is the same work), the
    gradient checkpointed at the autotuned interval (the full Ez history
    would be 327 GB).  Observed traces: a forward solve of the true layered
    model; starting model: its smoothed copy."""
    ms_mod = importlib.import_module(PKG + ".multiscale")
    autotune = importlib.import_module(PKG + ".autotune")
    wl = fg.workloads.config3()
    setup = _setup_of(fg, wl, dev)
    true_er, true_se, mr = (torch.tensor(a, device=dev) for a in (wl.er, wl.se, wl.mr))
    obs, _ = fg.Solve(dev, setup, tv=False).forward(true_er, true_se, mr, keep_history=False)
    torch.cuda.synchronize(dev)
    kernel = torch.ones((1, 1, 21, 21), device=dev) / 441.0
    smooth = lambda a: torch.nn.functional.conv2d(a[None, None], kernel, padding=10)[0, 0]
    er = smooth(true_er)[:, :, None].contiguous()
    se = smooth(true_se)[:, :, None].contiguous()
    mr3 = mr[:, :, None].contiguous()
    kw = wl.kwargs(dev)
    for key in ("er", "se", "mr", "tv", "device"):
        kw.pop(key)
    stages = []
    cells = setup.nx * setup.ny * setup.shots * setup.nt
    for f in (5e7, 1e8, 2e8):
        obs_f = ms_mod.apply_filter(obs, 1.0 / setup.dt, f)
        t_plan = time.perf_counter()
        inv = fg.Inversion(dev, dict(kw, freq=f), obs_f, er, se, mr3, tv_weight=1e-3, checkpoint="auto",
                           phase1_epochs=0)
        t_plan = time.perf_counter() - t_plan
        times, losses = [], []
        for _ in range(epochs_per_stage):
            t0 = torch.cuda.Event(enable_timing=True)
            t1 = torch.cuda.Event(enable_timing=True)
            t0.record()
            losses.append(round(inv.epoch(), 6))
            t1.record()
            torch.cuda.synchronize(dev)
            times.append(t0.elapsed_time(t1))
        ms = float(np.mean(times))
        k = inv.solve.interval
        stages.append({"cutoff_mhz": int(f / 1e6), "epoch_ms": round(ms, 1), "epochs": epochs_per_stage,
                       "losses": losses,
                       "value": round(cells / (ms * 1e-3) / 1e9, 3), "interval": k,
                       "checkpoints_plus_segment_gb": round(autotune.checkpoint_memory(inv.solve.plan, k) / 1e9, 2),
                       "plan_and_autotune_s": round(t_plan, 1)})
        er, se = inv.er.detach(), inv.se.detach()
        del inv
        torch.cuda.empty_cache()
    fp64 = fp64_error(fg, wl, dev, None, shots=1, nt=3000)
    total_ms = sum(st["epoch_ms"] for st in stages)   # one epoch of each stage
    return {"value": round(len(stages) * cells / (total_ms * 1e-3) / 1e9, 3), "unit": UNIT,
            "grid": [setup.nx, setup.ny], "shots": setup.shots, "nt": setup.nt, "stages": stages,
            "epoch": "forward + recomputed forward + fused-L1 reference adjoint + TV (weight 1e-3) + Adam",
            "full_history_gb": round(4 * cells / 1e9, 1), "fp64_err": fp64}


def serving_stream(fg, n=12, seed=4004):
    """A seeded stream drawn from the serving workload's distribution:
    physical grids uniform from 100x60 to 1024x1024 cells (plus a 20-cell
    CPML per side), dx 0.025 m, nt uniform in 1000-8000, 1-32 shots, 100-200
    MHz Ricker, layered models as the benchmark's, cross-hole geometry.  Half
    the requests are gradients, each on its own survey; the other half are
    forward requests in pairs that share a survey (grid, model, waveform)
    with different shot positions, which the server may merge."""
    serve = importlib.import_module(PKG + ".serve")
    wmod = fg.workloads
    rng = np.random.default_rng(seed)
    reqs = []
    survey = None
    for k in range(n):
        forward = k % 4 in (1, 2)               # pairs of forward requests: (1, 2), (5, 6), ...
        if not (forward and k % 4 == 2):
            nx_ = int(rng.integers(100, 1025))
            ny_ = int(rng.integers(60, 1025))
            nt = int(rng.integers(1000, 8001))
            freq = float(rng.uniform(1e8, 2e8))
            dx = 0.025
            er, se = wmod._layered_model(rng, nx_, ny_, dx)
            er = wmod._pad(er, wmod.PAD).astype(np.float32)
            se = wmod._pad(se, wmod.PAD).astype(np.float32)
            survey = (nx_, ny_, nt, freq, er, se)
        nx_, ny_, nt, freq, er, se = survey
        shots = int(rng.integers(1, 33))
        p = wmod.PAD * dx
        lx, ly = nx_ * dx, ny_ * dx
        wl = wmod.Workload("serve", nx_ + 2 * wmod.PAD, ny_ + 2 * wmod.PAD, dx, shots, nt, freq, er, se,
                           np.ones_like(er), source_location=[p + 0.05 * lx, p + 0.1 * ly, 0.0],
                           source_step=[0.9 * lx / shots, 0.0, 0.0],
                           receiver_location=[p + 0.05 * lx, p + 0.9 * ly, 0.0],
                           receiver_step=[0.9 * lx / 16, 0.0, 0.0], nrx=16, fixed_receiver=True)
        if forward and k % 4 == 2:
            wl.source_location[0] += 0.45 * lx / shots     # the pair's second request: shots in between
        kw = wl.kwargs("cuda")
        for key in ("er", "se", "mr", "device", "tv"):
            kw.pop(key)
        resid = None
        if not forward:
            resid = torch.tensor(rng.standard_normal((shots, nt, wl.nrx)).astype(np.float32) * 1e-3)
        reqs.append(serve.Request(kw, torch.tensor(wl.er), torch.tensor(wl.se), torch.tensor(wl.mr), resid,
                                  merge_key=("survey", k // 4) if forward else None))
    return serve, reqs


def _serve_once(serve, dev, reqs, gaps, active, policy="sjf", merge=True):
    srv = serve.Server(dev, max_active=active, policy=policy, merge=merge, batch=merge)
    futs = []
    for r, gap in zip(reqs, gaps):
        time.sleep(float(gap))
        futs.append(srv.submit(r))
    for f in futs:
        f.result()
    st = srv.stats()
    srv.close()
    return {"p50_ms": round(st["p50_s"] * 1e3, 1), "p99_ms": round(st["p99_s"] * 1e3, 1),
            "throughput_gcs": round(st["throughput_gcs"], 3), "peak_active": st["peak_active"],
            "merged": st["merged"], "batched": st["batched"]}


def run_serving_small(fg, dev, n=16, seed=5005):
    """A burst of small requests (grids 100x60 to 256x256 plus a 20-cell
    CPML, 8-32 shots, nt 800-1600, half gradients), all queued at once:
    continuous batching (small shot-lane requests batched into one persistent
    launch per direction, up to 4 launches on the GPU at once) against the
    plain one-request-at-a-time path."""
    serve = importlib.import_module(PKG + ".serve")
    wmod = fg.workloads
    rng = np.random.default_rng(seed)
    reqs = []
    for k in range(n):
        nx_, ny_ = int(rng.integers(100, 257)), int(rng.integers(60, 257))
        shots, nt = int(rng.integers(8, 33)), int(rng.integers(800, 1601))
        er, se = wmod._layered_model(rng, nx_, ny_, 0.025)
        er = wmod._pad(er, wmod.PAD).astype(np.float32)
        se = wmod._pad(se, wmod.PAD).astype(np.float32)
        p, lx, ly = wmod.PAD * 0.025, nx_ * 0.025, ny_ * 0.025
        wl = wmod.Workload("serve", nx_ + 40, ny_ + 40, 0.025, shots, nt, 2e8, er, se, np.ones_like(er),
                           source_location=[p + 0.05 * lx, p + 0.1 * ly, 0.0], source_step=[0.9 * lx / shots, 0.0, 0.0],
                           receiver_location=[p + 0.05 * lx, p + 0.9 * ly, 0.0], receiver_step=[0.9 * lx / 16, 0.0, 0.0],
                           nrx=16, fixed_receiver=True)
        kw = wl.kwargs("cuda")
        for key in ("er", "se", "mr", "device", "tv"):
            kw.pop(key)
        resid = None
        if k % 2:
            resid = torch.tensor(rng.standard_normal((shots, nt, wl.nrx)).astype(np.float32) * 1e-3)
        reqs.append(serve.Request(kw, torch.tensor(wl.er), torch.tensor(wl.se), torch.tensor(wl.mr), resid))
    warm = serve.Server(dev, max_active=1)
    warm.submit(reqs[0]).result()
    warm.close()
    out = {"requests": n, "arrivals": "all at once"}
    for name, active, plain in (("continuous", 4, False), ("one_at_a_time", 1, True)):
        out[name] = _serve_once(serve, dev, reqs, np.zeros(n), active, "fifo" if plain else "sjf", not plain)
    torch.cuda.empty_cache()
    return out


def run_serving(fg, dev, rates_x=(0.5, 1.0, 2.0)):
    """The stream at Poisson rates swept across saturation, served with
    continuous batching (up to 4 requests on the GPU at once, a GPU-filling
    request alone, forward requests of one survey merged, shortest job first
    with a 2 s bound on waiting), against the plain one-request-at-a-time
    path (first come, first served, no merging) at the highest rate.  The saturation rate is measured first: requests per second
    of the one-at-a-time path with all requests queued at once."""
    serve, reqs = serving_stream(fg)
    warm = serve.Server(dev, max_active=1)
    warm.submit(reqs[0]).result()                 # plans, kernels, allocator
    warm.close()
    t0 = time.perf_counter()
    base = _serve_once(serve, dev, reqs, np.zeros(len(reqs)), 1, "fifo", False)
    sat = len(reqs) / (time.perf_counter() - t0)
    rates = []
    for x in rates_x:
        gaps = np.random.default_rng(7).exponential(1.0 / (x * sat), size=len(reqs))
        rates.append(dict(rate_hz=round(x * sat, 3), **_serve_once(serve, dev, reqs, gaps, 4)))
    top = np.random.default_rng(7).exponential(1.0 / (rates_x[-1] * sat), size=len(reqs))
    one = dict(rate_hz=round(rates_x[-1] * sat, 3), **_serve_once(serve, dev, reqs, top, 1, "fifo", False))
    torch.cuda.empty_cache()
    small = run_serving_small(fg, dev)
    return {"requests": len(reqs), "saturation_hz": round(sat, 3), "all_queued_one_at_a_time": base,
            "rates": rates, "one_at_a_time": one, "small_burst": small,
            "stream": "grids 100x60-1024x1024 (+2x20 CPML), nt 1000-8000, 1-32 shots, 100-200 MHz; "
                      "half gradients, half forward requests in same-survey pairs",
            "unit": "Gcell-steps/s, nx*ny*shots*nt per request counted once (forward or gradient)"}


# ---------------------------------------------------------------------------
# CPU legs (the oracle: test infrastructure, used here only as the timed baseline)
# ---------------------------------------------------------------------------

def _cpu_problem(wl, setup, shots, nt, first=0):
    """Oracle problem for a sample of the workload: shots first..first+shots-1,
    the first `nt` steps, float32 coefficients restated on the host."""
    from oracle import oracle as orc
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import helpers
    coef = helpers.coefficients_f32(np.maximum(wl.er, 1), np.maximum(wl.se, 0), wl.mr, setup.dt32, setup.dx)
    pml = setup.profile.packed() if setup.profile is not None else np.zeros((8, 0), np.float32)
    sel = slice(first, first + shots)
    src = orc.positions2(setup.src.cpu().numpy()[sel], wl.nx, wl.ny)
    rx = orc.positions2(setup.rx.cpu().numpy()[sel], wl.nx, wl.ny)
    return orc.Problem(wl.nx, wl.ny, setup.th, shots, nt, setup.dx, setup.dt32, coef["uE0"], coef["uE1"],
                       coef["uE4"], coef["uH1"], coef["uH4"], coef["uE0a"], pml, src,
                       np.ascontiguousarray(setup.srcw[:, :nt]), rx)


def _cpu_sample_run(prob):
    from oracle import oracle as orc
    rng = np.random.default_rng(5)
    resid = rng.standard_normal((prob.shots, prob.nt, prob.rx.shape[1])).astype(np.float32)
    t0 = time.perf_counter()
    _, hist = orc.forward(prob, np.float32)
    orc.adjoint_reference(prob, hist, resid, np.float32)
    return time.perf_counter() - t0


def _cpu_sample(wl, setup, seconds):
    """Pick a sample of the workload that runs about `seconds`: `batches`
    consecutive batches of `shots` shots, each solved over the first `nt`
    steps (the history of one batch is kept under ~4 GB of host memory)."""
    from oracle import oracle as orc
    threads = orc.set_threads(os.cpu_count() or 1)
    shots = min(4, wl.shots)
    nt_cal = min(40, wl.nt)
    _cpu_sample_run(_cpu_problem(wl, setup, shots, nt_cal))           # thread pool and page warm-up
    nt_cal = min(120, wl.nt)
    t_cal = _cpu_sample_run(_cpu_problem(wl, setup, shots, nt_cal))
    per_step = t_cal / nt_cal
    nt = int(max(nt_cal, min(wl.nt, seconds / max(per_step, 1e-9))))
    nt = int(min(nt, 4e9 / (shots * wl.nx * wl.ny * 4)))
    batches = int(max(1, min(wl.shots // shots, round(seconds / max(per_step * nt, 1e-9)))))
    return shots, nt, batches, threads


def _cpu_sample_time(wl, setup, shots, nt, batches):
    return sum(_cpu_sample_run(_cpu_problem(wl, setup, shots, nt, b * shots)) for b in range(batches))


def _sample_text(wl, shots, nt, batches):
    return ("%s grid %dx%d, shots 0-%d in batches of %d, first %d of %d steps, fwd + reference adjoint"
            % (wl.name, wl.nx, wl.ny, shots * batches - 1, shots, nt, wl.nt))


def cpu_baseline(wl, setup, seconds):
    shots, nt, batches, threads = _cpu_sample(wl, setup, seconds)
    t = _cpu_sample_time(wl, setup, shots, nt, batches)
    cells = wl.nx * wl.ny * shots * batches * nt
    return {"value": round(cells / t / 1e9, 4), "unit": UNIT, "cores": threads, "kind": "port",
            "sample": _sample_text(wl, shots, nt, batches) + ", FP32 C++/OpenMP oracle, %.1f s" % t,
            "cpu": _cpu_model()}


def fp64_error(fg, wl, dev, tuning, shots=4, nt=1000):
    """Relative L2 error of the benchmark's FP32 solve against the FP64 oracle
    of the same update equations, on a bounded sample of the workload: its
    first `shots` shots over its first `nt` steps (long enough for the forward
    and adjoint fields to meet between the boreholes), solved on the GPU with
    the benchmark's launch shape (shot lanes) and on the host in double
    precision (FP64 coefficients, CPML profile and Ricker).  Traces, the reference-mode
    gradient (unit norm, as the step returns it) and the exact adjoint's
    gradient of the same weights."""
    from oracle import oracle as orc
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import helpers
    if wl.name == "config2":
        sample = fg.workloads.config2(shots=shots, nt=nt)
    elif wl.name == "config3":
        sample = fg.workloads.config3()
        sample.shots, sample.nt = shots, nt
    else:
        return None
    t0 = time.perf_counter()
    rng = np.random.default_rng(64)
    w = rng.standard_normal((shots, nt, sample.nrx)).astype(np.float32)
    prob, setup = helpers.oracle_problem_from_gpu(fg, sample, dev)
    p64 = helpers.fp64_problem(prob, setup, sample)
    o_tr, o_hist = orc.forward(p64, np.float64)
    oe, os_ = orc.adjoint_reference(p64, o_hist, w, np.float64)
    oe /= np.linalg.norm(oe)
    os_ /= np.linalg.norm(os_)
    s1, s2 = orc.exact_sums(p64, o_hist, w.astype(np.float64))
    xe, xs = orc.exact_gradient(s1, s2, np.maximum(sample.er, 1), np.maximum(sample.se, 0), setup.dt32)
    del o_hist
    wt = torch.tensor(w, device=dev)
    shot_lanes = dict(tuning or {}, lanes=1)
    tr, ge, gs = helpers.run_package(fg, sample, dev, wt, tuning=shot_lanes)
    _, ee, es = helpers.run_package(fg, sample, dev, wt, tuning=shot_lanes, adjoint="exact")
    r = lambda a, b: round(helpers.rel_l2(a.cpu().numpy(), b), 9)
    out = {"sample": "%s grid %dx%d, shots 0-%d, first %d of %d steps; FP32 GPU solve vs FP64 oracle"
                     % (wl.name, sample.nx, sample.ny, shots - 1, nt, wl.nt),
           "traces": r(tr, o_tr), "g_eps": r(ge, oe), "g_sig": r(gs, os_),
           "exact_g_eps": r(ee, xe), "exact_g_sig": r(es, xs), "seconds": round(time.perf_counter() - t0, 1)}
    torch.cuda.empty_cache()
    return out


def _cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def run_reference(args, rank, world):
    """Reference arm: the reference's update equations on the host cores."""
    if rank != 0:
        return
    fg = _fg()
    wl = workload(args)
    kw = wl.kwargs("cpu", tv=False)
    setup = fg.grid.build_setup("cpu", kw["dx"], kw["ny"], kw["nx"], kw["nz"], kw["time_windows"], kw["source"],
                                kw["source_location"], kw["source_step"], kw["receiver_location"],
                                kw["receiver_step"], kw["pmlthick"], kw["source_apmlitudes"], kw["step"],
                                torch.clamp(kw["er"], min=1), kw["mr"], kw["nsrc"], kw["nrx"], kw["dt"], None,
                                None, kw["Fixedreceiver"], None, None)
    seconds = max(2.0, min(args.cpu_seconds, 120.0 / max(1, args.steps + args.warmup)))
    shots, nt, batches, threads = _cpu_sample(wl, setup, seconds)
    for _ in range(args.warmup):
        _cpu_sample_time(wl, setup, shots, nt, batches)
    times = [_cpu_sample_time(wl, setup, shots, nt, batches) for _ in range(args.steps)]
    t = float(np.sum(times)) / args.steps
    cells = wl.nx * wl.ny * shots * batches * nt
    value = cells / t / 1e9
    sample = _sample_text(wl, shots, nt, batches) + " per step, FP32 C++/OpenMP restatement of the reference kernels"
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(t * 1e3, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "%s: %dx%d compute grid, %d shots, nt=%d (bounded CPU sample: %d shots x %d steps)"
                               % (wl.name, wl.nx, wl.ny, wl.shots, wl.nt, shots * batches, nt)},
        "cpu_baseline": {"value": round(value, 4), "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": sample, "cpu": _cpu_model()},
        "e2e": {"value": round(value, 4), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_aux(args):
    """The kernels around the solver at config-3 sizes, timed alone: the TV
    kernel on an 840x540 model (ADMM, up to 500 iterations, tol 1e-5, the
    reference's defaults) and the causal FIR kernel on 30 shots x 6000 steps
    x 120 receivers at the 50 MHz stage.  One JSON line (not the headline)."""
    fg = _fg()
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    ms_mod = importlib.import_module(PKG + ".multiscale")
    nat = importlib.import_module(PKG + "._native")
    wl = fg.workloads.config3()
    model = torch.tensor(wl.er, device=dev)
    gen = torch.Generator(device=dev)
    gen.manual_seed(5)
    traces = torch.randn((wl.shots, wl.nt, wl.nrx), device=dev, generator=gen)
    fs = 1.0 / wl.dt
    numtaps = int(fs / 5e7)
    taps = ms_mod.design_fir_filter(5e7, fs, numtaps)

    def timed(fn, reps):
        fn()
        torch.cuda.synchronize(dev)
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record()
        for _ in range(reps):
            out = fn()
        t1.record()
        torch.cuda.synchronize(dev)
        return t0.elapsed_time(t1) / reps, out

    reps = max(1, args.steps)
    tv_ms, (_, iters) = timed(lambda: nat.total_variation(model, 0.02, 1.0, 500, 1e-5), reps)
    fir_ms, _ = timed(lambda: nat.fir_causal(traces, taps), reps)
    moved = 2 * traces.numel() * 4
    line = {"aux": True, "config": "config-3 sizes: model 840x540; traces 30x6000x120, %d taps" % numtaps,
            "tv": {"ms": round(tv_ms, 3), "iterations": iters, "cells": model.numel()},
            "fir": {"ms": round(fir_ms, 3), "taps": numtaps, "bytes_in_out": moved,
                    "achieved_gbs": round(moved / (fir_ms * 1e-3) / 1e9, 1)},
            "steps": reps}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.aux:
        run_aux(args)
        return
    if args.impl == "reference":
        rank = int(os.environ.get("RANK", "0"))
        world = int(os.environ.get("WORLD_SIZE", "1"))
        run_reference(args, rank, world)
        return
    rank, local, world = dist_init(args.gpus)
    try:
        run_ours(args, rank, local, world)
    finally:
        if world > 1:
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
