#!/usr/bin/env python
"""Throughput of the elastic RTM hot path on B200.

One step = one RTM shot of the 3D workload: the source pass (src_steps = 2*nt/3 time
steps with excitation capture) and the receiver pass (nt time steps with data
injection and excitation-amplitude PP/PS/TP imaging), through the C ABI.

Workload (seeded synthetic, no dataset): 400 x 400 x 300 interior at 10 m with a
40-cell C-PML (480 x 480 x 380 = 87.55 M cells), 8th-order staggered grid, dt 0.8 ms,
nt 4000, 10 Hz Ricker at the surface centre, 200 x 200 receivers every 20 m.

Metric: Gcell-updates/s = cells x (src_steps + nt) / step time.  `value` has the
observed data and the images in HBM; `e2e` passes pinned host buffers through the
same API call (H2D of the data, D2H of the three images inside the timed region).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
Under torchrun each rank migrates its own shot (shots shard with no exchange);
the per-shot images are stacked with one NCCL reduce per step.
"""
from __future__ import annotations

import argparse
import ctypes as C
import datetime
import importlib
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

REPO = os.path.dirname(os.path.abspath(__file__))
PKG = "2d_and_3d_elastic_reverse_time_migration_b200"
sys.path.insert(0, REPO)

METRIC = "Gcell-updates/s (3D elastic RTM shot: source + receiver pass)"
UNIT = "Gcell/s"
# compulsory DRAM traffic of the elastic step: 9 fields read and written, 3 model arrays
COMPULSORY_B = 84
# DRAM bytes per cell of each source-pass step kernel (dram__bytes_read.sum +
# dram__bytes_write.sum, one ncu capture per kernel on the 240 x 240 x 190 grid with a
# 20-cell C-PML: the same slab fractions as the 3D workload)
TRAFFIC_B_PER_CELL = {"stress": 96.2, "velocity": 107.9}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--small", action="store_true", help="small grid (debugging only)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--kernel-steps", type=int, default=60)
    ap.add_argument("--grid", default="", help="interior nx,ny,nz (profiling cases only)")
    ap.add_argument("--pml", type=int, default=40, help="C-PML width (profiling cases only)")
    ap.add_argument("--step-variant", default="single", choices=["single", "pairs"],
                    help="3D step kernels: one cell per thread (default) or x-adjacent cell pairs")
    ap.add_argument("--kernels-only", action="store_true",
                    help="only time the step kernels (profiling cases)")
    ap.add_argument("--workload", default="shot",
                    choices=["shot", "windows", "unet", "lsrtm", "lsrtm-op", "lsrtm-cg", "refstep",
                             "passcheck"],
                    help="windows: batched aperture windows; unet: one U-Net training step at "
                         "256x512, batch 16; lsrtm: learned vs plain CG (each its own line); "
                         "lsrtm-op: Born forward + adjoint per shot on the 880x480 GSLS-3 LSRTM grid; "
                         "refstep: the reference's own 2D CUDA step kernels against this "
                         "library's 2D step on the same grids and GPU")
    ap.add_argument("--train-models", type=int, default=48)
    ap.add_argument("--test-models", type=int, default=6)
    ap.add_argument("--train-steps", type=int, default=1500)
    ap.add_argument("--lsrtm-geometry", default="small", choices=["small", "patch"],
                    help="lsrtm workload: small = 128x64 cells, 6 shots, 500 steps, 64x128 patches; "
                         "patch = 512x256 cells at 5 m, 8 shots, 2000 steps, one 256x512 patch per model")
    ap.add_argument("--train-batch", type=int, default=16)
    ap.add_argument("--shots", type=int, default=64, help="windows workload: shots")
    ap.add_argument("--lanes", type=int, default=10,
                    help="windows workload: shots per launch (1 .. 10, ertm_rtm_multi groups)")
    ap.add_argument("--cg-iters", type=int, default=20, help="lsrtm-cg workload: CG iterations")
    return ap.parse_args()


def workload(small: bool, grid: str = "", pml: int = 40):
    synth = importlib.import_module(PKG + ".synthetic")
    if grid:
        nx, ny, nz = (int(v) for v in grid.split(","))
        return synth.layered_3d(n_interior=(nz, ny, nx), pml=pml, nt=400, smooth_sigma=0)
    if small:
        return synth.layered_3d(n_interior=(60, 80, 80), pml=20, nt=400, smooth_sigma=4.0)
    return synth.layered_3d()


def _shot(ertm, wl, synth, rank):
    sx, sy, sz = wl.src
    if rank:  # other ranks migrate other shots: shift the source laterally
        nz, ny, nx = wl.shape
        sx = wl.pml + (sx - wl.pml + 37 * rank) % (nx - 2 * wl.pml)
        sy = wl.pml + (sy - wl.pml + 53 * rank) % (ny - 2 * wl.pml)
    w = synth.ricker(wl.freq, wl.dt_ms / 1000.0)
    return ertm.Shot(sx, sy, sz, wavelet=w, **wl.rec)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""
    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid: str):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", uuid, f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.p = None

    def stop(self) -> dict:
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        self.p.wait()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.count(",") >= 7]
        os.unlink(self.f.name)
        sm = [float(r[0]) for r in rows if r[0].strip().replace(".", "").isdigit()]
        mx = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        pw = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[4 + i].strip() == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(rows),
                "power_w": statistics.median(pw) if pw else None}


class CpuOracle:
    """FP32 OpenMP oracle (a port of the reference's update loops, same scheme) holding
    the full-grid state.  `run(n)` times n source-pass steps with excitation capture;
    `run_receiver(n)` times n receiver-pass steps (data injection at the surface
    receivers, P/S split, imaging at the excitation time)."""

    def __init__(self, wl):
        import numpy as np
        sys.path.insert(0, os.path.join(REPO, "oracle"))
        import oracle as orc
        self.orc, self.L = orc, orc.lib(32)
        nz, ny, nx = wl.shape
        self.cells = nx * ny * nz
        self.g = orc.make_grid(nx, ny, nz, wl.dx, wl.dy, wl.dz, wl.dt_ms, R=4, boundary=orc.CPML,
                               pml=(wl.pml,) * 6, pml_vmax=float(wl.svp.max()))
        self.st = self.L.orc_state_create(C.byref(self.g), orc._fp(wl.svp), orc._fp(wl.svs),
                                          orc._fp(wl.srho))
        if not self.st:
            raise RuntimeError("oracle state allocation failed")
        self.shot = orc.make_shot(*wl.src, orc.ricker(wl.freq, wl.dt_ms / 1000.0), **wl.rec)
        self.ex = orc.ExcitationArrays(wl.shape)
        self.es = self.ex.struct()
        self.nrec = wl.rec["nrx"] * wl.rec["nry"]
        self.data = np.zeros((3, 4, self.nrec), np.float32)     # 4 injected samples, cycled
        self.img = [np.zeros(wl.shape, np.float32) for _ in range(3)]
        self.it = 0
        self.run(1)  # first touch of every page, untimed by callers

    @property
    def threads(self):
        return self.L.orc_threads()

    def run(self, n: int) -> float:
        t0 = time.perf_counter()
        for _ in range(n):
            self.L.orc_state_step(self.st, C.byref(self.shot), self.orc.SOURCE, self.it, 1 << 30,
                                  None, C.byref(self.es), None, None, None)
            self.it += 1
        return time.perf_counter() - t0

    def run_receiver(self, n: int) -> float:
        f = self.orc._fp
        t0 = time.perf_counter()
        for q in range(n):
            self.L.orc_state_step(self.st, C.byref(self.shot), self.orc.RECEIVER, q % 4, 4,
                                  f(self.data), C.byref(self.es), *[f(a) for a in self.img])
        return time.perf_counter() - t0

    def rate_for(self, seconds: float):
        """Rate over rounds of 2 source-pass and 3 receiver-pass steps (the shot's ratio)."""
        n, el = 0, 0.0
        while el < seconds or n < 5:
            el += self.run(2) + self.run_receiver(3)
            n += 5
        return self.cells * n / el / 1e9, n

    def close(self):
        if self.st:
            self.L.orc_state_destroy(self.st)
            self.st = None


def shot_config(wl, world: int, nrec: int) -> dict:
    """The `config` of the RTM-shot workload, shared by both bench arms."""
    nz, ny, nx = wl.shape
    return {"workload": wl.name, "cells": nx * ny * nz, "nt": wl.nt, "src_steps": 2 * wl.nt // 3,
            "order": 8, "boundary": f"cpml{wl.pml}", "dt_ms": wl.dt_ms, "receivers": nrec,
            "parallelism": f"shots x{world}",
            "l2": "inputs larger than L2 (13 wavefields + model, ~8 GB)"}


def run_reference(args):
    """The reference arm: the FP32 OpenMP oracle, a port of the reference's update loops
    (the reference has no CPU implementation and its 3D kernels are absent from its
    tree), on the same RTM-shot workload as this library's arm: the 8th-order scheme
    with the 40-cell C-PML of the 3D workload, source-pass and receiver-pass steps in
    the shot's 2 : 3 ratio (2666 : 4000).  One step is a bounded sample of 2 source and
    3 receiver time steps of the full grid; rank 0 alone runs it."""
    if int(os.environ.get("RANK", "0")) != 0:
        return
    synth = importlib.import_module(PKG + ".synthetic")
    wl = (synth.layered_3d(n_interior=(60, 80, 80), pml=20, nt=400, smooth_sigma=0)
          if args.small else synth.layered_3d(smooth_sigma=0))
    cpu = CpuOracle(wl)
    ns, nr = 2, 3
    for _ in range(args.warmup):
        cpu.run(ns)
        cpu.run_receiver(nr)
    el = 0.0
    for _ in range(args.steps):
        el += cpu.run(ns) + cpu.run_receiver(nr)
    v = cpu.cells * (ns + nr) * args.steps / el / 1e9
    nz, ny, nx = wl.shape
    sample = (f"{ns} source-pass and {nr} receiver-pass time steps of the full {nx}x{ny}x{nz} "
              f"grid per step (the shot's 2:3 ratio); FP32 OpenMP port of the update loops, "
              f"{cpu.threads} threads")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": round(v, 4), "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(el / args.steps * 1e3, 2), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded layered model with an ellipsoid; observed data modelled "
                "in the true model)",
        "config": shot_config(wl, args.gpus, cpu.nrec),
        "cpu_baseline": {"value": round(v, 4), "unit": UNIT, "cores": cpu.threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": round(v, 4), "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }), flush=True)
    cpu.close()


def run_windows(args):
    """Batched RTM over aperture windows of a shared model: one step = the whole
    batch (every shot's source and receiver pass) through ertm_rtm_windows."""
    import numpy as np
    import torch
    ertm = importlib.import_module(PKG)
    synth = importlib.import_module(PKG + ".synthetic")
    (vp, vs, rho), wins, shots = synth.windows_3d(nshots=args.shots)
    nz, ny, nx = vp.shape
    pml = 40
    base = ertm.Config(nx=nx, ny=ny, nz=nz, dx=10.0, dy=10.0, dz=10.0, dt_ms=0.8, nt=1, order=8,
                       boundary=ertm.BOUNDARY_CPML, pml=(pml,) * 6, autotune=1)
    dev = torch.device("cuda", 0)
    w = synth.ricker(10.0, 0.8e-3)
    W = [ertm.Window(**d) for d in wins]
    S = [ertm.Shot(wavelet=w, **d) for d in shots]
    g = torch.Generator(device=dev).manual_seed(20261203)
    # seeded random traces stand in for recorded data (the cost does not depend on it)
    data = [torch.randn((3, win.nt, sh.nrec), generator=g, device=dev) * 1e-6 for win, sh in zip(W, S)]
    model = [torch.from_numpy(np.ascontiguousarray(a)).to(dev) for a in (vp, vs, rho)]
    outs = [torch.zeros((nz, ny, nx), device=dev) for _ in range(3)]
    updates = 0
    for win in W:
        cells = (win.wx + 2 * pml) * (win.wy + 2 * pml) * (nz + 2 * pml)
        updates += cells * (2 * win.nt // 3 + win.nt)
    ertm.rtm_windows(base, *model, W[:2], S[:2], data[:2], lanes=min(2, args.lanes))   # tune, warm
    torch.cuda.synchronize(dev)
    uuid = str(torch.cuda.get_device_properties(dev).uuid)
    clocks = ClockSampler(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
    t0 = time.perf_counter()
    ertm.rtm_windows(base, *model, W, S, data, lanes=args.lanes, pp=outs[0], ps=outs[1], tp=outs[2])
    torch.cuda.synchronize(dev)
    el = time.perf_counter() - t0
    clk = clocks.stop()
    print(json.dumps({
        "metric": "Gcell-updates/s (batched 3D elastic RTM over aperture windows)",
        "value": round(updates / el / 1e9, 3), "unit": UNIT, "n_gpus": 1, "steps": 1, "warmup": 1,
        "seconds": round(el, 2), "higher_is_better": True, "dtype": "f32",
        "data": "synthetic shared model (layered + ellipsoid); seeded random traces",
        "config": {"workload": f"windows-{args.shots}shots-{nx}x{ny}x{nz}", "shots": args.shots,
                   "shots_per_launch": min(args.lanes, ertm.MULTI_MAX),
                   "window": "U[64,192]^2 + 40-cell C-PML", "nt": "U[2000,3500]",
                   "cell_updates": updates, "autotune": 1},
        "clocks": clk}), flush=True)


def run_passcheck(args):
    """The 3D step inside a pass against the same kernels launched one step at a
    time: a source pass (2666 steps, CUDA events around the pass) and then 2000
    step pairs each followed by a host synchronisation (ertm_time_kernels), with
    the SM clock and board power sampled during each."""
    import torch
    ertm = importlib.import_module(PKG)
    synth = importlib.import_module(PKG + ".synthetic")
    wl = workload(False)
    nz, ny, nx = wl.shape
    ctx = ertm.Context(ertm.Config(nx=nx, ny=ny, nz=nz, dx=wl.dx, dy=wl.dy, dz=wl.dz, dt_ms=wl.dt_ms,
                                   nt=wl.nt, order=8, boundary=ertm.BOUNDARY_CPML, pml=(wl.pml,) * 6))
    dev = torch.device("cuda", 0)
    st = torch.cuda.current_stream(dev)
    ctx.set_stream(st.cuda_stream)
    ctx.set_model(ertm.MIGRATION_MODEL, wl.svp, wl.svs, wl.srho)
    shot = _shot(ertm, wl, synth, 0)
    uuid = str(torch.cuda.get_device_properties(dev).uuid)
    uuid = uuid if uuid.startswith("GPU-") else "GPU-" + uuid
    ctx.forward_together_using_smoothed_model(shot)          # warm-up pass
    torch.cuda.synchronize(dev)
    nsrc = 2 * wl.nt // 3
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clk = ClockSampler(uuid)
    e0.record(st)
    ctx.forward_together_using_smoothed_model(shot)
    e1.record(st)
    torch.cuda.synchronize(dev)
    c_pass = clk.stop()
    pass_ms = e0.elapsed_time(e1) / nsrc
    n = 2000
    clk = ClockSampler(uuid)
    ms_s, ms_v = ctx.time_kernels(shot, n)
    c_sync = clk.stop()
    print(json.dumps({"workload": wl.name, "pass": {"ms_per_step": round(pass_ms, 4), "steps": nsrc,
                                                    "clocks": c_pass},
                      "synchronised": {"stress_ms": round(ms_s / n, 4), "velocity_ms": round(ms_v / n, 4),
                                       "ms_per_step": round((ms_s + ms_v) / n, 4), "steps": n,
                                       "clocks": c_sync}}), flush=True)
    ctx.close()


def run_unet(args):
    """U-Net training step (forward, loss, backward, Adam) on 16 patches of 256 x 512:
    tensor-core throughput of the learned part, CUDA events on the current stream."""
    import torch
    nn = importlib.import_module(PKG + ".nn")
    dev = torch.device("cuda", 0)
    net = nn.UNet(dev, seed=0)
    n, h, w = 16, 256, 512
    g = torch.Generator(device="cpu").manual_seed(0)
    x = torch.randn(n, h, w, 3, generator=g).to(dev)
    t = torch.randn(n, h, w, 3, generator=g).to(dev)
    for _ in range(max(3, args.warmup)):
        net.step(x, t)
    st = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(dev)
    e0.record(st)
    for _ in range(args.steps):
        net.step(x, t)
    e1.record(st)
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1) / args.steps
    flops = 3 * n * net.flops_per_sample(h, w)     # forward + input and weight gradients
    peaks_path = os.path.join(REPO, "MEASURED_PEAKS.json")
    peak = float(json.load(open(peaks_path))["bf16_tflops"]) if os.path.exists(peaks_path) else 1590.0
    tf = flops / (ms / 1e3) / 1e12
    print(json.dumps({"metric": "U-Net training step (256x512, batch 16)", "value": round(ms, 3),
                      "unit": "ms/step", "higher_is_better": False, "dtype": "bf16 (fp32 accumulate)",
                      "steps": args.steps, "warmup": args.warmup,
                      "flops_per_step": flops, "tflops": round(tf, 2),
                      "roofline": {"bound": "tensor", "achieved": round(tf, 2), "peak": peak,
                                   "unit": "TFLOP/s", "frac": round(tf / peak, 4)},
                      "forward_gflop_per_patch": round(net.flops_per_sample(h, w) / 1e9, 3)}), flush=True)


def run_lsrtm(args):
    """Learned-preconditioned LSRTM (reduced scale): training pairs from CG on seeded
    layered-and-faulted models, U-Net training, plain vs learned CG on held-out models."""
    import numpy as np
    import torch
    nn = importlib.import_module(PKG + ".nn")
    L = importlib.import_module(PKG + ".learned")
    dev = torch.device("cuda", 0)
    if args.lsrtm_geometry == "patch":
        # the LSRTM workload's 5 m cells and generator, cut to one 256 x 512 training
        # patch per model (512 x 256 interior + 40-cell sponge), 8 shots, 2000 steps
        geo = L.Geometry(nzi=256, nxi=512, h=5.0, pml=40, nt=2000, dt_ms=0.5, nshots=8, f0=15.0,
                         sigma=10.0)
        patch = (256, 512)
    else:
        geo = L.Geometry()
        patch = (64, 128)
    t0 = time.perf_counter()
    pairs = []
    for k in range(args.train_models):
        case = L.make_case(1000 + k, geo)
        pairs.append(L.training_pair(case, cg_iters=10))
        case.ctx.close()
        if k in (0, 3) or (k + 1) % 16 == 0:
            print(json.dumps({"event": "training_pairs", "done": k + 1,
                              "seconds": round(time.perf_counter() - t0, 1)}), flush=True)
    t_data = time.perf_counter() - t0
    net = nn.UNet(dev, seed=0)
    log = L.train(net, pairs, steps=args.train_steps, batch=args.train_batch, patch=patch, lr=1e-3)
    print(json.dumps({"event": "trained", "seconds": round(log.seconds, 1),
                      "loss_first_last": [log.loss[0][1], log.loss[-1][1]]}), flush=True)
    target, niter = 1e-2, 20
    rows = []
    for k in range(args.test_models):
        case = L.make_case(5000 + k, geo)
        rows.append(L.compare(case, net, niter=niter, target=target))
        case.ctx.close()
        print(json.dumps({"event": "test_case", "seed": 5000 + k, **_fmt_case(rows[-1])}), flush=True)
    def med(key):
        v = [r[key] for r in rows if r[key] is not None]
        return float(np.median(v)) if v else None
    print(json.dumps({
        "metric": "LSRTM: learned vs plain CG (iterations and wall time to plain CG's 20-iteration misfit, and to 1e-2)",
        "unit": "iterations / s", "config": {"grid": f"{geo.nxi}x{geo.nzi} + sponge {geo.pml}",
                                           "dx": geo.h, "shots": geo.nshots, "nt": geo.nt,
                                           "patch": list(patch), "batch": args.train_batch,
                                           "train_models": args.train_models,
                                           "test_models": args.test_models,
                                           "train_steps": args.train_steps, "cg_iters_target": 10},
        "plain_iters_median": med("plain_iters"), "learned_iters_median": med("learned_iters"),
        "plain_time_median": med("plain_time_to_target"),
        "learned_time_median": med("learned_time_to_target"),
        "learned_iters_to_plain_20_median": med("learned_iters_to_plain_final"),
        "time_ratio_to_plain_20_median": med("time_ratio_to_plain_final"),
        "plain_model_err_median": med("plain_model_err"),
        "learned_model_err_median": med("learned_model_err"),
        "model_rel_diff_median": med("model_rel_diff"),
        "data_seconds": round(t_data, 1), "train_seconds": round(log.seconds, 1),
        "train_loss": log.loss[::max(1, len(log.loss) // 8)],
        "cases": [_fmt_case(r) for r in rows]}), flush=True)


def _lsrtm_setup(nshots: int):
    """The LSRTM workload: 880 x 480 cells (800 x 400 interior + 40-cell sponge) at 5 m,
    seeded layered-and-faulted model, GSLS with 3 mechanisms (Qp 100, Qs 50, f0 15 Hz),
    dt 0.5 ms, 4000 steps, 800 receivers at 10 m depth, 40 shot positions, checkpoints
    every 200 steps; migration model smoothed with sigma 10 cells; the true relative
    perturbations are the model against its smoothed version."""
    import numpy as np
    ertm = importlib.import_module(PKG)
    L = importlib.import_module(PKG + ".learned")
    syn = importlib.import_module(PKG + ".synthetic")
    g = L.Geometry(nzi=400, nxi=800, h=5.0, pml=40, nt=4000, dt_ms=0.5, nshots=40, f0=15.0,
                   sigma=10.0, visco=(3, 100.0, 50.0, 15.0))
    vp, vs, rho = syn.faulted_2d(20261203, g.nzi, g.nxi, g.h)
    pads = (g.pml, g.pml, 0, 0, g.pml, g.pml)
    vp, vs, rho = (syn.pad_edges(a, pads) for a in (vp, vs, rho))
    svp, svs, srho = (syn.gaussian_smooth(a, g.sigma) for a in (vp, vs, rho))
    true = tuple((a / b - 1.0).astype(np.float32) for a, b in ((vp, svp), (vs, svs), (rho, srho)))
    nz, _, nx = vp.shape
    cfg = ertm.Config(nx=nx, ny=1, nz=nz, dx=g.h, dy=g.h, dz=g.h, dt_ms=g.dt_ms, nt=g.nt, order=8,
                      boundary=ertm.BOUNDARY_SPONGE_CUBIC, pml=pads, sponge_coef=150.0,
                      checkpoint_every=200, visco_nmech=3, visco_qp=100.0, visco_qs=50.0, visco_f0=15.0)
    ctx = ertm.Context(cfg)
    ctx.set_model(ertm.MIGRATION_MODEL, svp, svs, srho)
    w = syn.ricker(g.f0, g.dt_ms / 1000.0)
    xs = np.linspace(g.pml + 4, nx - g.pml - 5, 40).round().astype(int)
    rz = g.pml + 2
    pick = xs[np.linspace(0, 39, max(1, min(nshots, 40))).round().astype(int)]
    shots = [ertm.Shot(int(x), 0, rz, wavelet=w, rx0=g.pml, nrx=nx - 2 * g.pml, drx=1, rz=rz)
             for x in pick]
    return ertm, ctx, cfg, shots, true, (nz, nx), g


LSRTM_WORKLOAD = ("LSRTM 880x480 (800x400 + 40-cell sponge), dx 5 m, GSLS-3 Qp 100 Qs 50 f0 15 Hz, "
                  "dt 0.5 ms, nt 4000, 800 receivers, checkpoints every 200 steps")


def run_lsrtm_op(args):
    """LSRTM operators at the LSRTM workload's size: the Born forward and its adjoint
    over `--shots` of the 40 shot positions, all shots in one batched call each (every
    step's kernels cover every shot), device arrays in and out, CUDA events on the
    context stream; projects one 40-shot CG iteration and the 20-iteration run."""
    import torch
    nshots = max(1, min(args.shots, 40))
    ertm, ctx, cfg, shots, true, (nz, nx), g = _lsrtm_setup(nshots)
    dev = torch.device("cuda", 0)
    st = torch.cuda.current_stream(dev)
    ctx.set_stream(st.cuda_stream)
    m = [torch.from_numpy(a).to(dev) for a in true]
    data = torch.zeros((len(shots), 3, g.nt, shots[0].nrec), device=dev)
    grads = [torch.zeros((nz, 1, nx), device=dev) for _ in range(3)]
    if args.warmup > 0:   # warm-up: allocations (--warmup 0 for profiling captures)
        ctx.born_forward_shots(shots[:1], *m, out=data[:1])
        ctx.born_adjoint_shots(shots[:1], data[:1], *grads)
    e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    torch.cuda.synchronize(dev)
    e[0].record(st)
    ctx.born_forward_shots(shots, *m, out=data)
    e[1].record(st)
    ctx.born_adjoint_shots(shots, data, *grads)
    e[2].record(st)
    torch.cuda.synchronize(dev)
    tf, ta = e[0].elapsed_time(e[1]) / 1e3, e[1].elapsed_time(e[2]) / 1e3
    cells = float(nx * nz)
    fwd_steps = 2.0 * cells * g.nt * len(shots)          # background + scattered
    adj_steps = 3.0 * cells * g.nt * len(shots)          # background, rebuild, adjoint
    per_shot = (tf + ta) / len(shots)
    print(json.dumps({
        "metric": "LSRTM operator throughput (Born forward + adjoint, GSLS-3, batched shots)",
        "value": round((fwd_steps + adj_steps) / (tf + ta) / 1e9, 3), "unit": "Gcell-steps/s",
        "higher_is_better": True, "dtype": "f32", "data": "synthetic",
        "config": {"workload": LSRTM_WORKLOAD, "shots_timed": len(shots)},
        "forward_s": round(tf, 3), "adjoint_s": round(ta, 3),
        "forward_gcell_steps_s": round(fwd_steps / tf / 1e9, 3),
        "adjoint_gcell_steps_s": round(adj_steps / ta / 1e9, 3),
        "projected_cg_iteration_40_shots_s": round(40 * per_shot, 2),
        "projected_20_iterations_s": round(20 * 40 * per_shot, 1),
        "timing": "CUDA events on the context stream around one batched call each, device arrays"}),
        flush=True)
    ctx.close()


def run_lsrtm_cg(args):
    """The LSRTM workload end to end: 20 CGLS iterations over the 40 shots, every CG
    vector on the device, data modelled with the Born operator from the true
    perturbations.  Reports the misfit curve and the wall time per iteration, the
    reflectivity error, and two checks at this size on one shot: the dot-product test
    of the operator pair and the centred finite difference of the misfit
    0.5 |F m - d|^2 along a random direction against the adjoint gradient."""
    import numpy as np
    import torch
    lsrtm = importlib.import_module(PKG + ".lsrtm")
    ertm, ctx, cfg, shots, true, (nz, nx), g = _lsrtm_setup(args.shots)
    dev = torch.device("cuda", 0)
    m_true = [torch.from_numpy(a).to(dev) for a in true]
    t0 = time.perf_counter()
    data_all = lsrtm.born_all(ctx, shots, m_true)
    torch.cuda.synchronize(dev)
    t_data = time.perf_counter() - t0
    data = [data_all[i] for i in range(len(shots))]
    times = []
    last = [time.perf_counter()]

    def cb(it, mis):
        now = time.perf_counter()
        times.append(now - last[0])
        last[0] = now

    t0 = time.perf_counter()
    last[0] = t0
    res = lsrtm.cgls(ctx, shots, data, niter=args.cg_iters, callback=cb)
    torch.cuda.synchronize(dev)
    t_cg = time.perf_counter() - t0
    err = [float(torch.linalg.norm(a - b) / torch.linalg.norm(b)) for a, b in zip(res.m, m_true)]
    # checks on the first shot at full size
    rng = np.random.default_rng(7)
    one = shots[:1]
    mh = [torch.from_numpy((0.05 * rng.standard_normal((nz, 1, nx))).astype(np.float32)).to(dev)
          for _ in range(3)]
    d = lsrtm.born_all(ctx, one, mh)
    dh = torch.from_numpy(rng.standard_normal(tuple(d.shape)).astype(np.float32)).to(dev)
    dh[:, 1] = 0
    gh = lsrtm.adjoint_all(ctx, one, dh)
    lhs = float((d.double() * dh.double()).sum())
    rhs = sum(float((a.double() * b.double()).sum()) for a, b in zip(mh, gh))
    # misfit phi(m) = 0.5 |F m - d1|^2 around m0 = 0.5 true along direction p
    d1 = data_all[:1]
    m0 = [0.5 * a for a in m_true]
    r0 = lsrtm.born_all(ctx, one, m0) - d1
    grad = lsrtm.adjoint_all(ctx, one, r0)
    p = mh
    h = 1.0
    phi = lambda mm: 0.5 * float(((lsrtm.born_all(ctx, one, mm) - d1).double() ** 2).sum())
    fd = (phi([a + h * b for a, b in zip(m0, p)]) - phi([a - h * b for a, b in zip(m0, p)])) / (2 * h)
    an = sum(float((a.double() * b.double()).sum()) for a, b in zip(grad, p))
    print(json.dumps({
        "metric": "LSRTM 20-iteration CGLS wall time (40 shots, GSLS-3)", "value": round(t_cg, 2),
        "unit": "s", "higher_is_better": False, "dtype": "f32", "data": "synthetic",
        "config": {"workload": LSRTM_WORKLOAD, "shots": len(shots), "cg_iterations": args.cg_iters,
                   "vectors": "device (torch CUDA tensors)"},
        "data_modelling_s": round(t_data, 2),
        "seconds_per_iteration": [round(x, 2) for x in times],
        "misfit": [round(x, 6) for x in res.misfit], "accepted": res.accepted,
        "reflectivity_rel_error": {"vp": round(err[0], 4), "vs": round(err[1], 4), "rho": round(err[2], 4)},
        "dot_test": {"lhs": lhs, "rhs": rhs, "rel": abs(lhs - rhs) / abs(lhs)},
        "fd_gradient": {"fd": fd, "adjoint": an, "rel": abs(fd - an) / abs(an), "h": h,
                        "note": "one shot; phi = 0.5 |F m - d|^2 is quadratic in m, so the centred "
                                "difference is exact up to rounding"}}), flush=True)
    ctx.close()


def run_refstep(args):
    """The reference's own 2D CUDA time step (its stress kernel
    fwd_txxzzxzpp_viscoelastic_and_memory_3parameterization and its velocity kernels
    adjoint_fwd_vx/vz_viscoelastic, 2D_elastic_RTM/viscoelastic_equation.cu:184-325,
    :1827-2122, compiled from the reference tree into oracle/_ref/libref2d.so) against
    this library's 2D step (k_stress + k_velocity, source-pass variant with the P
    stress, the reference's 12th-order coefficients and cubic sponge) on the same
    interior grids, CUDA events around every launch, after warm-up steps.  One line
    per grid.  The reference kernels also carry one memory-variable set per cell
    (viscoelastic form; tao = strain = 1 makes it elastic), so they move more bytes."""
    import numpy as np
    import torch
    ertm = importlib.import_module(PKG)
    lib_path = os.path.join(REPO, "oracle", "_ref", "libref2d.so")
    if not os.path.exists(lib_path):
        print(json.dumps({"workload": "refstep", "unavailable": "oracle/_ref/libref2d.so not built "
                          "(the reference tree is needed to build it)"}), flush=True)
        return
    L = C.CDLL(lib_path)
    coe = np.array([0.0, 1.2213363647, -0.096931457519, 0.017447662353, -0.0029672895159,
                    0.00035900539822, -0.00002184781161], np.float32)
    dt_ms, h = 0.5, 5.0
    steps, warm = max(args.kernel_steps, 20), 5
    for nx, nz in ((704, 384), (896, 480), (4096, 2048)):
        ms = (C.c_float * 3)()
        rc = L.ref_time_step(nx, nz, steps, warm, C.c_float(dt_ms), C.c_float(h), C.c_float(h),
                             coe.ctypes.data_as(C.POINTER(C.c_float)), ms)
        if rc != 0:
            raise RuntimeError(f"ref_time_step {nx}x{nz}: CUDA error {rc}")
        ref_ms = [m / steps for m in ms]
        cfg = ertm.Config(nx=nx, ny=1, nz=nz, dx=h, dy=h, dz=h, dt_ms=dt_ms, nt=steps, order=12,
                          coef_kind=ertm.COEF_REFERENCE12, boundary=ertm.BOUNDARY_SPONGE_CUBIC,
                          pml=(40, 40, 0, 0, 40, 40), sponge_coef=150.0)
        vp = np.full((nz, 1, nx), 2500.0, np.float32)
        vs = (vp / np.sqrt(3)).astype(np.float32)
        rho = np.full_like(vp, 2200.0)
        with ertm.Context(cfg) as ctx:
            ctx.set_model(ertm.MIGRATION_MODEL, vp, vs, rho)
            shot = ertm.Shot(nx // 2, 0, 45, wavelet=np.ones(8, np.float32) * 1e-3, rx0=40,
                             nrx=nx - 80, rz=45)
            ctx.time_kernels(shot, warm)
            ours = [m / steps for m in ctx.time_kernels(shot, steps)]
        cells = nx * nz
        ref_step, our_step = sum(ref_ms), sum(ours)
        print(json.dumps({
            "workload": "refstep", "grid": f"{nx}x{nz}", "cells": cells, "steps_timed": steps,
            "metric": "Gcell-updates/s (2D elastic time step, same GPU)", "unit": UNIT,
            "reference": {"value": round(cells / (ref_step / 1e3) / 1e9, 3),
                          "ms_per_step": round(ref_step, 4),
                          "kernels_ms": {"fwd_txxzzxzpp_viscoelastic_and_memory_3parameterization":
                                         round(ref_ms[0], 4),
                                         "adjoint_fwd_vx_viscoelastic": round(ref_ms[1], 4),
                                         "adjoint_fwd_vz_viscoelastic": round(ref_ms[2], 4)},
                          "build": "reference 2D kernels, nvcc -O2 sm_100a, tiles 32x16 (inferred)"},
            "ours": {"value": round(cells / (our_step / 1e3) / 1e9, 3), "ms_per_step": round(our_step, 4),
                     "kernels_ms": {"k_stress": round(ours[0], 4), "k_velocity": round(ours[1], 4)},
                     "scheme": "R=6 reference coefficients, cubic sponge 40, P stress + P velocity"},
            "speedup": round(ref_step / our_step, 2)}), flush=True)


def _fmt_case(r):
    out = {}
    for k, v in r.items():
        if isinstance(v, list):
            v = [round(float(x), 5) if isinstance(x, (int, float)) else x for x in v]
        elif isinstance(v, float):
            v = round(v, 5)
        out[k] = v
    return out


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "passcheck":
        return run_passcheck(args)
    if args.workload == "windows":
        return run_windows(args)
    if args.workload == "unet":
        return run_unet(args)
    if args.workload == "lsrtm":
        return run_lsrtm(args)
    if args.workload == "lsrtm-op":
        return run_lsrtm_op(args)
    if args.workload == "refstep":
        return run_refstep(args)
    if args.workload == "lsrtm-cg":
        return run_lsrtm_cg(args)
    import numpy as np
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=900), device_id=dev)

    ertm = importlib.import_module(PKG)
    synth = importlib.import_module(PKG + ".synthetic")
    wl = workload(args.small, args.grid, args.pml)
    nz, ny, nx = wl.shape
    cells = nx * ny * nz
    if args.kernels_only:
        ctx = ertm.Context(ertm.Config(nx=nx, ny=ny, nz=nz, dx=wl.dx, dy=wl.dy, dz=wl.dz,
                                       dt_ms=wl.dt_ms, nt=wl.nt, order=8, pml=(wl.pml,) * 6,
                                       device=local))
        ctx.set_model(ertm.MIGRATION_MODEL, wl.svp, wl.svs, wl.srho)
        out = {"workload": wl.name, "cells": cells, "steps": args.kernel_steps}
        for name, variant in (("pairs", ertm.STEP_PAIRS), ("single_cell", ertm.STEP_SINGLE)):
            ctx.set_step_variant(variant)
            ctx.time_kernels(_shot(ertm, wl, synth, 0), 2)          # warm-up launches
            ms = ctx.time_kernels(_shot(ertm, wl, synth, 0), args.kernel_steps)
            out[name] = {"ms_per_launch": [m / args.kernel_steps for m in ms],
                         "gcells": [cells / (m / args.kernel_steps) / 1e6 for m in ms]}
        print(json.dumps(out))
        ctx.close()
        return
    cfg = ertm.Config(nx=nx, ny=ny, nz=nz, dx=wl.dx, dy=wl.dy, dz=wl.dz, dt_ms=wl.dt_ms,
                      nt=wl.nt, order=8, boundary=ertm.BOUNDARY_CPML, pml=(wl.pml,) * 6,
                      device=local)
    src_steps = 2 * wl.nt // 3
    updates = cells * (src_steps + wl.nt)
    ctx = ertm.Context(cfg)
    stream = torch.cuda.current_stream(dev)
    ctx.set_stream(stream.cuda_stream)
    ctx.set_step_variant(ertm.STEP_PAIRS if args.step_variant == "pairs" else ertm.STEP_SINGLE)
    ctx.set_model(ertm.TRUE_MODEL, wl.vp, wl.vs, wl.rho)
    ctx.set_model(ertm.MIGRATION_MODEL, wl.svp, wl.svs, wl.srho)
    shot = _shot(ertm, wl, synth, rank)

    # observed data: modelling in the true model (setup, untimed), kept in HBM
    data = torch.zeros((3, wl.nt, shot.nrec), dtype=torch.float32, device=dev)
    ctx.forward_together_using_real_model(shot, out=data)
    imgs = [torch.zeros(wl.shape, dtype=torch.float32, device=dev) for _ in range(3)]

    def step():
        ctx.rtm_shot(shot, data, *imgs)
        if world > 1:
            for t in imgs:
                dist.reduce(t, dst=0)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)

    for _ in range(args.warmup):
        step()
    barrier()
    uuid = str(torch.cuda.get_device_properties(dev).uuid)
    uuid = uuid if uuid.startswith("GPU-") else "GPU-" + uuid
    clocks = ClockSampler(uuid)
    l0 = ctx.kernel_launches
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    barrier()
    launches = ctx.kernel_launches - l0
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    t = torch.tensor([ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms = float(t.item())
    ms_step = ms / args.steps
    value = world * updates / (ms_step / 1e3) / 1e9

    # end to end: pinned host data in, pinned host images out, through the same call
    data_h = torch.empty(data.shape, dtype=torch.float32, pin_memory=True)
    data_h.copy_(data)
    imgs_h = [torch.empty(wl.shape, dtype=torch.float32, pin_memory=True) for _ in range(3)]
    torch.cuda.synchronize(dev)
    ctx.rtm_shot(shot, data_h, *imgs_h)   # warm the host path
    reps = max(1, min(args.steps, 2))
    barrier()
    e0.record(stream)
    for _ in range(reps):
        ctx.rtm_shot(shot, data_h, *imgs_h)
    e1.record(stream)
    barrier()
    ms_e2e = e0.elapsed_time(e1) / reps
    t = torch.tensor([ms_e2e], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    e2e = world * updates / (float(t.item()) / 1e3) / 1e9
    h2d = data.numel() * 4
    d2h = 3 * cells * 4

    # per-kernel device time (CUDA events around each launch, source-pass kernels)
    ks = args.kernel_steps
    ms_stress, ms_vel = ctx.time_kernels(shot, ks)
    peaks_path = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(peaks_path):
        peak, peak_src = float(json.load(open(peaks_path))["hbm_gbs"]), "measured"
    else:
        peak, peak_src = 6650.0, "fallback"
    # The step's compulsory traffic: 84 B per cell-step (9 fields read and written,
    # 3 model arrays; FP32).  achieved = 84 B x cells x (src_steps + nt) / timed shot.
    achieved = COMPULSORY_B * updates / (ms_step / 1e3) / 1e9
    # Algorithmic bytes per cell of each source-pass kernel (FP32):
    #   stress:   read v(3) sigma(6) tp(1) M, mu(2); write sigma(6) tp(1)          = 76 B
    #   velocity: read sigma(6) tp(1) v(3) vP(3) b(1) |e|^2(1); write v(3) vP(3) = 84 B
    bytes_k = {"stress": 76 * cells, "velocity": 84 * cells}
    t_k = {"stress": ms_stress / ks, "velocity": ms_vel / ks}
    per_kernel = {k: {"ms": round(t_k[k], 4), "algorithmic_bytes": bytes_k[k],
                      "gbs": round(bytes_k[k] / (t_k[k] / 1e3) / 1e9, 1),
                      "frac": round(bytes_k[k] / (t_k[k] / 1e3) / 1e9 / peak, 4)} for k in t_k}
    # DRAM bytes per launch: the per-cell traffic of one ncu capture of each kernel on
    # the half-size grid with a proportionally half-width C-PML (same slab fractions),
    # scaled by the cell count (traffic grows with the cells at fixed slab fractions)
    traffic_step = sum(TRAFFIC_B_PER_CELL.values()) * cells
    traffic_ok = (not args.grid and not args.small and args.pml == 40)
    step_ms = (ms_stress + ms_vel) / ks

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            co = CpuOracle(wl)
            rate, n = co.rate_for(args.cpu_seconds)
            cpu = {"value": round(rate, 4), "unit": UNIT, "cores": co.threads, "kind": "port",
                   "sample": f"{n} time steps (source and receiver pass, 2:3) of the full "
                             f"{nx}x{ny}x{nz} grid, FP32 OpenMP oracle (same scheme), after one "
                             f"untimed step"}
            co.close()
        except Exception as e:  # a missing oracle build must not hide the GPU number
            cpu = {"value": None, "unit": UNIT, "cores": None, "kind": "port",
                   "sample": f"failed: {e}"}

    if rank == 0:
        out = {
            "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_step, 2),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded layered model with an ellipsoid; observed data modelled "
                    "in the true model)",
            "config": shot_config(wl, world, shot.nrec),
            "e2e": {"value": round(e2e, 3), "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "roofline": {"bound": "hbm",
                         "kernel": "3D elastic step (k_stress + k_velocity), whole RTM shot",
                         "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4),
                         "traffic": int(traffic_step) if traffic_ok else None,
                         "traffic_unit": "bytes per step (both kernels), scaled from a "
                                         "half-size ncu capture",
                         "peak_source": peak_src, "bytes_per_cell_step": COMPULSORY_B,
                         "kernels": per_kernel,
                         "rtm_algorithmic_bytes_per_cell_step": 160,
                         "rtm_algorithmic_frac": round(160 * cells / (step_ms / 1e3) / 1e9 / peak, 4),
                         "traffic_bytes_per_cell": TRAFFIC_B_PER_CELL},
            "gpu_launches": launches,
            "step_variant": args.step_variant,
            "clocks": clk,
        }
        if cpu is not None:
            out["cpu_baseline"] = cpu
        print(json.dumps(out), flush=True)
    ctx.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
