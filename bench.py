#!/usr/bin/env python
"""Benchmark of the CGFD time-stepping path: Gcell-updates/s per RK4 step.

Workload (default, --config hill600): the 600x600x250 Gaussian-hill model
(hybrid curvilinear grid, vertical spacing 50->150 m, 8 random layers with vp
2500..7000 m/s, double-couple source, 20-cell CFS-PML, 400 surface
receivers) on one B200, FP32.  --config hill400 is the 400x400x200 hill with
3 perturbed layers.  A "step" is one full RK4 time step (4 fused RHS+update
stages, source injection and the receiver record, replayed as a CUDA graph).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU runs are independent replicas (one model per GPU, no exchange);
value is the sum over ranks of cells*K divided by the slowest rank's time.
--impl reference runs the reference's own device runtime (src/calculate.cu,
built from its sources into oracle/_ref/) on the same model; that process
builds the model with the CPU oracle's pre-processing and never loads the
solver library.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "copara-cgfd3d_b200", "python"))

import numpy as np  # noqa: E402

METRIC = "Gcell-updates/s per RK4 step"
UNIT = "Gcell/s"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=200)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", choices=("ours", "reference"), default="ours")
    p.add_argument("--kernel", choices=("fused", "simple", "scalar"), default="fused")
    p.add_argument("--config", choices=("hill600", "hill400", "flat160", "hill256", "batch64"),
                   default="hill600")
    p.add_argument("--autotune", dest="autotune", action="store_true", default=True,
                   help="tune the work list before timing (state unchanged; the default for "
                        "single models; batch64 tunes only when asked)")
    p.add_argument("--no-autotune", dest="autotune", action="store_false")
    p.add_argument("--work-shape", default=None, metavar="ITEMS,CHUNK,PMLW",
                   help="single models: use this work shape (items per resident CTA, minimum "
                        "z-chunk, PML cost weight; a line's work_shape) instead of tuning")
    p.add_argument("--tune-batch", action="store_true",
                   help="batch64: tune the work list and launch shape before timing")
    p.add_argument("--storage", choices=("f32", "f16", "bf16"), default="f32",
                   help="storage type of the field sets (arithmetic is FP32)")
    p.add_argument("--ref-build", choices=("optimised", "shipped"), default="optimised",
                   help="reference arm: the reference's calculate.cu built -O3 for sm_100a "
                        "(default) or as it ships (-arch=sm_60 -G, PTX JIT on the B200)")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--cpu-seconds", type=float, default=15.0)
    p.add_argument("--pml", type=int, default=0, metavar="N",
                   help="single models: an N-cell CFS-PML on the five absorbing faces instead "
                        "of the workload's own")
    p.add_argument("--mlp", action="store_true",
                   help="single models: the learned thin layer (committed weights, width 4) "
                        "after every step; implies --pml 4 unless --pml is given")
    p.add_argument("--no-target", action="store_true",
                   help="skip the batched FP16 learned-thin-layer timing on the same model")
    p.add_argument("--target-accuracy", type=int, default=0, metavar="STEPS",
                   help="instead of the benchmark: reflected energy and 16-bit error of the "
                        "thin-layer configurations over STEPS steps (one JSON line)")
    return p.parse_args()


def build_model(cfg, nt, nabs=None):
    """The workload's model; nabs replaces its CFS-PML widths (the same grid,
    media and sources with another absorbing layer)."""
    import models
    kw = {} if nabs is None else {"nabs": tuple(nabs)}
    if cfg == "hill600":
        return models.config_c5(nt=nt, **kw)
    if cfg == "hill400":
        return models.gaussian_hill(nt=nt, name="gaussian_hill_400x400x200", **kw)
    if cfg == "hill256":
        return models.hill_256(nt=nt, **kw)
    return models.flat_halfspace(nt=nt, name="flat_halfspace_160x160x80",
                                 **({"nabs": tuple(nabs)} if nabs else {}))


def workload_name(cfg, pml=0, mlp=False):
    """The workload's name; pml replaces its CFS-PML width, mlp adds the
    learned layer."""
    name = {"hill600": "gaussian_hill_600x600x250_random_layers_pml20",
            "hill400": "gaussian_hill_400x400x200_pml20",
            "flat160": "flat_halfspace_160x160x80_pml12",
            "hill256": "gaussian_hill_256x256x128_pml20",
            "batch64": "batch_64_hill_models_96-256_pml12"}[cfg]
    if pml:
        name = name[:name.rindex("_pml")] + f"_pml{pml}"
    return name + ("_mlp" if mlp else "")


def config_dict(cfg, m, storage="f32", pml=0, mlp=False):
    """The workload description both arms print (same keys, same values)."""
    return {"workload": workload_name(cfg, pml, mlp), "cells": m.cells,
            "grid": [m.ni, m.nj, m.nk], "pml_cells": list(m.nabs), "storage": storage,
            "receivers": int(len(m.rcv_loc)),
            "l2": "state >> L2 (126 MB), no flush needed"}


def product_library_mapped() -> bool:
    """True when this process has mapped one of the solver's own shared
    libraries (copara-cgfd3d_b200/*.so)."""
    try:
        with open("/proc/self/maps") as f:
            return any("copara-cgfd3d_b200" in line for line in f)
    except OSError:
        return False


def run_batch(args, dist, rank, world, local):
    """64 uneven hill models (seed 7) stepped together as one batch."""
    import cgfd
    import models
    K, W = args.steps, args.warmup
    ms_models = models.batch_models(n=64, seed=7, nt=W + K + 2 + (6 if args.tune_batch else 0))
    storage = {"f32": cgfd.STORE_F32, "f16": cgfd.STORE_F16, "bf16": cgfd.STORE_BF16}[args.storage]
    b = cgfd.Batch([m.desc(device=local, storage=storage) for m in ms_models])
    for m, s in zip(ms_models, b.models):
        m.load(s)
    b.prepare()
    tuned = None
    if args.tune_batch:
        tuned = b.autotune(steps=3)
    b.step(W)
    b.sync()
    barrier(dist)
    with ClockSampler(local) as clk:
        ms = b.step_timed(K)
    ms = allmax(dist, ms)
    cells = sum(m.cells for m in ms_models)
    nbad = sum(s.check_finite() for s in b.models)
    shape = "members" if b.launch == cgfd.BATCH_MEMBERS else "persistent"
    b.close()
    if rank != 0:
        return
    value = world * cells * K / (ms / 1e3) / 1e9
    bps = sum(algorithmic_bytes_per_step(m, 4 if args.storage == "f32" else 2) for m in ms_models)
    achieved = bps / (ms / K / 1e3) / 1e9
    peak, peak_kind = measured_peak()
    n_src = sum(1 for m in ms_models if len(m.mnt_loc) + len(m.frc_loc))
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K,
        "warmup": W, "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded model generator)",
        "config": {"workload": workload_name(args.config), "models": len(ms_models),
                   "cells": cells, "kernel": "fused", "storage": args.storage, "replicas": world,
                   "autotuned_ms_per_step": tuned, "launch_shape": shape,
                   "l2": "state >> L2 (126 MB), no flush needed",
                   "parallelism": "replicas" if world > 1 else "single"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": None,
                     "peak_source": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)",
                     "algorithmic_bytes_per_step": bps,
                     "launch": "whole batched step (4 stages: velocity + stress pair_kernel, "
                               "timg, sources; receiver record)"},
        "clocks": clk.summary(),
        "gpu_launches": K * (4 * (3 + (1 if n_src else 0)) + 1),
        "nonfinite": nbad,
    }
    print(json.dumps(line))


def algorithmic_bytes_per_step(m, elem=4):
    """Minimum HBM bytes of one RK4 step of the fused design: 144 state values
    per cell (27+45+45+27 over the 4 stages: reads of W, FW, tW, writes of W,
    tW, FW) of elem bytes each, the same again for each (cell, PML direction)
    pair (ADE auxiliaries, FP32), and (3 media + m metric) FP32 coefficients
    per cell per stage (m = 3 above ConIndex, 1 below, 0 for a trivial
    metric)."""
    nxy = m.ni * m.nj
    cells = m.cells
    state = 144 * elem * cells
    nab = m.nabs
    pml_pairs = ((nab[0] + nab[1]) * m.nj * m.nk + (nab[2] + nab[3]) * m.ni * m.nk +
                 (nab[4] + nab[5]) * m.ni * m.nj)
    aux = 144 * 4 * pml_pairs
    zz = m.metric["zeta_z"][3:-3, 3:-3, 3:-3]
    flat = bool(np.all(zz == 1.0) and np.all(m.metric["jac"][3:-3, 3:-3, 3:-3] == 1.0)
                and np.all(m.metric["zeta_x"][3:-3, 3:-3, 3:-3] == 0.0))
    if flat:
        coef = 3 * 4 * 4 * cells
    else:
        n_curved = nxy * (m.nk + 3 - m.con_index)
        coef = 4 * 4 * (6 * n_curved + 4 * (cells - n_curved))
    return state + aux + coef


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, dev):
        self.dev = dev
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for r in self.rows:
            try:
                sm.append(float(r[0]))
                mx = float(r[1])
            except (ValueError, IndexError):
                continue
            for n, v in zip(names, r[4:8]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def committed_traffic(workload, kernel):
    """Per-launch DRAM bytes of the stage kernel from the committed ncu
    summary (profiles/stage_traffic.json) and the work shape it was captured
    at (None where the summary does not name one), or (None, None)."""
    p = os.path.join(ROOT, "profiles", "stage_traffic.json")
    if not os.path.exists(p):
        return None, None
    with open(p) as f:
        d = json.load(f)
    e = d.get(workload, {}).get(kernel)
    if e is None:
        return None, None
    return float(e["dram_bytes_per_launch"]), e.get("work_shape")


def cpu_sample_model(cfg, nt):
    """The model the CPU oracle is timed on: the workload itself, except for
    the 600x600x250 hill, whose FP64 state (~45 GB) is cut to a 200x200x250
    window of the same generator (layers, grid spacing, PML, dt)."""
    import models
    if cfg == "hill600":
        return models.config_c5(nt=nt, ni=200, nj=200, n_side=5, rcv_spacing=1000.0,
                                name="gaussian_hill_200x200x250_window")
    return build_model(cfg, nt)


def cpu_baseline(cfg, seconds):
    """FP64 C++/OpenMP oracle (the CPU restatement of the reference path) on
    the same model, for a bounded number of steps."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    m = cpu_sample_model(cfg, nt=64)
    o = pyoracle.OracleSolver(m.desc(), 0)
    m.load(o)
    o.step(1)  # warm caches, first touch
    steps, t0 = 0, time.perf_counter()
    while steps < 60:
        o.step(1)
        steps += 1
        if time.perf_counter() - t0 > seconds:
            break
    el = time.perf_counter() - t0
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return {"value": m.cells * steps / el / 1e9, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{m.name} ({m.ni}x{m.nj}x{m.nk}, of {workload_name(cfg)}), {steps} RK4 "
                      f"steps after 1 warm-up step, FP64 oracle, {el:.1f} s"}


def dist_init(n, backend=None):
    """One process per GPU (replicas): the process group of a torchrun launch.
    backend: "nccl" (default with a GPU) or "gloo" (CPU; the tests' ranks)."""
    import torch
    import torch.distributed as dist
    if n <= 1:
        return None, 0, 1, 0
    rank = int(os.environ["RANK"])
    world = int(os.environ["WORLD_SIZE"])
    local = int(os.environ.get("LOCAL_RANK", rank))
    backend = backend or ("nccl" if torch.cuda.is_available() else "gloo")
    import datetime
    if backend == "nccl":
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    else:
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    return dist, rank, world, local


def allmax(dist, x):
    """The maximum of x over ranks (device-timed values: the slowest rank)."""
    if dist is None:
        return x
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(dist):
    if dist is not None:
        import torch
        dist.barrier()
        if dist.get_backend() == "nccl":
            torch.cuda.synchronize()


def replica_value(world, cells, steps, ms):
    """Whole-job Gcell/s of `world` independent replicas of a model of
    `cells` cells, each stepped `steps` times, the slowest taking ms."""
    return world * cells * steps / (ms / 1e3) / 1e9


def run_reference(args):
    """The reference's own runtime (oracle/_ref/ref_wavesim: src/calculate.cu
    built from its sources) on the same model.  The model is built with the
    CPU oracle's pre-processing, so this process never maps libcgfd.so."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import refio
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    if not refio.available():
        print(json.dumps({"impl": "reference", "unavailable":
                          "reference parity driver oracle/_ref/ref_wavesim not built"}))
        return
    import models
    models.use_preprocessing("oracle")
    nt = args.warmup + args.steps + 2
    m = build_model(args.config, nt)
    shipped = args.ref_build == "shipped"
    r = refio.run(m, args.warmup + args.steps, timeout=3600, fields=False,
                  binary=refio.REF_BIN_SHIPPED if shipped else None)
    mapped = product_library_mapped()
    if mapped:
        raise RuntimeError("the reference arm mapped the solver library")
    secs = float(np.sum(r["step_secs"][args.warmup:args.warmup + args.steps]))
    value = m.cells * args.steps / secs / 1e9
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": secs / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded model generator)", "impl": "reference",
        "reference_build": args.ref_build,
        "config": config_dict(args.config, m),
        "product_library_mapped": mapped,
        "preprocessing": "CPU oracle (FP64 restatement of calmetric / CalCFSfactors / "
                         "wavelets / angle2moment)",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "reference",
                         "sample": f"{workload_name(args.config)}, {args.steps} steps after "
                                   f"{args.warmup} warm-up; the reference's own calculate.cu "
                                   "(CUDA-only path) built from its sources "
                                   + ("as it ships (-arch=sm_60 -G, PTX JIT)" if shipped else
                                      "(-O3, sm_100a)")
                                   + ", driven by one host thread on the B200"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


MLP_WEIGHTS = os.path.join(ROOT, "copara-cgfd3d_b200", "data", "layer_mlp_w4.npz")
THIN = (4, 4, 4, 4, 4, 0)  # the learned layer's CFS-PML widths


def thin_members(m, n=2):
    """n members of the same model with a 4-cell CFS-PML for the learned
    layer: the model's own source, then the source moved by (+60, -40)
    cells with the mechanism rotated (independent shots on one model)."""
    import dataclasses
    out = [m]
    for q in range(1, n):
        loc = m.mnt_loc.copy()
        loc[:, 0] += 60 * q
        loc[:, 1] -= 40 * q
        out.append(dataclasses.replace(m, mnt_loc=loc, mnt_m6=np.roll(m.mnt_m6, q, axis=1)))
    return out


def set_layer(s):
    """The learned thin layer with the committed weights and gains."""
    d = np.load(MLP_WEIGHTS)
    s.set_boundary_mlp(THIN[0], d["weights"].astype(np.float16))
    s.set_boundary_mlp_gains(d["gains"].astype(np.float32))


def thin_batch(ms, storage, device, mlp=True):
    import cgfd
    b = cgfd.Batch([mm.desc(storage=storage, device=device) for mm in ms])
    for mm, s in zip(ms, b.models):
        mm.load(s)
        if mlp:
            set_layer(s)
    b.prepare()
    return b


def run_target(args, plain_value, plain_ms, local):
    """The batched FP16-storage learned-thin-layer solver on the same model:
    two shots of the model with a 4-cell CFS-PML and the learned layer
    stepped as one batch with FP16 field storage, timed like the plain run."""
    import cgfd
    K, W = args.steps, args.warmup
    m4 = build_model(args.config, W + K + 2 + 6, nabs=THIN)
    ms = thin_members(m4)
    b = thin_batch(ms, cgfd.STORE_F16, local)
    tuned = b.autotune(steps=2)  # work list and launch shape; state restored
    shape = "members" if b.launch == cgfd.BATCH_MEMBERS else "persistent"
    b.step(W)
    b.sync()
    ms_b = b.step_timed(K)
    nbad = sum(s.check_finite() for s in b.models)
    b.close()
    value = len(ms) * m4.cells * K / (ms_b / 1e3) / 1e9
    return {"what": "batched FP16-storage learned-thin-layer solver (4-cell CFS-PML + boundary "
                    "MLP, committed weights) on the same model, 2 shots in one batch",
            "value": value, "unit": UNIT, "ms_per_step": ms_b / K, "members": len(ms),
            "launch_shape": shape, "autotuned_ms_per_step": tuned,
            "plain_fp32_pml20_value": plain_value, "plain_fp32_pml20_ms_per_step": plain_ms,
            "speedup_vs_plain_fp32_pml20": value / plain_value, "nonfinite": nbad,
            "accuracy": "bench.py --target-accuracy STEPS (reflected energy against the "
                        "20-cell PML, FP16 against FP32 storage)"}


def near_face_receivers(m, inset=30, spacing=25):
    """Receivers inset cells inside the absorbing faces (outside a 20-cell
    layer): on the surface along the four side faces, and on a grid inset
    cells above the bottom; reference indices."""
    LFD = 3
    top = m.nk + LFD - 1
    pts = set()
    for i in range(inset, m.ni - inset, spacing):
        pts.add((LFD + i, LFD + inset, top))
        pts.add((LFD + i, LFD + m.nj - 1 - inset, top))
    for j in range(inset, m.nj - inset, spacing):
        pts.add((LFD + inset, LFD + j, top))
        pts.add((LFD + m.ni - 1 - inset, LFD + j, top))
    for i in range(inset, m.ni - inset, 4 * spacing):
        for j in range(inset, m.nj - inset, 4 * spacing):
            pts.add((LFD + i, LFD + j, LFD + inset))
    return np.array(sorted(pts), np.int32)


def run_target_accuracy(args, local):
    """Reflected-energy fraction of the thin-layer configurations against the
    plain 20-cell CFS-PML run, and the seismogram error of FP16 storage
    against FP32 storage, over args.target_accuracy steps of the workload:
    at the model's surface receivers and at receivers 30 cells inside the
    absorbing faces (near_face_receivers)."""
    import dataclasses
    import cgfd
    n = args.target_accuracy

    def with_face_receivers(m):
        return dataclasses.replace(m, rcv_loc=np.concatenate([m.rcv_loc, near_face_receivers(m)]))

    m20 = with_face_receivers(build_model(args.config, n + 2))
    nsurf = len(m20.rcv_loc) - len(near_face_receivers(m20))
    s = cgfd.Solver(m20.desc(device=local))
    m20.load(s)
    s.step(n)
    u20 = s.seismograms()[:3, :, :n].astype(np.float64)
    s.close()
    m4 = with_face_receivers(build_model(args.config, n + 2, nabs=THIN))
    out = {"receivers_surface": nsurf, "receivers_near_faces": len(m20.rcv_loc) - nsurf}

    def refl(u, sel):
        return float(((u[:, sel] - u20[:, sel]) ** 2).sum() / (u20[:, sel] ** 2).sum())

    runs = {}
    for name, storage, mlp in (("pml4_f32", cgfd.STORE_F32, False),
                               ("pml4_mlp_f32", cgfd.STORE_F32, True),
                               ("pml4_mlp_f16_batched", cgfd.STORE_F16, True)):
        b = thin_batch([m4] if storage == cgfd.STORE_F32 else thin_members(m4), storage, local, mlp)
        b.step(n)
        b.sync()
        runs[name] = b.models[0].seismograms()[:3, :, :n].astype(np.float64)
        b.close()
        out["reflected_energy_" + name] = refl(runs[name], slice(0, nsurf))
        out["reflected_energy_near_faces_" + name] = refl(runs[name], slice(nsurf, None))
    f16, f32 = runs["pml4_mlp_f16_batched"], runs["pml4_mlp_f32"]
    out["seismogram_rel_l2_f16_vs_f32"] = [float(np.linalg.norm(f16[c] - f32[c]) /
                                                 np.linalg.norm(f32[c])) for c in range(3)]
    line = {"mode": "target accuracy", "workload": workload_name(args.config), "steps": n,
            "reference": "plain FP32 run with the 20-cell CFS-PML, same grid",
            **out}
    print(json.dumps(line))


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    if args.target_accuracy > 0:
        run_target_accuracy(args, 0)
        return
    dist, rank, world, local = dist_init(args.gpus)
    if args.config == "batch64":
        run_batch(args, dist, rank, world, local)
        if dist is not None:
            dist.destroy_process_group()
        return
    import cgfd
    kernel = {"fused": cgfd.KERNEL_FUSED, "simple": cgfd.KERNEL_SIMPLE,
              "scalar": cgfd.KERNEL_SCALAR}[args.kernel]
    K, W = args.steps, args.warmup
    K2 = min(K, 20)
    nt = W + K + K2 + 2 + (4 if args.autotune else 0)
    pml = args.pml or (THIN[0] if args.mlp else 0)
    m = build_model(args.config, nt, nabs=(pml,) * 5 + (0,) if pml else None)
    storage = {"f32": cgfd.STORE_F32, "f16": cgfd.STORE_F16, "bf16": cgfd.STORE_BF16}[args.storage]
    s = cgfd.Solver(m.desc(kernel=kernel, device=local, storage=storage))
    m.load(s)
    if args.mlp:
        set_layer(s)
    s.prepare()
    tuned = None
    if args.work_shape and args.kernel == "fused":
        ws = args.work_shape.split(",")
        s.work_shape = (int(ws[0]), int(ws[1]), float(ws[2]))
    elif args.autotune and args.kernel == "fused":
        tuned = s.autotune(steps=2)
    work_shape = list(s.work_shape) if args.kernel == "fused" else None
    s.step(W)
    s.sync()
    barrier(dist)
    with ClockSampler(local) as clk:
        ms, _ = s.step_timed(K)
    ms = allmax(dist, ms)
    # mean duration of one stage kernel launch (stages issued individually)
    _, stage_ms = s.step_timed(K2, per_stage=True)
    stage_ms = allmax(dist, stage_ms)
    nbad = s.check_finite()
    s.close()
    value = replica_value(world, m.cells, K, ms)

    e2e = None
    if not args.no_e2e:
        barrier(dist)
        t0 = time.perf_counter()
        s2 = cgfd.Solver(m.desc(kernel=kernel, device=local, storage=storage))
        m.load(s2)
        if args.mlp:
            set_layer(s2)
        if work_shape is not None:  # the shape the autotuner chose, as a user reuses it
            s2.prepare()
            s2.work_shape = work_shape
        s2.step(K)
        seis = s2.seismograms()
        s2.sync()
        el = allmax(dist, time.perf_counter() - t0)
        s2.close()
        e2e = {"value": world * m.cells * K / el / 1e9, "unit": UNIT,
               "h2d_bytes_per_step": int(m.upload_bytes() / K),
               "d2h_bytes_per_step": int(seis.nbytes / m.nt),
               "what": "cgfd_create + uploads of the model from host arrays + K steps + "
                       "seismogram download, wall clock"}
    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return
    bps = algorithmic_bytes_per_step(m, 4 if args.storage == "f32" else 2)
    achieved = bps / 4 / (stage_ms / 1e3) / 1e9
    peak, peak_kind = measured_peak()
    traffic, traffic_shape = committed_traffic(
        workload_name(args.config, pml, args.mlp),
        args.kernel if args.storage == "f32" else f"{args.kernel}_{args.storage}")
    traffic_src = None
    if traffic:
        traffic_src = ("profiles/stage_traffic.json: ncu dram__bytes of an earlier capture of "
                       "this workload, per stage, not measured in this run")
        if traffic_shape is not None:
            traffic_src += f" (captured at work shape {traffic_shape})"
    n_src = 1 if (len(m.mnt_loc) + len(m.frc_loc)) else 0
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K,
        "warmup": W, "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded model generator)",
        "config": config_dict(args.config, m, args.storage, pml, args.mlp),
        "kernel": args.kernel, "replicas": world, "autotuned_ms_per_step": tuned,
        "work_shape": work_shape,
        "parallelism": "replicas" if world > 1 else "single",
        "product_library_mapped": product_library_mapped(),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "traffic_source": traffic_src,
                     "peak_source": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)",
                     "algorithmic_bytes_per_step": bps, "stage_kernel_ms": stage_ms},
        "clocks": clk.summary(),
        "gpu_launches": K * (4 * (1 if args.kernel == "simple" else 3) + 4 * n_src + 1 +
                             (2 if args.mlp else 0)),
        "nonfinite": nbad,
    }
    if e2e:
        line["e2e"] = e2e
    if (not args.no_target and world == 1 and args.storage == "f32" and args.kernel == "fused"
            and not pml):
        line["target"] = run_target(args, value, ms / K, local)
    if not args.no_cpu_baseline and world == 1:  # the host-core baseline: N = 1 only
        line["cpu_baseline"] = cpu_baseline(args.config, args.cpu_seconds)
    print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
