#!/usr/bin/env python
"""Benchmark of the B200 LBM time step (FlowCraft's LbmSolver::Step hot path).

Workload (default, the large configuration the target is stated on): D3Q19,
1024x512x512 = 268.4M cells, a procedural high-wing aircraft mesh of 57,516
triangles (ellipsoidal fuselage, tapered NACA 2412 wing, NACA 0012 tails)
voxelized on the device by the library's voxelizer (fc_lbm_voxelize, solid
mask and signed distance, so the Bouzidi links come from the mesh), inlet
U = 0.05, Re = 1e5 on the 60-cell root chord (tau = 0.50009), Smagorinsky
Cs = 0.1, free-slip side walls. Synthetic input: the mesh is generated
procedurally; there is no mesh file or dataset.

One "step" is one full lattice update (every cell streamed, collided and
written). ``value`` = whole-job GLUPS (cells x steps / s, solid cells
included) with the lattice resident in HBM, timed with CUDA events on the
solver's stream, max over ranks. The headline is the metric's pairing: FP16
offset populations with the learned sub-grid closure (the MLP trained by
flowcraft_b200.closure_train, flowcraft_b200/data/closure_c4.json, evaluated
per cell on the tensor cores inside the collision); FP16 with plain
Smagorinsky and the plain FP32 path (bit-identical to the reference) are
timed beside it.

The learned variants are timed in the developed flow: after ``--spinup``
untimed steps from the seed (default 2000 of the configuration's 3000-step
run). The MLP runs only in warps with a cell whose inputs are in its
training range, and that share grows from about a fifth of the warps in the
first hundred steps to nearly all of them once the wake has developed. The
plain variants do the same work in every flow state.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
For N > 1 run under torchrun; every rank steps its own lattice (replicas, no
data-path collective).
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "D3Q19 GLUPS & %HBM roofline: FP16+learned SGS vs plain FP32, same GPU/accuracy"
FALLBACK_HBM_GBS = 6650.0

CONFIGS = {
    # the large configuration: 1024x512x512, aircraft, Re 1e5 on a 60-cell root chord
    "large": dict(nx=1024, ny=512, nz=512, geom="aircraft", u=0.05, re=1e5, lref=60.0, cs=0.1,
                  desc="D3Q19 1024x512x512 (268.4M cells), procedural high-wing aircraft mesh (57,516 triangles) "
                       "voxelized on the device, U=0.05, Re=1e5 on the 60-cell root chord (tau=0.50009), "
                       "Smagorinsky Cs=0.1"),
    # the plain-FP32 parity lattice: 128x64x64, sphere r=10, Re=100
    "c1": dict(nx=128, ny=64, nz=64, geom="sphere", u=0.05, re=100.0, lref=20.0, cs=0.1,
               desc="D3Q19 128x64x64 (524k cells), sphere r=10 at (40,32,32), U=0.05, Re=100 (tau=0.53), Cs=0.1"),
    # the batched-throughput set: 16 NACA 2412 lattices of seeded sizes 64x32x32 .. 256x128x128
    "c3": dict(nx=0, ny=0, nz=0, geom="batch", u=0.0, re=0.0, lref=0.0, cs=0.1,
               desc="D3Q19 batch of 16 NACA 2412 wing lattices, sizes 64x32x32..256x128x128 (2:1:1) drawn with seed "
                    "20261203, chord 0.375 nx, AoA -8..14 deg, U 0.04-0.08, Re 1e3-2e4, FP16 offset, Smagorinsky "
                    "Cs=0.1, all lattices stepped as one batch per step in a CUDA graph (autotuned: one launch over "
                    "every lattice's tiles, persistent or one block per tile, or the lattices' own bulk kernels "
                    "side by side)"),
    # the precision-study lattice size: 384x192x192 NACA 0012 wing, chord 96, 4 deg
    "c2": dict(nx=384, ny=192, nz=192, geom="naca0012", u=0.06, re=1e4, lref=96.0, cs=0.1,
               desc="D3Q19 384x192x192 (14.2M cells), NACA 0012 wing chord 96 span 128 at 4 deg, U=0.06, "
                    "Re=1e4 (tau=0.50173), Smagorinsky Cs=0.1"),
}

BYTES_PER_ELEM = {"fp32": 4, "fp16_offset": 2, "bf16_offset": 2, "fp16_learned": 2, "bf16_learned": 2,
                  "fp32_aa": 4, "fp16_aa": 2, "bf16_aa": 2, "fp16_tma": 2, "fp16_aa_learned": 2,
                  "bf16_aa_learned": 2, "fp16_tc_learned": 2}
# per-cell bytes beyond the populations: the closure's wall-distance byte
EXTRA_BYTES = {"fp16_learned": 1, "bf16_learned": 1, "fp16_aa_learned": 1, "bf16_aa_learned": 1, "fp16_tc_learned": 1}
CLOSURE_WEIGHTS = os.path.join(ROOT, "flowcraft_b200", "data", "closure_c4.json")


def parse_args(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--config", choices=sorted(CONFIGS), default="large")
    ap.add_argument("--variants", default="fp16_learned,fp16_offset,fp32,fp16_aa,fp32_aa,fp16_aa_learned",
                    help="first one is the headline; *_aa*: one population set streamed in place; "
                         "*_learned: the learned closure; *_tc_*: its MLP on the tcgen05 tensor cores per block; "
                         "*_tma: interior rows staged by TMA")
    ap.add_argument("--spinup", type=int, default=2000,
                    help="untimed steps from the seed before the warm-up of the learned variants (flow state)")
    ap.add_argument("--batch-shape", default=None,
                    help="c3 only: ROWSxMULT (e.g. 4x2; 8x0 for one block per tile; 0x1 for per-member launches) "
                         "instead of the autotuner")
    ap.add_argument("--shard", action="store_true",
                    help="one lattice split into z-slabs across the ranks (NCCL point-to-point halo exchange), "
                         "FP16 offset storage with Smagorinsky; on one GPU, --shard-ranks slabs emulated with "
                         "device copies as the exchange")
    ap.add_argument("--shard-ranks", type=int, default=2, help="slabs emulated on one GPU with --shard at N=1")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--batch-steps", type=int, default=200,
                    help="steps of the 16-lattice sweep set (C3) timed after the default run's variants; 0 skips")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    return ap.parse_args(argv)


def tau_for(cfg) -> float:
    nu = cfg["u"] * cfg["lref"] / cfg["re"]
    return 0.5 + 3.0 * nu


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clock / throttle-reason samples while the timed region runs."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        import torch
        self.lines = []
        self.proc = None
        try:
            uuid = str(torch.cuda.get_device_properties(device_index).uuid)
            ident = uuid if uuid.startswith("GPU-") else f"GPU-{uuid}"
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader",
                                          "-lms", "50", "--id=" + ident], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.time(), line.strip()))

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        time.sleep(0.12)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, smax, reasons, power = [], [], set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for _, line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(re.sub(r"[^0-9.]", "", parts[1])))
                smax.append(float(re.sub(r"[^0-9.]", "", parts[2])))
                power.append(float(re.sub(r"[^0-9.]", "", parts[3]) or 0))
            except ValueError:
                continue
            for name, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm), "power_w_max": max(power) if power else None}


# ---------------------------------------------------------------- helpers
def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def ncu_traffic_per_cell(variant: str, developed: bool = False):
    """DRAM bytes per bulk cell update from the committed ncu summaries of
    the bulk kernels (a line 'traffic_bytes_per_cell <variant> = X'; the
    learned kernel in the developed flow as <variant>_developed), or None."""
    key = variant + ("_developed" if developed else "")
    for name in ("bulk_pairs_ncu_c2.md", "bulk_pairs_learned_developed_c2.md"):
        try:
            text = open(os.path.join(ROOT, "profiles", name)).read()
        except OSError:
            continue
        m = re.search(rf"traffic_bytes_per_cell\s+{key}\s*=\s*([0-9.]+)", text)
        if m:
            return float(m.group(1))
    return None


def aircraft_on_device(cfg, device):
    """The aircraft mesh voxelized on the device by the library: (solid u8,
    sdf f32) torch tensors (nz, ny, nx) on `device` (a cuda device)."""
    import torch

    from flowcraft_b200 import meshes
    from flowcraft_b200.voxelizer import VoxelizeOnGrid
    nx, ny, nz = cfg["nx"], cfg["ny"], cfg["nz"]
    pos, idx = meshes.aircraft_c5(nx)
    g = VoxelizeOnGrid(pos, idx, (nx, ny, nz), 1.0, meshes.aircraft_c5_origin(nx, ny, nz),
                       device=torch.device(device).index or 0)
    return g.solid.view(nz, ny, nx), g.signedDistance.view(nz, ny, nx)


def aircraft_on_host(cfg, z_lo, z_hi):
    """Layers [z_lo, z_hi) of the same voxelization computed on the host by the
    CPU restatement of the voxelizer (for the reference arm, which runs none
    of the library's kernels). It voxelizes the aircraft's bounding box plus
    a margin of 8 cells: a signed distance is finite only within a few cells
    of a triangle, the cell centres are exact (whole-cell origin), and the
    flood fill starts outside the aircraft, so that box classifies its cells
    as the full lattice does, and every cell outside it is fluid with
    distance +infinity."""
    import numpy as np

    from flowcraft_b200 import meshes
    from oracle import oracle as orc
    nx, ny, nz = cfg["nx"], cfg["ny"], cfg["nz"]
    pos, idx = meshes.aircraft_c5(nx)
    ox, oy, oz = meshes.aircraft_c5_origin(nx, ny, nz)
    # lattice index ranges of the box: grid x spans world y, grid y world x
    lo = [int(np.floor(pos[:, 1].min() - oy)) - 8, int(np.floor(pos[:, 0].min() - ox)) - 8,
          int(np.floor(pos[:, 2].min() - oz)) - 8]
    hi = [int(np.ceil(pos[:, 1].max() - oy)) + 8, int(np.ceil(pos[:, 0].max() - ox)) + 8,
          int(np.ceil(pos[:, 2].max() - oz)) + 8]
    lo = [max(0, v) for v in lo]
    hi = [min(d, v) for d, v in zip((nx, ny, nz), hi)]
    bs, bd = orc.voxelize(pos, idx, (hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]), 1.0,
                          np.asarray((ox + lo[1], oy + lo[0], oz + lo[2]), np.float32))
    solid = np.zeros((z_hi - z_lo, ny, nx), np.uint8)
    sdf = np.full((z_hi - z_lo, ny, nx), np.inf, np.float32)
    a, b = max(z_lo, lo[2]), min(z_hi, hi[2])
    if a < b:
        solid[a - z_lo:b - z_lo, lo[1]:hi[1], lo[0]:hi[0]] = bs[a - lo[2]:b - lo[2]]
        sdf[a - z_lo:b - z_lo, lo[1]:hi[1], lo[0]:hi[0]] = bd[a - lo[2]:b - lo[2]]
    return solid, sdf


def build_geometry(cfg, device, z_lo=0, z_hi=None):
    """(solid u8, sdf f32) torch tensors (nz, ny, nx), or layers [z_lo, z_hi)."""
    import torch

    from flowcraft_b200 import geometry
    z_hi = cfg["nz"] if z_hi is None else z_hi
    if cfg["geom"] == "aircraft":
        if str(device).startswith("cuda"):
            solid, sdf = aircraft_on_device(cfg, device)
            return solid[z_lo:z_hi], sdf[z_lo:z_hi]
        solid, sdf = aircraft_on_host(cfg, z_lo, z_hi)
        return torch.from_numpy(solid), torch.from_numpy(sdf)
    if cfg["geom"] == "sphere":
        solid, sdf = geometry.sphere_grid(cfg["nx"], cfg["ny"], cfg["nz"], 40, 32, 32, 10)
        return (torch.from_numpy(solid[z_lo:z_hi].copy()).to(device),
                torch.from_numpy(sdf[z_lo:z_hi].copy()).to(device))
    solid, sdf = geometry.naca_wing_grid(cfg["nx"], cfg["ny"], cfg["nz"], chord=96, span=128, aoa_deg=4,
                                         digits="0012", xp=torch, device=device)
    return solid[z_lo:z_hi].contiguous(), sdf[z_lo:z_hi].contiguous()


def storage_of(variant):
    from flowcraft_b200 import Storage
    return {"fp32": Storage.FP32, "fp16_offset": Storage.FP16_OFFSET, "bf16_offset": Storage.BF16_OFFSET,
            "fp16_learned": Storage.FP16_OFFSET, "bf16_learned": Storage.BF16_OFFSET, "fp32_aa": Storage.FP32,
            "fp16_aa": Storage.FP16_OFFSET, "bf16_aa": Storage.BF16_OFFSET, "fp16_tma": Storage.FP16_OFFSET,
            "fp16_aa_learned": Storage.FP16_OFFSET, "bf16_aa_learned": Storage.BF16_OFFSET,
            "fp16_tc_learned": Storage.FP16_OFFSET}[variant]


def streaming_of(variant):
    """The *_aa* variants keep one population set streamed in place."""
    from flowcraft_b200 import Streaming
    return Streaming.AA if "_aa" in variant else Streaming.PINGPONG


def spinup_of(args, variant) -> int:
    """Untimed steps before the warm-up: the learned variants' cost depends on
    the flow state (how many warps run the MLP), the others' does not."""
    return args.spinup if variant.endswith("_learned") else 0


def workload_config(args, cfg, world) -> dict:
    """The `config` of the bench line: the workload and the headline variant's
    formats, the same for both arms (no run-dependent values)."""
    head = [v.strip() for v in args.variants.split(",") if v.strip()][0]
    learned = head.endswith("_learned")
    spin = spinup_of(args, head)
    return {"workload": cfg["desc"], "lattice": "D3Q19", "nx": cfg["nx"], "ny": cfg["ny"], "nz": cfg["nz"],
            "cells": cfg["nx"] * cfg["ny"] * cfg["nz"], "storage": head, "collision": "regularized, FP32",
            "closure": ("learned 5-32-32-1 MLP per cell (BF16 mma.sync, FP32 accumulate), Smagorinsky "
                        f"Cs={cfg['cs']} outside its range; data/closure_c4.json" if learned else "Smagorinsky"),
            "streaming": "AA pattern, one set in place" if "_aa" in head else "pull, ping-pong",
            "flow_state": (f"timed after {spin} + {args.warmup} steps from the mid-speed seed" if spin
                           else f"timed after {args.warmup} steps from the seed"),
            "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
            "l2": "no flush: populations 10.2 GB (fp16) / 20.4 GB (fp32) per copy, L2 126 MB"}


def kernel_of(variant) -> str:
    name = ("k_bulk_pairs" + ("_aa" if "_aa" in variant else "") + ("_learned" if variant.endswith("_learned") else "")
            + ("_tc" if "_tc_" in variant else ""))
    return f"{name}<19,{variant}>"


def make_solver(cfg, solid, sdf, variant, device_index):
    from flowcraft_b200 import LatticeModel, LbmSolver, Params, VoxelGrid
    s = LbmSolver()
    grid = VoxelGrid(cfg["nx"], cfg["ny"], cfg["nz"], solid=solid, signedDistance=sdf)
    from flowcraft_b200.lbm import OPTION_TC_CLOSURE, OPTION_TMA_STAGING
    flags = OPTION_TMA_STAGING if variant.endswith("_tma") else 0  # interior rows staged by TMA tensor copies
    if "_tc_" in variant:
        flags |= OPTION_TC_CLOSURE  # the closure's MLP on the tcgen05 tensor cores, per block
    if not s.Init(device_index, grid, LatticeModel.D3Q19, storage_of(variant), streaming_of(variant), flags):
        raise RuntimeError(s.LastError())
    s.Reset(Params(tau=tau_for(cfg), inletVelocity=cfg["u"], smagorinskyCs=cfg["cs"]), True)
    if variant.endswith("_learned"):
        from flowcraft_b200.closure import ClosureWeights
        s.SetClosure(ClosureWeights.load(CLOSURE_WEIGHTS))
    return s


def barrier_sync(dist_on):
    import torch
    if dist_on:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()


def allreduce_max(x: float, dist_on) -> float:
    if not dist_on:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------- CPU baseline
def subbox_range(cfg, cores):
    """A z-truncated sub-box of the same lattice around the wing, deep enough
    that every host thread gets z-layers (the reference splits work by z)."""
    nz_sub = int(min(cfg["nz"], max(16, 2 * cores)))
    z0 = max(0, min(cfg["nz"] - nz_sub, int(0.55 * cfg["nz"]) - nz_sub // 2))
    return z0, z0 + nz_sub


def cpu_subbox(cfg, solid, sdf, cores):
    z0, z1 = subbox_range(cfg, cores)
    s = solid[z0:z1].contiguous().cpu().numpy()
    d = sdf[z0:z1].contiguous().cpu().numpy()
    return s, d, z0


def run_cpu_reference(cfg, solid_np, sdf_np, steps, warmup, seconds=None):
    """Times FlowCraft's own LbmReference (oracle/_ref, -O3) — or the restated
    oracle if the reference build is absent — on the given sub-box."""
    from oracle import oracle as orc
    kind = "reference" if orc.available("ref_fast") else "port"
    prec = "ref_fast" if kind == "reference" else "f32"
    p = orc.Params(tau=tau_for(cfg), inlet_velocity=cfg["u"], smagorinsky_cs=cfg["cs"])
    o = orc.Oracle(solid_np, sdf_np, 19, p, True, prec)
    for _ in range(warmup):
        o.step(1)
    done = 0
    t0 = time.perf_counter()
    while True:
        o.step(1)
        done += 1
        el = time.perf_counter() - t0
        if seconds is None and done >= steps:
            break
        if seconds is not None and (el >= seconds or done >= steps):
            break
    el = time.perf_counter() - t0
    cells = solid_np.size
    o.close()
    return {"glups": cells * done / el / 1e9, "steps": done, "seconds": el, "cells": cells, "kind": kind}


# ---------------------------------------------------------------- main arms
def run_reference_arm(args, cfg, rank, world):
    import numpy as np
    if rank != 0:
        return 0
    cores = os.cpu_count() or 1
    # the same procedural geometry, built on the host for the sub-box only
    z0, z1 = subbox_range(cfg, cores)
    solid, sdf = build_geometry(cfg, "cpu", z0, z1)
    s_np, d_np = solid.numpy(), sdf.numpy()
    r = run_cpu_reference(cfg, s_np, d_np, args.steps, args.warmup)
    sample = (f"z-truncated sub-box {cfg['nx']}x{cfg['ny']}x{s_np.shape[0]} (z0={z0}) of the {cfg['nx']}x{cfg['ny']}x"
              f"{cfg['nz']} lattice, {r['steps']} LbmReference::Step calls after {args.warmup} warm-up")
    line = {
        "impl": "reference", "metric": METRIC, "value": r["glups"], "unit": "GLUPS", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * r["seconds"] / r["steps"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(args, cfg, world),
        "cpu_baseline": {"value": r["glups"], "unit": "GLUPS", "cores": cores, "kind": r["kind"], "sample": sample,
                         "sample_cells": r["cells"]},
        "e2e": {"value": r["glups"], "unit": "GLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    del np
    return 0


def time_variant(args, cfg, solid, sdf, variant, dev_index, dist_on, sample_clocks):
    s = make_solver(cfg, solid, sdf, variant, dev_index)
    info = s.BoundaryInfo()
    s.Step(None, spinup_of(args, variant) + args.warmup)
    s.Sync()
    barrier_sync(dist_on)
    sampler = ClockSampler(dev_index) if sample_clocks else None
    l0 = s.LaunchCount()
    t = s.StepTimed(args.steps)  # events around every launch, waits at the end
    launches = s.LaunchCount() - l0
    coverage = s.ClosureCoverage() if variant.endswith("_learned") else None
    clocks = sampler.stop() if sampler else None
    barrier_sync(dist_on)
    total_ms = allreduce_max(t["total_ms"], dist_on)
    stats = s.ReadbackStats()
    s.close()
    cells = cfg["nx"] * cfg["ny"] * cfg["nz"]
    elem = BYTES_PER_ELEM[variant]
    bulk_avg_s = t["bulk_ms"] / args.steps / 1e3
    per_cell = 19 * 2 * elem + EXTRA_BYTES.get(variant, 0)
    bulk_bytes = info["bulk_cells"] * per_cell
    return {
        "variant": variant, "total_ms": total_ms, "ms_per_step": total_ms / args.steps,
        "glups_rank": cells * args.steps / (t["total_ms"] / 1e3) / 1e9,
        "bulk_ms_per_launch": t["bulk_ms"] / args.steps, "boundary_ms_per_launch": t["boundary_ms"] / args.steps,
        "bulk_cells": info["bulk_cells"], "boundary_cells": info["boundary_cells"],
        "bouzidi_links": info["bouzidi_links"], "bulk_bytes_per_launch": bulk_bytes,
        "bulk_gbs": bulk_bytes / bulk_avg_s / 1e9 if bulk_avg_s > 0 else None,
        "launches": launches, "clocks": clocks, "bytes_per_cell": per_cell, "closure_coverage": coverage,
        "spinup_steps": spinup_of(args, variant),
        "stats_after": {"avg_density": stats.avgDensity, "avg_speed": stats.avgSpeed, "has_nan": stats.hasNaN,
                        "force_x": stats.forceX, "force_z": stats.forceZ},
    }


def run_e2e(args, cfg, solid, sdf, variant, dev_index, world=1, dist_on=False):
    """The same metric end to end through the public API with host buffers:
    Init from pinned host geometry (H2D), Reset, then per step Step(1) plus
    ProbeSliceHealth of one z-layer (D2H), then ReadbackStats and the full
    4-float field into host memory (D2H). Wall clock around the host calls,
    the slowest rank's under torchrun (every rank runs its own lattice), and
    the value and bytes are the whole job's.
    For the learned variants the spin-up steps are part of the job and of the
    timed region, so the number is the whole run's rate from the seed."""
    import numpy as np
    import torch

    from flowcraft_b200 import LatticeModel, LbmSolver, Params, VoxelGrid
    h_solid = solid.cpu().pin_memory()
    h_sdf = sdf.cpu().pin_memory()
    n = cfg["nx"] * cfg["ny"] * cfg["nz"]
    out = np.empty(n * 4, dtype=np.float32)
    out[::1024] = 0  # fault the pages in before timing
    out.fill(0)
    st = storage_of(variant)
    steps = spinup_of(args, variant) + args.steps
    grid = VoxelGrid(cfg["nx"], cfg["ny"], cfg["nz"], solid=h_solid.numpy(), signedDistance=h_sdf.numpy())
    torch.cuda.synchronize()
    barrier_sync(dist_on)
    s = LbmSolver()
    t0 = time.perf_counter()
    if not s.Init(dev_index, grid, LatticeModel.D3Q19, st, streaming_of(variant)):
        raise RuntimeError(s.LastError())
    s.Reset(Params(tau=tau_for(cfg), inletVelocity=cfg["u"], smagorinskyCs=cfg["cs"]), True)
    if variant.endswith("_learned"):
        from flowcraft_b200.closure import ClosureWeights
        s.SetClosure(ClosureWeights.load(CLOSURE_WEIGHTS))
    diverged = False
    for k in range(steps):
        s.Step(None, 1)
        diverged |= s.ProbeSliceHealth(k % cfg["nz"])
    stats = s.ReadbackStats()
    s.ReadbackFieldRange(0, cfg["nz"], out)
    el = allreduce_max(time.perf_counter() - t0, dist_on)
    s.close()
    h2d = world * n * (1 + 4)
    d2h = world * (4 * steps + n * 16 + 96)  # the probe's verdict flag per step, the stats, the field
    return {"value": round(world * n * steps / el / 1e9, 3), "unit": "GLUPS", "seconds": round(el, 3), "steps": steps,
            "h2d_bytes_per_step": h2d // steps, "d2h_bytes_per_step": d2h // steps,
            "diverged": diverged, "avg_density": round(stats.avgDensity, 6),
            "timed": "Init(host grid)+Reset+SetClosure+steps*(Step(1)+ProbeSliceHealth)+ReadbackStats+"
                     "ReadbackFieldRange(all z); steps include the learned variants' spin-up"}


def time_batch(args, cfg, local_rank, dist_on, steps, sample_clocks):
    """The c3 set stepped as one batch (autotuned), timed with events; and the
    same lattices stepped one after another for contrast."""
    import torch

    from flowcraft_b200.batch import LbmBatch
    from flowcraft_b200.sweep import c3_lattices, make_members
    mem = make_members(c3_lattices(), "FP16_OFFSET", cfg["cs"], local_rank)
    solvers = [m[0] for m in mem]
    cells = sum(s.CellCount() for s in solvers)
    b = LbmBatch(solvers)
    if args.batch_shape:
        rows, mult = (int(v) for v in args.batch_shape.lower().split("x"))
        b.Config(rows, mult)
        tuned = {"rows": rows, "grid_mult": mult, "fixed": True}
    else:
        tuned = b.Tune(4)
    b.Step(2 * args.warmup)
    torch.cuda.synchronize()
    barrier_sync(dist_on)
    sampler = ClockSampler(local_rank) if sample_clocks else None
    steps = steps + (steps & 1)
    start = torch.cuda.Event(enable_timing=True)
    stop = torch.cuda.Event(enable_timing=True)
    # the batch runs on its own stream, ordered after and before the members'
    # streams; events on the first member's stream bracket it
    s0 = torch.cuda.ExternalStream(solvers[0].Stream())
    start.record(s0)
    b.Step(steps)
    stop.record(s0)
    stop.synchronize()
    ms = start.elapsed_time(stop)
    clocks = sampler.stop() if sampler else None
    # the same members stepped one after another on one stream, for contrast
    seq = torch.cuda.Stream()
    torch.cuda.synchronize()
    seq_start = torch.cuda.Event(enable_timing=True)
    seq_stop = torch.cuda.Event(enable_timing=True)
    seq_start.record(seq)
    for s in solvers:
        s.Step(seq.cuda_stream, steps)
    seq_stop.record(seq)
    seq_stop.synchronize()
    seq_ms = seq_start.elapsed_time(seq_stop)
    barrier_sync(dist_on)
    ms = allreduce_max(ms, dist_on)
    diverged = any(s.HasDiverged() for s in solvers)
    bulk_cells = sum(s.BoundaryInfo()["bulk_cells"] for s in solvers)
    b.close()
    for s in solvers:
        s.close()
    return dict(cells=cells, bulk_cells=bulk_cells, steps=steps, ms=ms, seq_ms=seq_ms, tuned=tuned, clocks=clocks,
                diverged=diverged, sizes=[m[1]["nx"] for m in mem], lattices=len(solvers))


def run_batch(args, cfg, rank, world, local_rank):
    """The c3 set: every rank steps its own batch of 16 lattices."""
    import torch
    dist_on = world > 1
    torch.cuda.set_device(local_rank)
    r = time_batch(args, cfg, local_rank, dist_on, args.steps, rank == 0)
    if rank != 0:
        return 0
    cells, steps, ms, seq_ms, tuned, clocks = r["cells"], r["steps"], r["ms"], r["seq_ms"], r["tuned"], r["clocks"]
    value = world * cells * steps / (ms / 1e3) / 1e9
    line = {"metric": METRIC, "value": value, "unit": "GLUPS", "n_gpus": world, "steps": steps,
            "warmup": args.warmup, "ms_per_step": ms / steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic: analytic NACA 2412 lattices on the device",
            "config": {"workload": cfg["desc"], "lattices": r["lattices"], "cells": cells,
                       "sizes": r["sizes"], "autotune": tuned,
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
            "diverged": r["diverged"], "gpu_launches": (2 if tuned["rows"] else r["lattices"] + 1) * steps,
            "clocks": clocks,
            "sequential": {"glups": world * cells * steps / (seq_ms / 1e3) / 1e9, "ms_per_step": seq_ms / steps,
                           "how": "the same lattices stepped one after another on one stream with LbmSolver.Step"}}
    print(json.dumps(line), flush=True)
    return 0


def run_shard(args, cfg, rank, world, local_rank):
    """One lattice split into z-slabs (flowcraft_b200.shard): each rank steps
    its slab and exchanges per step the 5 planes that stream across each cut
    with its neighbours (NCCL point-to-point on the slab stream, overlapped
    with the slab's interior layers). Events on the slab stream split a step
    into the edge layers and their packing, the interior layers, the part
    of the exchange the interior did not hide, and the unpacking. With one
    process, --shard-ranks slabs are emulated on one GPU (device copies as
    the exchange, no overlap)."""
    import torch

    from flowcraft_b200 import LatticeModel, Params, Storage, shard
    dist_on = world > 1
    torch.cuda.set_device(local_rank)
    solid, sdf = build_geometry(cfg, f"cuda:{local_rank}")
    params = Params(tau=tau_for(cfg), inletVelocity=cfg["u"], smagorinskyCs=cfg["cs"])
    cells = cfg["nx"] * cfg["ny"] * cfg["nz"]
    keys = ("edges_ms", "interior_ms", "exposed_exchange_ms", "unpack_ms")
    split = dict.fromkeys(keys, 0.0)
    if dist_on:
        s, lay, st = shard.nccl_rank(solid, sdf, LatticeModel.D3Q19, Storage.FP16_OFFSET, params)
        del solid, sdf
        torch.cuda.empty_cache()
        st.step(args.warmup)
        barrier_sync(dist_on)
        with st.on_stream():
            start = torch.cuda.Event(enable_timing=True)
            stop = torch.cuda.Event(enable_timing=True)
            evs = [[torch.cuda.Event(enable_timing=True) for _ in range(5)] for _ in range(args.steps)]
            start.record()
            for ev in evs:
                ev[0].record()
                st.edges()
                h = st.ex.post(st.posts(st.dir_rows))
                ev[1].record()
                st.interior()
                ev[2].record()
                st.ex.wait(h)
                ev[3].record()
                st.finish()
                ev[4].record()
            stop.record()
        stop.synchronize()
        for ev in evs:
            for k, key in enumerate(keys):
                split[key] += ev[k].elapsed_time(ev[k + 1])
        ms = start.elapsed_time(stop)
        nranks, slabs = world, world
        closers = [s]
    else:
        ranks = shard.emulated_ranks(solid, sdf, args.shard_ranks, local_rank, LatticeModel.D3Q19,
                                     Storage.FP16_OFFSET, params)
        del solid, sdf
        torch.cuda.empty_cache()
        steppers = [r[2] for r in ranks]
        shard.step_emulated(steppers, args.warmup)
        cmd = steppers[0].cmd
        start = torch.cuda.Event(enable_timing=True)
        stop = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        start.record(cmd)
        shard.step_emulated(steppers, args.steps)
        stop.record(cmd)
        stop.synchronize()
        ms = start.elapsed_time(stop)
        split = None
        nranks, slabs = 1, args.shard_ranks
        closers = [r[0] for r in ranks]
    ms = allreduce_max(ms, dist_on)
    if split is not None:
        split = {k: allreduce_max(v, dist_on) / args.steps for k, v in split.items()}
    for s in closers:
        s.close()
    if rank != 0:
        return 0
    halo = shard.DIR_PLANES * cfg["nx"] * cfg["ny"] * 2
    line = {"metric": METRIC, "value": cells * args.steps / (ms / 1e3) / 1e9, "unit": "GLUPS", "n_gpus": nranks,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic: procedural aircraft mesh voxelized on the device, no dataset",
            "config": {"workload": cfg["desc"], "lattice": "D3Q19", "storage": "fp16_offset", "closure": "Smagorinsky",
                       "parallelism": (f"z-slabs x{world}, NCCL point-to-point halo exchange" if dist_on else
                                       f"{slabs} z-slabs emulated on one GPU, device copies as the exchange"),
                       "halo_bytes_per_side_per_step": halo},
            "step_split_ms": split, "gpu_launches": None}
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args, cfg, rank, world, local_rank):
    import torch
    if cfg["geom"] == "batch":
        return run_batch(args, cfg, rank, world, local_rank)
    if args.shard:
        return run_shard(args, cfg, rank, world, local_rank)
    dist_on = world > 1
    torch.cuda.set_device(local_rank)
    dev_index = local_rank
    solid, sdf = build_geometry(cfg, f"cuda:{local_rank}")
    torch.cuda.synchronize()
    variants = [v.strip() for v in args.variants.split(",") if v.strip()]
    results = {}
    for i, v in enumerate(variants):
        results[v] = time_variant(args, cfg, solid, sdf, v, dev_index, dist_on, sample_clocks=(rank == 0))
        torch.cuda.empty_cache()
    head = results[variants[0]]
    cells = cfg["nx"] * cfg["ny"] * cfg["nz"]
    total_s = head["total_ms"] / 1e3
    value = world * cells * args.steps / total_s / 1e9

    peak, peak_src = measured_peak()
    trf = ncu_traffic_per_cell(head["variant"], developed=head["spinup_steps"] > 0)
    roofline = {
        "bound": "hbm", "achieved": round(head["bulk_gbs"], 1) if head["bulk_gbs"] else None, "peak": peak,
        "unit": "GB/s", "frac": round(head["bulk_gbs"] / peak, 4) if head["bulk_gbs"] else None,
        "traffic": int(trf * head["bulk_cells"]) if trf else None,
        "kernel": kernel_of(head["variant"]) + " (all bulk-mask cells)",
        "algorithmic_bytes_per_launch": head["bulk_bytes_per_launch"],
        "peak_source": ("measured: MEASURED_PEAKS.json hbm_gbs" if peak_src == "measured"
                        else f"fallback: {FALLBACK_HBM_GBS:.0f} GB/s, an earlier copy measurement on this GPU type "
                             "(no MEASURED_PEAKS.json)"),
    }
    # the batched sweep set (C3), compact, so the default run records it too
    batch_c3 = None
    if args.config == "large" and args.batch_steps > 0:
        del solid, sdf
        torch.cuda.empty_cache()
        r = time_batch(args, CONFIGS["c3"], local_rank, dist_on, args.batch_steps, False)
        bg = world * r["cells"] * r["steps"] / (r["ms"] / 1e3) / 1e9
        bb = r["bulk_cells"] * 76 * r["steps"] / (r["ms"] / 1e3) / 1e9  # FP16 bytes per bulk cell update
        from flowcraft_b200.batch import candidate_name
        shape = candidate_name((r["tuned"]["rows"], r["tuned"]["grid_mult"]))
        batch_c3 = {"glups": round(bg, 2), "frac": round(bb / peak, 3), "shape": shape, "steps": r["steps"],
                    "sequential_glups": round(world * r["cells"] * r["steps"] / (r["seq_ms"] / 1e3) / 1e9, 2),
                    "cells": r["cells"], "diverged": r["diverged"]}
        solid, sdf = build_geometry(cfg, f"cuda:{local_rank}")
    e2e = None
    if not args.no_e2e:
        torch.cuda.empty_cache()
        e2e = run_e2e(args, cfg, solid, sdf, variants[0], dev_index, world, dist_on)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cores = os.cpu_count() or 1
        s_np, d_np, z0 = cpu_subbox(cfg, solid, sdf, cores)
        r = run_cpu_reference(cfg, s_np, d_np, 10 ** 6, 1, seconds=args.cpu_seconds)
        cpu = {"value": r["glups"], "unit": "GLUPS", "cores": cores, "kind": r["kind"],
               "sample": f"LbmReference::Step, {cfg['nx']}x{cfg['ny']}x{s_np.shape[0]} sub-box (z0={z0}) of the "
                         f"lattice, {r['steps']} steps in {r['seconds']:.1f}s after 1 warm-up"}
    if rank != 0:
        return 0
    variants_out = {}
    for v, r in results.items():
        # compact, so that every variant fits in a short tail of the output
        variants_out[v] = {
            "glups": round(world * cells * args.steps / (r["total_ms"] / 1e3) / 1e9, 2),
            "ms": round(r["ms_per_step"], 3), "bulk_ms": round(r["bulk_ms_per_launch"], 3),
            "frac": round(r["bulk_gbs"] / peak, 3) if r["bulk_gbs"] else None, "B_cell": r["bytes_per_cell"],
            "mhz": r["clocks"]["sm_mhz"] if r["clocks"] else None,
        }
        if r["closure_coverage"]:
            variants_out[v]["mlp_warps"] = round(r["closure_coverage"]["warp_fraction"], 4)
        if r["stats_after"]["has_nan"]:
            variants_out[v]["nan"] = True
    line = {
        "metric": METRIC, "value": value, "unit": "GLUPS", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": head["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32",
        "data": "synthetic: procedural aircraft mesh voxelized on the device, no dataset",
        "config": workload_config(args, cfg, world),
        "lattice_run": {"boundary_cells": head["boundary_cells"], "bouzidi_links": head["bouzidi_links"],
                        "closure_coverage": ({"cell_fraction": round(head["closure_coverage"]["cell_fraction"], 4),
                                              "warp_fraction": round(head["closure_coverage"]["warp_fraction"], 4)}
                                             if head["closure_coverage"] else None)},
        "variants": variants_out,
        "batch_c3": batch_c3,
        "roofline": roofline,
        "cpu_baseline": cpu,
        "e2e": e2e,
        "gpu_launches": head["launches"],
        "clocks": head["clocks"],
    }
    print(json.dumps(line, separators=(",", ":")), flush=True)
    return 0


def main(argv=None) -> int:
    args = parse_args(argv)
    cfg = CONFIGS[args.config]
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference_arm(args, cfg, rank, world)
    import datetime

    import torch
    if world > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        return run_ours(args, cfg, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
