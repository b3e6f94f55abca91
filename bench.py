#!/usr/bin/env python
"""Benchmark of the in-place Esoteric-Pull step on B200.

Workload (N = 1): D3Q19, 512^3, TRT (magic 3/16) + Smagorinsky Cs = 0.1,
lid-driven cavity (half-way bounce-back on five walls, moving lid u = (0.1, 0, 0)),
tau = 0.51, FP32 populations, started at rest with rho = 1.  One bench step is
one fused stream+collide launch over the whole lattice.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0).  ``value`` is whole-job GLUPS (lattice cells x
steps / device time, max over ranks).  With N > 1 the lattice is a
512 x 512 x (512 N) cavity cut into z-slabs of 512^3 per GPU (weak scaling):
every step is the step kernel on each slab plus one halo exchange per cut
(5 plane runs each way for D3Q19, NCCL point-to-point over NVLink).
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
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "D3Q19/27 GLUPS + % of HBM roofline, FP16-store vs FP32; adjoint/forward time"
L2_BYTES = 126 * 1024 * 1024
PEAKS_FILE = ROOT / "MEASURED_PEAKS.json"
FALLBACK_HBM_GBS = 6650.0
STEP_KERNEL_PROFILE = ROOT / "profiles" / "k_step_d3q19_fp32_cavity512.md"


def parse_args(argv=None):
    p = argparse.ArgumentParser(description=__doc__)
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=500)
    p.add_argument("--warmup", type=int, default=10)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--n", type=int, default=512, help="cavity edge (cells)")
    p.add_argument("--lattice", choices=["d3q19", "d3q27"], default="d3q19")
    p.add_argument("--storage", choices=["fp32", "fp16s"], default="fp32")
    p.add_argument("--variant", type=int, default=0,
                   help="step kernel of the headline lattice: 0 automatic, 1 one cell per thread, 2 paired cells, "
                        "3 / 4 wall-aware FP16 pairs with / without shared-memory prefetch")
    p.add_argument("--planes", type=int, default=0, help="z-planes per thread of variants 3 and 4 (0: default)")
    p.add_argument("--no-variants", action="store_true", help="skip the FP16S / D3Q27 side measurements")
    p.add_argument("--slabs", action="store_true",
                   help="run the z-slab path (used for N > 1) also on one GPU: one slab that is the whole ring")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-differentiation", action="store_true",
                   help="skip the adjoint workloads (128^3 D3Q19 FP32 and 256^3 D3Q27 FP16 gray TRT)")
    p.add_argument("--subinterval", type=int, default=0,
                   help="--case adjoint: sub-checkpoint interval of the reverse sweep (0: one level)")
    p.add_argument("--case", choices=["cavity", "adjoint", "precision"], default="cavity",
                   help="cavity: the headline line (default); adjoint / precision: only that workload at --n "
                        "(adjoint: gray TRT --lattice/--storage, --steps steps; precision: n x n/2 x n/2 sphere "
                        "pack, --steps steps), one JSON line -- small cases for profiling")
    p.add_argument("--no-precision", action="store_true",
                   help="skip the 512x256x256 sphere-pack FP16/FP32/FP64 precision study (20000 steps)")
    return p.parse_args(argv)


# ------------------------------------------------------------------ helpers
def bytes_per_update(q: int, storage: str) -> int:
    s = {"fp32": 4, "fp16s": 2, "fp64": 8}[storage]
    return 2 * q * s


def cavity_fluid_cells(n: int) -> int:
    # walls on x = 0, x = n-1, y = 0, z = 0, z = n-1; lid on y = n-1
    return (n - 2) * (n - 2) * (n - 2)


def algorithmic_bytes_per_launch(n: int, q: int, storage: str) -> int:
    """Populations read + written once per fluid cell, plus the 1-byte flag of every cell."""
    return cavity_fluid_cells(n) * bytes_per_update(q, storage) + n ** 3


def hbm_peak():
    try:
        peaks = json.loads(PEAKS_FILE.read_text())
        return float(peaks["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def profiled_traffic():
    """dram bytes per launch of the step kernel from the committed ncu summary, if any."""
    try:
        for line in STEP_KERNEL_PROFILE.read_text().splitlines():
            if line.strip().startswith("traffic_bytes_per_launch:"):
                return float(line.split(":", 1)[1].split()[0])
    except Exception:
        pass
    return None


class ClockSampler:
    """Samples SM clocks and throttle reasons with nvidia-smi during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-f", self.path], stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            for line in Path(self.path).read_text().splitlines():
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    mx.append(float(parts[2]))
                except ValueError:
                    continue
                for name, val in zip(names, parts[5:9]):
                    if val.lower() == "active":
                        reasons.add(name)
            os.unlink(self.path)
        except Exception:
            pass
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# --------------------------------------------------------------- our engine
def make_cavity(cs, n, lattice="d3q19", storage="fp32", device=0, variant=0, planes=0):
    s = cs.EsotericPullCudaSolver(cs.InPlaceLbmConfig(
        nx=n, ny=n, nz=n, tau=0.51, lattice=lattice, collision="trt", trt_magic=3.0 / 16.0, smagorinsky_les=True,
        smagorinsky_cs=0.1, storage=storage, device=device))
    if variant or planes:
        s.set_launch_shape(0, 0, variant)
        s.set_step_planes(planes)
    return s


def setup_cavity(s, cs, n, flags=None):
    s.set_flags(cs.cavity_flags(n, n, n) if flags is None else flags)
    s.set_wall_velocity(2, 0.1, 0.0, 0.0)
    s.initialize_uniform()


def time_steps(torch, s, steps):
    """Device time (ms) of `steps` step launches, CUDA events on the solver's own stream."""
    stream = torch.cuda.ExternalStream(s.stream())
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    s.wait()
    e0.record(stream)
    s.step(steps)
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1)


def e2e_job(torch, cs, n, steps, device):
    """The whole job through the public API with host buffers, timed end to end.

    Upload the cavity flags from pinned host memory, initialise, run `steps`
    steps, download rho/u (4 floats per cell) into pinned host memory and the
    FP64 reductions.  Returns (GLUPS, h2d bytes, d2h bytes).
    """
    cells = n ** 3
    flags_host = torch.from_numpy(cs.cavity_flags(n, n, n)).pin_memory()
    out = [torch.empty(cells, dtype=torch.float32).pin_memory() for _ in range(4)]
    s = make_cavity(cs, n, device=device)
    lib = s.library.raw
    import ctypes

    try:
        s.wait()
        t0 = time.perf_counter()
        lib.cfdx_lbm_set_flags(s.handle, ctypes.c_void_p(flags_host.data_ptr()), cs.bindings.HOST)
        s.set_wall_velocity(2, 0.1, 0.0, 0.0)
        s.initialize_uniform()
        s.step(steps)
        s.library.check(lib.cfdx_lbm_macroscopic(s.handle, *[ctypes.c_void_p(o.data_ptr()) for o in out],
                                                 cs.bindings.HOST))
        red = s.reduce()
        t1 = time.perf_counter()
        stats = s.transfer_stats()
    finally:
        s.close()
    if red["nonfinite"]:
        raise RuntimeError("e2e job produced non-finite populations")
    return cells * steps / (t1 - t0) / 1e9, stats.host_to_device_bytes, stats.device_to_host_bytes


def cavity_slab_flags(n: int, nz: int, planes) -> np.ndarray:
    """cavity_flags of an n x n x nz cavity restricted to the global z `planes` (a slab's local planes)."""
    from cfd_solvers_b200 import bindings as B

    planes = np.asarray(planes)
    fl = np.zeros((len(planes), n, n), np.uint8)
    fl[:, :, 0] = B.WALL
    fl[:, :, n - 1] = B.WALL
    fl[:, 0, :] = B.WALL
    fl[(planes == 0) | (planes == nz - 1)] = B.WALL
    fl[:, n - 1, :] = 2
    return fl.reshape(-1)


def cavity_config(cs, n, nz, lattice, storage, device):
    return cs.InPlaceLbmConfig(nx=n, ny=n, nz=nz, tau=0.51, lattice=lattice, collision="trt",
                               trt_magic=3.0 / 16.0, smagorinsky_les=True, smagorinsky_cs=0.1, storage=storage,
                               device=device)


def slab_exchange_overhead(torch, cs, n, steps, device, whole_ms, slabs=2):
    """The 512^3 cavity as `slabs` z-slabs on this one GPU, exchanged after every step.

    Both slabs run the same kernels as the whole lattice; the difference in
    device time per step is the cost of the halo copies (one copy kernel per
    cut, both directions) and of running the slabs' steps as separate launches.
    """
    from cfd_solvers_b200 import slabs as S

    cfg = cavity_config(cs, n, n, "d3q19", "fp32", device)
    ss = S.virtual_slabs(cfg, slabs)
    try:
        for s in ss:
            s.set_flags(cavity_slab_flags(n, n, s.slab.local_planes))
            s.set_wall_velocity(2, 0.1, 0.0, 0.0)
            s.initialize_uniform()
        S.virtual_step(ss, 3)
        torch.cuda.synchronize()
        # the last cut's exchange makes slab 0's stream wait for every slab's work
        stream = torch.cuda.ExternalStream(ss[0].stream())
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        S.virtual_step(ss, steps)
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / steps
        red = S.virtual_reduce(ss)
        msg = ss[0].halo_bytes()
    finally:
        for s in ss:
            s.close()
    return {"slabs": slabs, "glups": n ** 3 / (ms / 1e3) / 1e9, "ms_per_step": ms,
            "whole_lattice_ms_per_step": whole_ms, "overhead_frac": ms / whole_ms - 1.0,
            "message_bytes": msg, "exchange_bytes_per_step": 2 * slabs * msg,
            "launches_per_step": 2 * slabs, "nonfinite": red["nonfinite"]}


def measure_variant(torch, cs, n, lattice, storage, steps, device):
    s = make_cavity(cs, n, lattice=lattice, storage=storage, device=device)
    try:
        setup_cavity(s, cs, n)
        time_steps(torch, s, 3)
        ms = time_steps(torch, s, steps)
        red = s.reduce()
    finally:
        s.close()
    q = 19 if lattice == "d3q19" else 27
    glups = n ** 3 * steps / (ms / 1e3) / 1e9
    gbs = algorithmic_bytes_per_launch(n, q, storage) / (ms / steps / 1e3) / 1e9
    return {"glups": glups, "ms_per_step": ms / steps, "achieved_gbs": gbs, "nonfinite": red["nonfinite"]}


# ------------------------------------------------- differentiation (adjoint)
def gray_solver(cs, lattice, n, storage, device, gx=1e-5, tau=0.6):
    """Gray-LBM TRT (magic 3/16) channel, periodic in x, body force gx (the adjoint configurations)."""
    from cfd_solvers_b200.cases import channel_flags

    s = cs.EsotericPullCudaSolver(cs.InPlaceLbmConfig(
        nx=n, ny=n, nz=n, tau=tau, lattice=lattice, collision="trt", trt_magic=3.0 / 16.0, acceleration_x=gx,
        storage=storage, device=device))
    flags = channel_flags(n, n, n)
    s.set_flags(flags)
    return s, flags == 0


def misfit_target(s, ns_hidden, steps):
    """u* = u(steps) of the forward model run with the hidden solid fraction (float64 host)."""
    s.set_solid_fraction(ns_hidden)
    s.initialize_uniform()
    s.step(steps)
    f = s.compute_macroscopic()
    return np.stack([np.asarray(f.ux, np.float64), np.asarray(f.uy, np.float64), np.asarray(f.uz, np.float64)])


def misfit(s, ns, fluid, target, steps):
    """J = 1/2 sum over fluid cells |u(steps) - u*|^2, FP64 fields (FP64 storage)."""
    s.set_solid_fraction(ns)
    s.initialize_uniform()
    s.step(steps)
    import ctypes

    from cfd_solvers_b200 import bindings as B

    out = [np.zeros(s.cells(), np.float64) for _ in range(4)]
    s.library.call("cfdx_lbm_macroscopic_f64", s.handle, *[ctypes.c_void_p(o.ctypes.data) for o in out], B.HOST)
    r = (np.stack(out[1:]) - target) * fluid
    return 0.5 * float(np.sum(r * r))


def adjoint_gradient(torch, s, ns, fluid, target, steps, interval, subinterval=0):
    """(dJ/dn_s, dJ/dtau, timings) of the misfit through the discrete adjoint."""
    stream = torch.cuda.ExternalStream(s.stream())
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    s.set_solid_fraction(ns)
    s.initialize_uniform()
    s.wait()
    ev[0].record(stream)
    s.adjoint_forward(steps, interval, subinterval)
    ev[1].record(stream)
    f = s.compute_macroscopic()
    g = ((np.stack([f.ux, f.uy, f.uz]).astype(np.float64) - target) * fluid).astype(np.float32)
    gd = torch.from_numpy(g).cuda()
    grad = torch.empty(s.cells(), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    e2 = torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    gns, gtau = s.adjoint_backward(gd[0], gd[1], gd[2], grad_ns_out=grad)
    ev[2].record(stream)
    ev[2].synchronize()
    return grad.cpu().numpy(), gtau, ev[0].elapsed_time(ev[1]), e2.elapsed_time(ev[2])


def adjoint_case(torch, cs, lattice, n, storage, steps, interval, device, seeds=(1, 2), subinterval=0):
    """One differentiation workload: timings of forward, checkpointed forward and reverse sweep.

    `subinterval` > 0 reverses each checkpoint segment in two levels of recompute (sub-checkpoints
    every `subinterval` steps), which holds fewer frames for more recompute steps.
    """
    from cfd_solvers_b200.cases import gray_field

    s, fluid = gray_solver(cs, lattice, n, storage, device)
    try:
        cells = n ** 3
        ns = gray_field(cells, seeds[0])
        target = misfit_target(s, gray_field(cells, seeds[1]), steps)
        s.set_solid_fraction(ns)
        s.initialize_uniform()
        time_steps(torch, s, 3)
        s.initialize_uniform()
        fwd_ms = time_steps(torch, s, steps)
        free0 = torch.cuda.mem_get_info()[0]
        gns, gtau, afwd_ms, bwd_ms = adjoint_gradient(torch, s, ns, fluid, target, steps, interval, subinterval)
        mem = s.adjoint_memory()
        s.adjoint_release()
    finally:
        s.close()
    return {
        "lattice": lattice, "n": n, "storage": storage, "steps": steps, "checkpoint_interval": interval,
        "recompute_subinterval": subinterval,
        "forward_ms_per_step": fwd_ms / steps, "checkpointed_forward_ms_per_step": afwd_ms / steps,
        "adjoint_ms_per_step": bwd_ms / steps, "adjoint_over_forward": bwd_ms / fwd_ms,
        "forward_glups": cells * steps / (fwd_ms / 1e3) / 1e9,
        "adjoint_buffers_gb": mem / 1e9, "lattice_gb": None, "free_gb_before_adjoint": free0 / 1e9,
        "grad_tau": gtau, "grad_ns_l2": float(np.linalg.norm(gns)),
    }, gns, gtau


def adjoint_fd_check(torch, cs, n, steps, interval, device, cells=32, seeds=(1, 2, 3), h=1e-5):
    """FP32-storage adjoint vs FP64 central finite differences on `cells` random fluid cells."""
    from cfd_solvers_b200.cases import gray_field

    s64, fluid = gray_solver(cs, "d3q19", n, "fp64", device)
    s32, _ = gray_solver(cs, "d3q19", n, "fp32", device)
    try:
        N = n ** 3
        ns = gray_field(N, seeds[0])
        target = misfit_target(s64, gray_field(N, seeds[1]), steps)
        g32, gt32, _, _ = adjoint_gradient(torch, s32, ns, fluid, target, steps, interval)
        g64, gt64, _, _ = adjoint_gradient(torch, s64, ns, fluid, target, steps, interval)
        pick = np.random.default_rng(seeds[2]).choice(np.flatnonzero(fluid), cells, replace=False)
        fd = []
        for c in pick:
            p, m = ns.copy(), ns.copy()
            p[c] += np.float32(h)
            m[c] -= np.float32(h)
            fd.append((misfit(s64, p, fluid, target, steps) - misfit(s64, m, fluid, target, steps)) /
                      (float(p[c]) - float(m[c])))
        fd = np.array(fd)
    finally:
        s64.close()
        s32.close()
    def errors(g):
        e = g[pick] - fd
        return {"rel_l2": float(np.linalg.norm(e) / np.linalg.norm(fd)),
                "max_rel_to_max": float(np.max(np.abs(e)) / np.max(np.abs(fd))),
                "max_rel_per_cell": float(np.max(np.abs(e) / np.abs(fd)))}

    return {
        "lattice": f"D3Q19 {n}^3 copy", "steps": steps, "cells": cells, "fd_step": h,
        "fd": "central differences of the FP64-storage GPU forward (FP64 arithmetic)",
        "fp32_adjoint_vs_fd": errors(g32), "fp64_adjoint_vs_fd": errors(g64),
        "fp32_vs_fp64_adjoint_grad_tau_rel": abs(gt32 - gt64) / abs(gt64),
    }


def grad_errors(g, ref, gt, gt_ref):
    return {"grad_ns_rel_l2": float(np.linalg.norm(g - ref) / np.linalg.norm(ref)),
            "grad_ns_max_rel_to_max": float(np.max(np.abs(g - ref)) / np.max(np.abs(ref))),
            "grad_tau_rel": abs(gt - gt_ref) / abs(gt_ref)}


def differentiation_variants(torch, cs, device, full=True):
    """The two differentiation configurations: adjoint/forward time, memory, gradient error."""
    out = {}
    c4, _, _ = adjoint_case(torch, cs, "d3q19", 128, "fp32", 2000, 64, device)
    c4["fd_check"] = adjoint_fd_check(torch, cs, 32, 2000, 64, device)
    out["gray_d3q19_128_fp32"] = c4
    if full:
        c5, g5, t5 = adjoint_case(torch, cs, "d3q27", 256, "fp16s", 4000, 64, device)
        # The same run with two levels of recompute (sub-checkpoints every 8 steps): the ~57 GB of
        # checkpoints plus 14 frames instead of 63, for about twice the recompute steps.
        c5b, g5b, t5b = adjoint_case(torch, cs, "d3q27", 256, "fp16s", 4000, 64, device, subinterval=8)
        c5["two_level_recompute"] = {k: c5b[k] for k in ("recompute_subinterval", "adjoint_ms_per_step",
                                                         "adjoint_over_forward", "adjoint_buffers_gb")}
        c5["two_level_recompute"]["gradients_bitwise_equal"] = bool(np.array_equal(g5, g5b) and t5 == t5b)
        # Gradient errors of FP16 storage against FP32 storage and the FP64 GPU adjoint (itself
        # pinned to the FP64 CPU adjoint) at 128^3: the FP32/FP64 checkpoints of the 256^3 run
        # would not fit in 180 GB with one level of checkpointing.
        runs = {st: adjoint_case(torch, cs, "d3q27", 128, st, 4000, 64, device) for st in ("fp16s", "fp32", "fp64")}
        c5["gradient_errors_128"] = {
            "fp16_vs_fp32": grad_errors(runs["fp16s"][1], runs["fp32"][1], runs["fp16s"][2], runs["fp32"][2]),
            "fp16_vs_fp64": grad_errors(runs["fp16s"][1], runs["fp64"][1], runs["fp16s"][2], runs["fp64"][2]),
            "fp32_vs_fp64": grad_errors(runs["fp32"][1], runs["fp64"][1], runs["fp32"][2], runs["fp64"][2]),
        }
        out["gray_d3q27_256_fp16s"] = c5
    return out


# ------------------------------------------------------- precision study
def precision_study(torch, cs, device, shape=(512, 256, 256), steps=20000, seed=1):
    """FP16-shifted and FP32 storage against FP64 storage (FP64 arithmetic) on the same GPU.

    D3Q19 TRT (magic 3/16) channel, periodic in x, no-slip y/z walls, a seeded
    random sphere pack (radii uniform in [4, 12], 10 % solid), gx = 1e-6,
    tau 0.55, from rest.  The FP64-storage run is the at-scale FP64 reference
    (the same kernels in double, pinned to the FP64 CPU oracle at 1e-12 on
    small lattices).  Errors over fluid cells: L2 relative and max relative
    (to max |u|) of u; mass drift of each run.
    """
    import ctypes

    from cfd_solvers_b200 import bindings as B
    from cfd_solvers_b200.cases import sphere_pack

    nx, ny, nz = shape
    cells = nx * ny * nz
    flags = sphere_pack(nx, ny, nz, fraction=0.10, rmin=4.0, rmax=12.0, seed=seed)
    fluid = torch.from_numpy(flags == 0).to(device)
    runs = {}
    for storage in ("fp64", "fp32", "fp16s"):
        s = cs.EsotericPullCudaSolver(cs.InPlaceLbmConfig(
            nx=nx, ny=ny, nz=nz, tau=0.55, collision="trt", trt_magic=3.0 / 16.0, acceleration_x=1e-6,
            storage=storage, device=device))
        try:
            s.set_flags(flags)
            s.initialize_uniform()
            m0 = s.reduce()["mass"]
            ms = time_steps(torch, s, steps)
            red = s.reduce()
            u = torch.empty((3, cells), dtype=torch.float64, device=device)
            rho = torch.empty(cells, dtype=torch.float64, device=device)
            torch.cuda.synchronize()
            s.library.call("cfdx_lbm_macroscopic_f64", s.handle, ctypes.c_void_p(rho.data_ptr()),
                           *[ctypes.c_void_p(u[k].data_ptr()) for k in range(3)], B.DEVICE)
        finally:
            s.close()
        runs[storage] = {"u": u, "glups": cells * steps / (ms / 1e3) / 1e9, "mass0": m0, "mass": red["mass"],
                         "nonfinite": red["nonfinite"]}
    ref = runs["fp64"]["u"] * fluid
    ref_norm = float(torch.linalg.vector_norm(ref))
    ref_max = float(ref.abs().max())
    out = {"workload": f"D3Q19 TRT channel {nx}x{ny}x{nz}, sphere pack 10% (r 4-12, seed {seed}), gx 1e-6, "
                       f"tau 0.55, {steps} steps from rest",
           "solid_fraction": float(np.count_nonzero(flags) / cells), "max_u_fp64": ref_max}
    for storage, r in runs.items():
        e = r["u"] * fluid - ref
        out[storage] = {
            "glups": r["glups"], "mass_drift_rel": (r["mass"] - r["mass0"]) / r["mass0"], "nonfinite": r["nonfinite"],
            "u_l2_rel_vs_fp64": float(torch.linalg.vector_norm(e)) / ref_norm,
            "u_max_rel_vs_fp64": float(e.abs().max()) / ref_max,
        }
    out["fp16s_speedup_vs_fp32"] = runs["fp16s"]["glups"] / runs["fp32"]["glups"]
    return out


def target_summary(line, variants):
    """The three headline targets, read off the measurements above."""
    t = {"fp32_d3q19_512_roofline_frac": line["roofline"]["frac"]}
    if "d3q19_fp16s" in variants:
        t["fp16_speedup_vs_fp32_cavity512"] = variants["d3q19_fp16s"]["speedup_vs_fp32"]
    p = variants.get("precision_study")
    if p:
        t["fp16_speedup_vs_fp32_sphere_pack"] = p["fp16s_speedup_vs_fp32"]
        t["fp16_u_l2_rel_vs_fp64_sphere_pack"] = p["fp16s"]["u_l2_rel_vs_fp64"]
        t["fp32_u_l2_rel_vs_fp64_sphere_pack"] = p["fp32"]["u_l2_rel_vs_fp64"]
    d = variants.get("differentiation")
    if d:
        c4 = d["gray_d3q19_128_fp32"]
        t["adjoint_over_forward_d3q19_128_fp32"] = c4["adjoint_over_forward"]
        t["grad_vs_fd_rel_l2_fp32_adjoint"] = c4["fd_check"]["fp32_adjoint_vs_fd"]["rel_l2"]
        if "gray_d3q27_256_fp16s" in d:
            t["adjoint_over_forward_d3q27_256_fp16s"] = d["gray_d3q27_256_fp16s"]["adjoint_over_forward"]
    return t


# ----------------------------------------------------------- reference (CPU)
def cpu_reference_sample(n, warmup, steps, threads=0):
    """The reference's CPU path on the closest feature set: EsotericPullSolver<D3Q19>
    BGK + Smagorinsky with the cavity's walls and lid as a static solid mask
    (its 3-pass solid step; it has no in-place TRT or moving wall)."""
    from oracle import oracle as O

    mask = (O.cavity_flags(n, n, n) != 0).astype(np.uint8)
    mlups, seconds, _ = O.ref_bench(19, n, n, n, 0.51, warmup, steps, threads=threads, les=True, mask=mask)
    return mlups, seconds, O.ref_threads()


# The reference CPU sample of the cavity workload, shared by cpu_baseline and
# the --impl reference arm: the 3-pass solid step at SOLID_SAMPLE_N^3 (about
# 1.5 s per step on 16 host threads).
SOLID_SAMPLE_N = 384
CPU_SAMPLE_SECONDS = 20.0


def cpu_solid_baseline(max_seconds=CPU_SAMPLE_SECONDS):
    """cpu_baseline of the cavity line: the shared sample, timed steps sized to about max_seconds."""
    n = SOLID_SAMPLE_N
    _, per_step, _ = cpu_reference_sample(n, 0, 1)
    steps = max(2, int(max_seconds / max(per_step, 1e-3)))
    mlups, secs, cores = cpu_reference_sample(n, 1, steps)
    return {
        "value": mlups / 1e3, "unit": "GLUPS", "cores": cores, "kind": "reference",
        "sample": f"reference EsotericPullSolver<D3Q19> BGK+Smagorinsky, cavity as static solid mask (its 3-pass "
                  f"solid step), {n}^3, 1 warmup + {steps} timed steps ({secs:.1f} s), all host threads",
    }


def cpu_inplace_sample(n, seconds=CPU_SAMPLE_SECONDS, warmup=10):
    """The reference's own benchmark CLI on its plain in-place path (apps/cfd-bench.cpp:173-191):
    D3Q19 periodic BGK Taylor-Green, cfd-bench --streaming in-place, all host threads, timed steps
    sized to about `seconds`.  Returns the parsed cfd_solvers.benchmark.v1 record."""
    import subprocess

    from oracle import oracle as O

    threads = os.cpu_count() or 1

    def cli(w, k):
        out = subprocess.run([str(O.REF_CLI), "--lattice", "d3q19", "--nx", str(n), "--ny", str(n), "--nz", str(n),
                              "--warmup", str(w), "--steps", str(k), "--streaming", "in-place", "--threads",
                              str(threads), "--json"], capture_output=True, text=True, check=True).stdout
        return json.loads(out.strip().splitlines()[-1])

    probe = cli(1, 2)
    per_step = probe["seconds"] / 2
    steps = max(3, int(seconds / max(per_step, 1e-6)))
    rec = cli(min(warmup, steps), steps)
    rec["threads"] = threads
    return rec


def cpu_inplace_baselines():
    """cfd-bench in-place at the plain-method size (64^3) and at 512^3, one sample length each."""
    out = {}
    for n in (64, 512):
        r = cpu_inplace_sample(n)
        out[f"in_place_periodic_{n}"] = {
            "value": r["mlups"] / 1e3, "unit": "GLUPS", "cores": r["threads"], "kind": "reference",
            "sample": f"reference cfd-bench --lattice d3q19 --nx {n} --ny {n} --nz {n} --streaming in-place "
                      f"--threads {r['threads']} (periodic BGK, Taylor-Green), {r['steps']} timed steps "
                      f"({r['seconds']:.1f} s)",
        }
    return out


def c1_plain_method(torch, cs, device, warmup=10, steps=100):
    """The plain-method configuration on the GPU: D3Q19 BGK, 64^3 periodic, tau 0.6, Taylor-Green A = 0.05,
    FP32, 10 warmup + 100 timed steps; fields and checksum against the reference's own dump of the same run
    (tests/golden/reference_fixtures, made by the reference CPU build)."""
    root = os.path.dirname(os.path.abspath(__file__))
    data = np.load(os.path.join(root, "tests", "golden", "reference_fixtures.npz"))
    meta = json.load(open(os.path.join(root, "tests", "golden", "reference_fixtures.json")))["c1_d3q19_tg64"]
    n = 64
    s = cs.EsotericPullCudaSolver(cs.InPlaceLbmConfig(nx=n, ny=n, nz=n, tau=0.6, device=device))
    try:
        s.initialize_taylor_green(0.05)
        ms_warm = time_steps(torch, s, warmup)
        ms = time_steps(torch, s, steps)
        got = [np.asarray(a)[:: meta["stride"]] for a in s.compute_macroscopic()]
        checksum = s.checksum()
    finally:
        s.close()
    ref = [data[f"c1_d3q19_tg64_{k}"] for k in ("rho", "ux", "uy", "uz")]
    err = max(float(np.abs(a.astype(np.float64) - b).max()) for a, b in zip(got, ref))
    return {
        "workload": "D3Q19 BGK 64^3 periodic, tau 0.6, Taylor-Green A 0.05 (k = 2 pi / 64), FP32, "
                    f"{warmup} warmup + {steps} timed steps",
        "glups": n ** 3 * steps / (ms / 1e3) / 1e9, "ms_per_step": ms / steps, "warmup_ms": ms_warm,
        "l2": "lattice 19.9 MB < 126 MB L2 (L2-resident, as the configuration is)",
        "parity": {"max_abs_rho_u_vs_reference": err, "gate": 2e-5, "checksum": checksum,
                   "reference_checksum": meta["checksum"], "checksum_rel": abs(checksum - meta["checksum"]) /
                   abs(meta["checksum"]), "pass": err < 2e-5 and abs(checksum - meta["checksum"]) <
                   1e-6 * abs(meta["checksum"])},
    }


def voxelizer_measure(torch, device, n=512, subdivisions=7, cpu_sample=True):
    """The device voxelizer on a closed sphere of 20*4^s triangles over an n^3 grid.

    Device time of one whole cfdx_voxelize call (triangle upload, row lists,
    cells; output in device memory), host wall clock around it after a warm-up
    call.  The reference's voxelize_surface (single-threaded, every cell against
    every triangle) is timed on a bounded sample (48^3 cells x 1280 triangles) and
    reported as ray-triangle tests per second.
    """
    from cfd_solvers_b200 import geometry as G

    tris = G.transform_surface(G.icosphere((0.0, 0.0, 0.0), 0.35, subdivisions), (0.5, 0.5, 0.5), (0.3, 1.0, 0.2),
                               0.7)
    grid = G.VoxelGrid3D(n, n, n)
    out = torch.empty(n ** 3, dtype=torch.uint8, device=f"cuda:{device}")
    G.voxelize_surface(tris, grid, out=out)
    times = []
    for _ in range(3):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        G.voxelize_surface(tris, grid, out=out)
        torch.cuda.synchronize()
        times.append(time.perf_counter() - t0)
    sec = min(times)
    res = {"triangles": len(tris), "grid": f"{n}^3", "ms": sec * 1e3, "gcells_per_s": n ** 3 / sec / 1e9,
           "solid_fraction": float(out.float().mean().item()),
           "note": "one cfdx_voxelize call incl. triangle upload and scratch; best of 3 after a warm-up"}
    if cpu_sample:
        from oracle import oracle as O

        if O.reference_available():
            small = G.transform_surface(G.icosphere((0.0, 0.0, 0.0), 0.35, 3), (0.5, 0.5, 0.5), (0.3, 1.0, 0.2), 0.7)
            m = 48
            t0 = time.perf_counter()
            O.ref_voxelize(small, m, m, m, (0, 0, 0), (1, 1, 1))
            cpu = time.perf_counter() - t0
            rate = m ** 3 * len(small) / cpu
            res["cpu_reference"] = {"sample": f"{m}^3 cells x {len(small)} triangles", "seconds": cpu, "cores": 1,
                                    "ray_triangle_tests_per_s": rate,
                                    "projected_seconds_for_this_case": n ** 3 * len(tris) / rate}
    return res


def q_criterion_measure(torch, cs, n, device, cpu_sample=True):
    """The device Q-criterion of the cavity's velocity (macroscopic + Q kernels, output in
    device memory), best of 3 after a warm-up; the reference's q_criterion_3d (one core)
    timed on a 96^3 sample of the same field for comparison."""
    s = make_cavity(cs, n, device=device)
    try:
        setup_cavity(s, cs, n)
        s.step(20)
        out = torch.empty(n ** 3, dtype=torch.float64, device=f"cuda:{device}")
        s.q_criterion(out=out)
        times = []
        for _ in range(3):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            s.q_criterion(out=out)
            times.append(time.perf_counter() - t0)
        sec = min(times)
        res = {"grid": f"{n}^3", "ms": sec * 1e3, "gcells_per_s": n ** 3 / sec / 1e9,
               "note": "cfdx_lbm_q_criterion: FP64 macroscopic + Q kernels, device output, incl. scratch"}
        if cpu_sample:
            from oracle import oracle as O

            if O.reference_available():
                import ctypes

                m = 96
                rng = np.random.default_rng(1)
                vel = np.ascontiguousarray(rng.normal(0, 0.05, (m ** 3, 3)))
                q = np.zeros(m ** 3)
                lib = O.ref_lib()
                dp = ctypes.POINTER(ctypes.c_double)
                lib.ref_q_criterion.argtypes = [ctypes.c_size_t] * 3 + [dp] + [ctypes.c_double] * 3 + [dp]
                t0 = time.perf_counter()
                lib.ref_q_criterion(m, m, m, vel.ctypes.data_as(dp), 1.0, 1.0, 1.0, q.ctypes.data_as(dp))
                cpu = time.perf_counter() - t0
                res["cpu_reference"] = {"sample": f"{m}^3 random field", "seconds": cpu, "cores": 1,
                                        "gcells_per_s": m ** 3 / cpu / 1e9}
    finally:
        s.close()
    return res


def resident_coupling_measure(torch, cs, n, device, particles=1 << 20, reps=5):
    """One resident coupling cycle on the n^3 cavity, every kernel on the flow's stream and timed
    there with CUDA events (best of `reps`): the device macroscopic view, a D3Q7 thermal step,
    the cleared acceleration and Boussinesq term, a free-surface advection, its geometry and
    surface tension, a two-way particle push and the FP32 Q-criterion; then one flow step that
    consumes the acceleration.  Achieved GB/s use the algorithmic bytes per cell of each kernel
    (thermal 68, advection 20, geometry + tension 64, Q 16)."""
    from cfd_solvers_b200.multiphysics import (ImmersedBoundaryParticle, ParticleVector3, ResidentFlowDiagnostics3D,
                                               ResidentFreeSurface3D, ResidentParticles3D, ResidentThermalD3Q7)

    s = make_cavity(cs, n, device=device)
    cells = n ** 3
    res = {"grid": f"{n}^3", "particles": particles}
    try:
        setup_cavity(s, cs, n)
        s.step(10)
        stream = torch.cuda.ExternalStream(s.stream())
        th = ResidentThermalD3Q7(s, 0.02)
        fs = ResidentFreeSurface3D(s)
        diag = ResidentFlowDiagnostics3D(s)
        parts = ResidentParticles3D(s, particles)
        try:
            th.initialize_uniform(300.0)
            fs.initialize_half_space_x(n / 2 + 0.25)
            rng = np.random.default_rng(3)
            rec = np.zeros((particles, 8))
            rec[:, :3] = rng.uniform(0, n, (particles, 3))
            rec[:, 6], rec[:, 7] = 1.0, 0.5
            parts.upload(rec)
            macro = s.refresh_device_macroscopic()
            force = s.device_local_acceleration(clear=True)
            stages = {
                "macroscopic_view": lambda: s.refresh_device_macroscopic(),
                "thermal_step": lambda: th.step(macro, 1),
                "clear_acceleration": lambda: s.device_local_acceleration(clear=True),
                "boussinesq": lambda: th.add_boussinesq_acceleration(force, 300.0, 3e-3, ParticleVector3(0, -1, 0)),
                "free_surface_advect": lambda: fs.advect(macro, 0.5),
                "surface_tension": lambda: fs.add_surface_tension_acceleration(force, 0.072),
                "particles_two_way": lambda: parts.advance(macro, force, 0.5, True),
                "q_criterion_fp32": lambda: diag.q_criterion(macro),
                "flow_step": lambda: s.step(1),
            }
            def moved():
                return sum(o.transfer_stats().host_to_device_bytes + o.transfer_stats().device_to_host_bytes
                           for o in (s, th, fs, parts))

            moved0 = moved()
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(len(stages) + 1)]
            best = {k: float("inf") for k in stages}
            for _ in range(reps + 1):
                s.wait()
                ev[0].record(stream)
                for i, fn in enumerate(stages.values()):
                    fn()
                    ev[i + 1].record(stream)
                ev[-1].synchronize()
                for i, k in enumerate(stages):
                    best[k] = min(best[k], ev[i].elapsed_time(ev[i + 1]))
            bytes_per_cell = {"thermal_step": 68, "free_surface_advect": 20, "surface_tension": 64,
                              "q_criterion_fp32": 16}
            peak = hbm_peak()[0]
            res["ms"] = best
            res["cycle_ms"] = sum(best.values())
            res["achieved_gbs"] = {k: bytes_per_cell[k] * cells / (best[k] / 1e3) / 1e9 for k in bytes_per_cell}
            res["roofline_frac"] = {k: v / peak for k, v in res["achieved_gbs"].items()}
            res["mparticles_per_s"] = particles / (best["particles_two_way"] / 1e3) / 1e6
            res["host_transfer_bytes_in_cycles"] = moved() - moved0
            res["note"] = ("all kernels on the flow's stream through its device views; host bytes counted by the "
                           "C ABI over all timed cycles")
        finally:
            for o in (parts, diag, fs, th):
                o.close()
    finally:
        s.close()
    return res


def run_reference_arm(args, rank, world):
    """The reference's own CPU path for the cavity workload on the host cores: the same lattice as
    cpu_baseline (SOLID_SAMPLE_N^3, 3-pass solid step, Smagorinsky), smaller only when W + K steps of
    it would not end within about two minutes."""
    if rank != 0:
        return 0
    _, per_step, _ = cpu_reference_sample(SOLID_SAMPLE_N, 0, 1)
    budget = 110.0
    edge = SOLID_SAMPLE_N
    if per_step * (args.steps + args.warmup) > budget:
        edge = int(SOLID_SAMPLE_N * (budget / (per_step * (args.steps + args.warmup))) ** (1.0 / 3.0))
        edge = max(48, edge)
    mlups, secs, cores = cpu_reference_sample(edge, args.warmup, args.steps)
    glups = mlups / 1e3
    sample = (f"reference EsotericPullSolver<D3Q19> BGK+Smagorinsky, cavity as static solid mask (its 3-pass "
              f"solid step), {edge}^3, {args.warmup} warmup + {args.steps} timed steps ({secs:.1f} s), "
              f"all host threads")
    line = {
        "impl": "reference", "metric": METRIC, "value": glups, "unit": "GLUPS", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": secs / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"D3Q19 lid-driven cavity {args.n}^3 (reference CPU sample {edge}^3)",
                   "lattice": "d3q19", "n": args.n, "sample_n": edge,
                   "convention": "GLUPS = all cells (walls included) x steps / time, the reference's MLUPS "
                                 "convention (apps/cfd-bench.cpp:109-112)"},
        "cpu_baseline": {"value": glups, "unit": "GLUPS", "cores": cores, "kind": "reference", "sample": sample},
        "e2e": {"value": glups, "unit": "GLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "gpu_launches": 0,
    }
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------- N > 1: slabs
def slab_main(args, torch, cs, rank, world, local_rank):
    """Weak scaling over z-slabs: rank r owns planes [r n, (r+1) n) of an n x n x (n world) cavity."""
    import ctypes
    import datetime

    import torch.distributed as dist

    from cfd_solvers_b200.slabs import DistributedEsotericPullSolver

    if world == 1:
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        os.environ.setdefault("MASTER_PORT", "29531")
        os.environ.setdefault("RANK", "0")
        os.environ.setdefault("WORLD_SIZE", "1")
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                            device_id=torch.device(f"cuda:{local_rank}"))
    n = args.n
    q = 19 if args.lattice == "d3q19" else 27
    nz = n * world
    cfg = cavity_config(cs, n, nz, args.lattice, args.storage, local_rank)

    def build():
        d = DistributedEsotericPullSolver(cfg)
        return d

    d = build()
    g = d.slab
    local_flags = cavity_slab_flags(n, nz, g.local_planes)
    d.set_flags(local_flags, local=True)
    d.set_wall_velocity(2, 0.1, 0.0, 0.0)
    d.initialize_uniform()
    d.step(args.warmup)
    stream = d.solver.torch_stream()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    sampler = ClockSampler(local_rank)
    dist.barrier()
    torch.cuda.synchronize()
    sampler.start()
    time.sleep(0.3)
    e0.record(stream)
    d.step(args.steps)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    clocks = sampler.stop()
    dist.barrier()
    red = d.reduce()  # FP64 sums all-reduced over the ranks
    halo = d.solver.halo_bytes()
    d.close()

    t = torch.tensor([ms], device="cuda", dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    cells = n * n * nz
    value = cells * args.steps / (ms_max / 1e3) / 1e9

    # end to end: local flags from pinned host memory, init, steps, own-plane rho/u download, reductions
    e2e = None
    if not args.no_e2e:
        flags_host = torch.from_numpy(local_flags).pin_memory()
        d = build()  # the solver is created outside the timed job, as in the single-GPU e2e
        # rho/u of the local planes (ghosts included) into pinned host memory through the C ABI, as
        # the single-GPU e2e downloads; the rank's own planes are a contiguous range of them
        out = [torch.empty(d.solver.cells(), dtype=torch.float32).pin_memory() for _ in range(4)]
        lib = d.solver.library
        d.solver.wait()
        dist.barrier()
        t0 = time.perf_counter()
        try:
            lib.check(lib.raw.cfdx_lbm_set_flags(d.solver.handle, ctypes.c_void_p(flags_host.data_ptr()),
                                                 cs.bindings.HOST))
            d.set_wall_velocity(2, 0.1, 0.0, 0.0)
            d.initialize_uniform()
            d.step(args.steps)
            lib.check(lib.raw.cfdx_lbm_macroscopic(d.solver.handle, *[ctypes.c_void_p(o.data_ptr()) for o in out],
                                                   cs.bindings.HOST))
            d.reduce()
            t1 = time.perf_counter()
            stats = d.solver.transfer_stats()
        finally:
            d.close()
        w = torch.tensor([t1 - t0], device="cuda", dtype=torch.float64)
        dist.all_reduce(w, op=dist.ReduceOp.MAX)
        e2e = {"value": cells * args.steps / float(w.item()) / 1e9, "unit": "GLUPS",
               "h2d_bytes_per_step": stats.host_to_device_bytes / args.steps,
               "d2h_bytes_per_step": stats.device_to_host_bytes / args.steps,
               "job": f"per rank: slab flags upload (pinned) + init + {args.steps} steps with halo exchange + "
                      "own-plane rho/u download + all-reduced FP64 reductions; host wall clock, max over ranks; "
                      "bytes per step = rank 0's job bytes / steps"}

    if rank == 0:
        peak, peak_kind = hbm_peak()
        fluid = int(np.count_nonzero(g.own(local_flags) == 0))  # rank 0's own fluid cells
        alg = fluid * bytes_per_update(q, args.storage) + n * n * (n + 2)
        achieved = alg / (ms / args.steps / 1e3) / 1e9
        line = {
            "metric": METRIC, "value": value, "unit": "GLUPS", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if args.storage == "fp32" else "f16 storage / f32 arithmetic", "data": "synthetic",
            "config": {
                "workload": f"{args.lattice.upper()} lid-driven cavity {n}x{n}x{nz} in {world} z-slabs of {n}^3, "
                            f"TRT magic 3/16 + Smagorinsky Cs 0.1, tau 0.51, lid u=(0.1,0,0), "
                            f"{args.storage.upper()} populations, from rest",
                "lattice": args.lattice, "n": n, "storage": args.storage, "collision": "trt+les",
                "parallelism": f"z-slabs x{world}, halo exchange {halo} B per cut and direction per step "
                               "(NCCL send/recv over NVLink)",
                "l2": "populations per GPU > 126 MB L2 (no flush needed)",
            },
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": f"{peak_kind} hbm_gbs",
                         "traffic": None, "algorithmic_bytes_per_launch": alg,
                         "kernel": "cfdx::k_step per slab; achieved over the whole step incl. the exchange"},
            "clocks": clocks,
            "gpu_launches": (5 if world > 1 else 2) * args.steps,
            "checks": {"nonfinite_cells": red["nonfinite"], "mass": red["mass"]},
            "e2e": e2e,
        }
        print(json.dumps(line), flush=True)
    dist.barrier()
    dist.destroy_process_group()
    return 0


# --------------------------------------------------------------------- main
def main(argv=None):
    args = parse_args(argv)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference_arm(args, rank, world)
    if args.warmup < 3:
        raise SystemExit("--warmup must be >= 3")

    import torch

    import cfd_solvers_b200 as cs

    if not torch.cuda.is_available():
        raise SystemExit("bench.py needs a CUDA device (no CPU fallback)")
    torch.cuda.set_device(local_rank)
    if args.case != "cavity":
        if world != 1:
            raise SystemExit("--case adjoint/precision run on one GPU")
        if args.case == "adjoint":
            out, _, _ = adjoint_case(torch, cs, args.lattice, args.n, args.storage, args.steps,
                                     min(64, args.steps), local_rank, subinterval=args.subinterval)
        else:
            out = precision_study(torch, cs, local_rank, shape=(args.n, args.n // 2, args.n // 2), steps=args.steps)
        print(json.dumps(out), flush=True)
        return 0
    if world > 1 or args.slabs:
        return slab_main(args, torch, cs, rank, world, local_rank)
    dist = None

    def barrier():
        if dist is not None:
            dist.barrier()

    n = args.n
    q = 19 if args.lattice == "d3q19" else 27
    s = make_cavity(cs, n, lattice=args.lattice, storage=args.storage, device=local_rank, variant=args.variant,
                    planes=args.planes)
    setup_cavity(s, cs, n)
    time_steps(torch, s, args.warmup)

    sampler = ClockSampler(local_rank)
    barrier()
    torch.cuda.synchronize()
    sampler.start()
    time.sleep(0.3)
    ms = time_steps(torch, s, args.steps)
    clocks = sampler.stop()
    barrier()
    red = s.reduce()
    s.close()

    t = torch.tensor([ms], device="cuda", dtype=torch.float64)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    cells = n ** 3
    value = cells * args.steps * world / (ms_max / 1e3) / 1e9

    line = None
    if rank == 0:
        peak, peak_kind = hbm_peak()
        per_launch_s = ms / args.steps / 1e3
        alg = algorithmic_bytes_per_launch(n, q, args.storage)
        achieved = alg / per_launch_s / 1e9
        line = {
            "metric": METRIC, "value": value, "unit": "GLUPS", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if args.storage == "fp32" else "f16 storage / f32 arithmetic", "data": "synthetic",
            "config": {
                "workload": f"{args.lattice.upper()} lid-driven cavity {n}^3, TRT magic 3/16 + Smagorinsky Cs 0.1, "
                            f"tau 0.51, lid u=(0.1,0,0), {args.storage.upper()} populations, from rest",
                "lattice": args.lattice, "n": n, "storage": args.storage, "collision": "trt+les",
                "parallelism": "single GPU",
                "l2": f"populations {cells * q * (4 if args.storage == 'fp32' else 2) / 1e9:.1f} GB > 126 MB L2 "
                      "(no flush needed)",
                "fluid_cells": cavity_fluid_cells(n),
                "glups_fluid": cavity_fluid_cells(n) * args.steps * world / (ms_max / 1e3) / 1e9,
                "convention": "value = all cells (walls included) x steps / time, the reference's MLUPS "
                              "convention (apps/cfd-bench.cpp:109-112); glups_fluid counts fluid cells only, "
                              "as roofline.achieved's bytes do",
            },
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": f"{peak_kind} hbm_gbs",
                         "traffic": profiled_traffic(), "algorithmic_bytes_per_launch": alg,
                         "kernel": "cfdx::k_step (one launch per step)"},
            "clocks": clocks,
            "gpu_launches": args.steps,
            "checks": {"nonfinite_cells": red["nonfinite"], "mass": red["mass"]},
        }

    # ---- end to end through the public API with host buffers (each rank its own job)
    e2e = None
    if not args.no_e2e:
        barrier()
        glups_e2e, h2d, d2h = e2e_job(torch, cs, n, args.steps, local_rank)
        t = torch.tensor([glups_e2e], device="cuda", dtype=torch.float64)
        if dist is not None:
            dist.all_reduce(t, op=dist.ReduceOp.MIN)
        e2e = {"value": float(t.item()) * world, "unit": "GLUPS",
               "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": d2h / args.steps,
               "job": f"host flags upload (pinned) + init + {args.steps} steps + rho/u download (pinned) + "
                      "FP64 reductions, host wall clock; bytes per step = job bytes / steps"}

    # ---- side measurements on rank 0 (FP16 storage, D3Q27)
    variants = {}
    if rank == 0 and not args.no_variants and world == 1:
        vs = max(20, args.steps // 2)
        if args.storage == "fp32" and args.lattice == "d3q19":
            variants["c1_plain_method_64"] = c1_plain_method(torch, cs, local_rank)
            f16 = measure_variant(torch, cs, n, "d3q19", "fp16s", vs, local_rank)
            f16["speedup_vs_fp32"] = f16["glups"] / value
            f16["roofline_frac"] = f16["achieved_gbs"] / hbm_peak()[0]
            variants["d3q19_fp16s"] = f16
            d27 = measure_variant(torch, cs, n, "d3q27", "fp32", vs, local_rank)
            d27["roofline_frac"] = d27["achieved_gbs"] / hbm_peak()[0]
            variants["d3q27_fp32"] = d27
            variants["z_slabs_one_gpu"] = slab_exchange_overhead(torch, cs, n, vs, local_rank, ms / args.steps)
            variants["voxelizer"] = voxelizer_measure(torch, local_rank, n, cpu_sample=not args.no_cpu_baseline)
            variants["q_criterion"] = q_criterion_measure(torch, cs, n, local_rank,
                                                          cpu_sample=not args.no_cpu_baseline)
            variants["resident_coupling"] = resident_coupling_measure(torch, cs, n, local_rank)
        if not args.no_differentiation:
            variants["differentiation"] = differentiation_variants(torch, cs, local_rank)
        if not args.no_precision:
            variants["precision_study"] = precision_study(torch, cs, local_rank)

    if rank == 0:
        line["e2e"] = e2e
        if variants:
            line["variants"] = variants
            line["targets"] = target_summary(line, variants)
        if not args.no_cpu_baseline and world == 1:
            line["cpu_baseline"] = cpu_solid_baseline()
            line["cpu_baseline_in_place"] = cpu_inplace_baselines()
        print(json.dumps(line), flush=True)

    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
