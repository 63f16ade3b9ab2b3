#!/usr/bin/env python
"""Benchmark of the RKDG residual + time-step path on one B200 (or N replicas).

Workload (default): the unstructured isentropic vortex -- periodic [0,10]^2,
Delaunay triangulation of a 700 x 700 lattice jittered by U(-0.3h, 0.3h)
(seed 2, 980,000 triangles), P2, 6-point volume and 3-point edge rules,
HLLC, SSP-RK3, CFL 0.2; synthetic data (seeded), no external dataset.

One JSON line on rank 0:
  value        FP32 DOF-stage updates/s with the state resident in HBM
               (FP32 state/arithmetic, FP64 geometry and dt), K steps timed
               with CUDA events on the solver's stream, max over ranks;
  fp64         the same for the plain FP64 path;
  roofline     achieved HBM GB/s of the fused stage kernel: algorithmic bytes
               per element-stage B = 4 Nb w (2 + r_s) + 56 (r_s = 2/3 mean
               over SSP-RK3) times elements, over the event-timed launch;
  e2e          the same metric through the C ABI with host buffers in the
               reference's layout and basis: set_state + K steps + get_state;
  cpu_baseline the reference's own code (oracle/_ref, compiled from its
               sources for the host) on a bounded sample, all host threads;
  l2           vortex L2(rho) error vs the exact solution at t_final for FP32
               and FP64 (the FP64 path is the one parity-checked against the
               oracle at 1e-12).

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "DOF-stage updates/s"
UNIT = "DOF-stage/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--lattice", type=int, default=700)
    ap.add_argument("--t-final", type=float, default=2.0, help="vortex time of the L2 error runs")
    ap.add_argument("--no-accuracy", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--precision", default="both", choices=["both", "fp32", "fp64"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end C-ABI run")
    return ap.parse_args()


# ------------------------------------------------------------ distributed --
class Dist:
    def __init__(self):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = False

    def init(self):
        import torch

        if self.world > 1:
            import datetime

            import torch.distributed as dist

            torch.cuda.set_device(self.local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
            self.pg = True
        else:
            torch.cuda.set_device(0)

    def barrier(self):
        if self.pg:
            import torch.distributed as dist

            dist.barrier()

    def max(self, x: float) -> float:
        if not self.pg:
            return x
        import torch
        import torch.distributed as dist

        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def sum(self, x: float) -> float:
        if not self.pg:
            return x
        import torch
        import torch.distributed as dist

        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        return float(t.item())

    def close(self):
        if self.pg:
            import torch.distributed as dist

            dist.destroy_process_group()


# ----------------------------------------------------------------- clocks --
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during a region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.out = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.out.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.out:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------- workload --
def vortex_mesh(lattice: int):
    from rkdg_heter_calculate_b200 import meshgen

    return meshgen.periodic_delaunay(lattice, L=10.0, jitter=0.3, seed=2)


FAR = (1.0, 1.0, 1.0, 2.5 + 1.0)  # rho=1, u=v=1, p=1, gamma=1.4: E = p/0.4 + 1


def solver_for(mesh, precision):
    from rkdg_heter_calculate_b200 import CUDARkdgSolver

    return CUDARkdgSolver(mesh, order=2, nq=6, ng=3, flux="hllc", rk=3, precision=precision,
                          gamma=1.4, cfl=0.2, farfield=FAR, reorder=True)


def bytes_per_elem_stage(nb: int, word: int, rk: int = 3) -> float:
    r = {3: 2.0 / 3.0, 2: 0.5}[rk]
    return 4 * nb * word * (2 + r) + 56


def time_steps(s, U0, K, W, dist, stream_ptr):
    import torch

    s.setFreedom(U0, basis="native")
    s.set_time(0.0)
    s.advance(W)
    st = torch.cuda.ExternalStream(stream_ptr)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    dist.barrier()
    torch.cuda.synchronize()
    e0.record(st)
    _, n = s.advance(K)
    e1.record(st)
    torch.cuda.synchronize()
    dist.barrier()
    ms = e0.elapsed_time(e1)
    assert n == K
    return dist.max(ms)


def stage_roofline(s, T, nb, word, peak_gbs):
    t0 = s.time_stage(0, 10)
    t1 = s.time_stage(1, 10)
    t_avg = (t0 + 2 * t1) / 3.0  # SSP-RK3: one stage without U^n, two with
    B = bytes_per_elem_stage(nb, word)
    achieved = T * B / (t_avg * 1e-3) / 1e9
    return {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak_gbs, "unit": "GB/s",
            "frac": round(achieved / peak_gbs, 4), "traffic": None,
            "kernel": "stage_kernel", "ms_per_launch": {"stage_without_U0": round(t0, 5),
                                                        "stage_with_U0": round(t1, 5)},
            "bytes_per_element_stage": B}


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        try:
            return float(json.load(open(p))["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


def e2e_run(s, U0_native, K, dist, stream_ptr):
    """set_state (host, reference basis) + K steps + get_state (host)."""
    import torch

    s.setFreedom(U0_native, basis="native")
    Uref = s.copyFreedomToHost(basis="reference")
    pinned = torch.empty(Uref.shape, dtype=torch.float64, pin_memory=True)
    host = pinned.numpy()
    host[...] = Uref
    out_pinned = torch.empty(Uref.shape, dtype=torch.float64, pin_memory=True)
    out = out_pinned.numpy()
    # warm (allocates the conversion tables and staging once)
    s.setFreedom(host, basis="reference")
    s.advance(2)
    s.copyFreedomToHost(basis="reference")
    dist.barrier()
    torch.cuda.synchronize()
    t = time.perf_counter()
    s.setFreedom(host, basis="reference")
    s.set_time(0.0)
    s.advance(K)
    from rkdg_heter_calculate_b200 import capi

    capi.check(capi.lib().rkdg_get_state(s.h, capi.dptr(out), s.T, capi.BASIS_REFERENCE))
    torch.cuda.synchronize()
    wall = time.perf_counter() - t
    dist.barrier()
    return dist.max(wall), host.nbytes


def accuracy(mesh, U0, t_final):
    from rkdg_heter_calculate_b200 import vortex

    ex = lambda X, Y: vortex.exact(X, Y, t_final)  # noqa: E731
    out = {"t_final": t_final}
    for prec in ("fp64", "fp32"):
        s = solver_for(mesh, prec)
        s.setFreedom(U0, basis="native")
        t, n = s.advance(10 ** 7, t_final=t_final)
        U = s.copyFreedomToHost(basis="native")
        out[prec] = {"l2_rho": vortex.l2_error(mesh, U, ex), "steps": n, "t": t}
        s.close()
    out["ratio_fp32_over_fp64"] = out["fp32"]["l2_rho"] / out["fp64"]["l2_rho"]
    return out


# --------------------------------------------------------- CPU baselines --
def cpu_reference_sample(seconds: float, threads: int | None = None):
    """The reference's own code (oracle/_ref) when built, else the oracle
    port, on a 20,000-triangle periodic Delaunay vortex mesh; returns
    (DOF-stage/s, descriptor)."""
    from oracle import oracle, ref
    from rkdg_heter_calculate_b200 import meshgen

    threads = threads or os.cpu_count() or 1
    mesh = meshgen.periodic_delaunay(100, L=10.0, jitter=0.3, seed=2)
    T = mesh.ntri
    if ref.available():
        ref.set_threads(threads)
        c = ref.RefCase(mesh, gamma=1.4, alpha_deg=45.0, mach=math.sqrt(2.0 / 1.4), cfl=0.2,
                        threads_per_block=64)
        c.init_freestream()
        c.advance(1)
        t = time.perf_counter()
        n = 0
        while time.perf_counter() - t < seconds:
            c.advance(1)
            n += 1
        el = time.perf_counter() - t
        kind = "reference"
        sample = (f"reference multi_gpuRkdg kernels compiled for the host (oracle/_ref), "
                  f"P2 7-point LLF SSP-RK3 (its only method), {T}-triangle periodic Delaunay "
                  f"vortex mesh, {n} steps")
    else:
        oracle.set_threads(threads)
        o = oracle.Oracle(mesh, order=2, nq=6, ng=3, flux=oracle.HLLC, rk=3, cfl=0.2, farfield=FAR)
        U = np.zeros((4, 6, T))
        U[:, 0, :] = np.array(FAR)[:, None]
        o.set_state(U)
        o.step()
        t = time.perf_counter()
        n = 0
        while time.perf_counter() - t < seconds:
            o.step()
            n += 1
        el = time.perf_counter() - t
        kind = "port"
        sample = f"oracle C port, P2 6-point HLLC SSP-RK3, {T}-triangle mesh, {n} steps"
    value = T * 24 * 3 * n / el
    return value, {"value": value, "unit": UNIT, "cores": threads, "kind": kind, "sample": sample}


def run_reference_arm(args, dist):
    if dist.rank != 0:
        return
    per_step = max(1.0, args.cpu_seconds / max(1, args.steps))
    vals = []
    desc = None
    for i in range(args.warmup + args.steps):
        v, desc = cpu_reference_sample(per_step)
        if i >= args.warmup:
            vals.append(v)
    value = float(np.mean(vals))
    desc["value"] = value
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "unstructured isentropic vortex (bounded CPU sample)"},
            "cpu_baseline": desc,
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------- main --
def main():
    args = parse()
    dist = Dist()
    if args.impl == "reference":
        run_reference_arm(args, dist)
        return
    dist.init()
    import torch  # noqa: F401

    from rkdg_heter_calculate_b200 import vortex

    K, W = args.steps, args.warmup
    mesh = vortex_mesh(args.lattice)
    T = mesh.ntri
    U0 = vortex.project_native(mesh, lambda X, Y: vortex.exact(X, Y, 0.0), 6)
    peak, peak_kind = measured_peak()
    res = {}
    clocks = None
    precs = [(p, w) for p, w in (("fp32", 4), ("fp64", 8)) if args.precision in ("both", p)]
    for prec, word in precs:
        s = solver_for(mesh, prec)
        sp = s.stream()
        if prec == "fp32":
            with ClockSampler(dist.local) as cs:
                ms = time_steps(s, U0, K, W, dist, sp)
            clocks = cs.summary()
        else:
            ms = time_steps(s, U0, K, W, dist, sp)
        dofs = T * 24
        value = dist.sum(dofs * 3 * K) / (ms * 1e-3)
        roof = stage_roofline(s, T, 6, word, peak)
        roof["peak_kind"] = peak_kind
        e2e = None
        if not args.no_e2e:
            e2e_wall, state_bytes = e2e_run(s, U0, K, dist, sp)
            e2e = {"value": dist.sum(dofs * 3 * K) / e2e_wall, "unit": UNIT,
                   "h2d_bytes_per_step": state_bytes / K, "d2h_bytes_per_step": state_bytes / K}
        res[prec] = {"value": value, "ms_per_step": ms / K, "roofline": roof, "e2e": e2e}
        s.close()
    acc = None
    if not args.no_accuracy:
        acc = accuracy(mesh, U0, args.t_final)
    cpu = None
    if dist.rank == 0 and not args.no_cpu:
        _, cpu = cpu_reference_sample(args.cpu_seconds)
    if dist.rank == 0:
        head = "fp32" if "fp32" in res else "fp64"
        r = res[head]
        other = res.get("fp64") if head == "fp32" else None
        line = {
            "metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": dist.world,
            "steps": K, "warmup": W, "ms_per_step": r["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32" if head == "fp32" else "f64",
            "data": "synthetic",
            "config": {"workload": "unstructured isentropic vortex: periodic Delaunay of a "
                                   f"{args.lattice}x{args.lattice} lattice jittered +-0.3h (seed 2), "
                                   f"{T} triangles, P2, 6-pt volume / 3-pt edge, HLLC, SSP-RK3, CFL 0.2",
                       "triangles": T, "dofs": T * 24, "precision": "FP32 state/arithmetic, FP64 geometry+dt",
                       "parallelism": f"{dist.world} independent replica(s), no collective",
                       "l2_flush": "inputs larger than L2 (state 3 x 94 MB FP32 / 188 MB FP64 per step)"},
            "roofline": r["roofline"], "e2e": r["e2e"],
            "fp64": other,
            "fp32_over_fp64": (r["value"] / other["value"]) if other else None,
            "cpu_baseline": cpu, "clocks": clocks, "gpu_launches": 4 * K,
            "l2": acc,
        }
        print(json.dumps(line), flush=True)
    dist.close()


if __name__ == "__main__":
    main()
