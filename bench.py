#!/usr/bin/env python
"""Benchmark of the RKDG residual + time-step path on one B200 (or N replicas).

Headline workload (default, --workload batched): 64 independent isentropic-
vortex solves, vortex strength U[1,5] and free-stream angle U[0, 2 pi)
(free-stream speed sqrt(2)), seeded (numpy default_rng(4)); periodic
Delaunay meshes of jittered lattices with triangle counts log-uniform in
[5k, 200k]; P1 and P2 (Bernoulli 1/2); FP32 arithmetic with FP64 geometry and
dt, the state in the FP32C form (cell means as high + low float pairs updated
in FP64; --headline fp32 times the plain FP32 form instead); HLLC, SSP-RK3,
CFL 0.2; one launch per RK stage over all solves, CUDA graph, autotuned launch
shape.  Synthetic data, no dataset.

Beside it, the plain FP64 single solve on the unstructured vortex (periodic
Delaunay of a 700 x 700 lattice jittered by +-0.3h, seed 2, 980,000
triangles, P2, 6/3-point rules, HLLC, SSP-RK3) and its FP32 form.

One JSON line on rank 0:
  value        batched FP32C DOF-stage updates/s, state resident in HBM, K steps
               timed with CUDA events on the batch's stream, max over ranks
               (batched_forms: the FP32, FP32C and FP64 forms);
  plain_fp64   single-solve FP64 DOF-stage/s on the 980k mesh (and its FP32 form);
  roofline     achieved HBM GB/s of the fused stage kernel over all solves:
               algorithmic bytes per element-stage 16 rows (2 + r_s) + 56
               (16-byte rows per element: 2 Nb in FP64, Nb in FP32, Nb + 1 in
               FP32C; r_s = 2/3 mean over SSP-RK3) over the event-timed launch;
  e2e          the batched metric through the C ABI with host buffers: every
               solve's set_state + K steps + get_state;
  cpu_baseline the reference's own code (oracle/_ref, compiled from its
               sources for the host) on a bounded sample, all host threads;
  l2           vortex L2(rho) error vs the exact solution: batched FP32 and FP32C
               vs FP64 per solve after 200 steps, and the 980k solve at t = 2;
  step_fp32_vs_fp64  the Mach-3 step (P1, LLF, TVB) in each form: rate, roofline,
               and the cell-mean density's distance from FP64, with the FP64
               control run from a perturbed state;
  serving      the request server under Poisson arrivals: p50/p90/p99 latency,
               DOF-stage/s, the loop's time split.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]
"""
from __future__ import annotations

import argparse
import contextlib
import gc
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
GAMMA = 1.4


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="batched", choices=["batched", "vortex", "serving", "step", "decomp"])
    ap.add_argument("--decomp-parts", default="1,2,4",
                    help="--workload decomp at N = 1: part counts sharing the GPU (under torchrun: one per rank)")
    ap.add_argument("--no-step", action="store_true", help="skip the Mach-3 step FP32/FP64 comparison")
    ap.add_argument("--step-h", type=int, default=400, help="1/h of the Mach-3 step lattice")
    ap.add_argument("--step-times", default="0.05,0.5", help="output times of the Mach-3 step runs")
    ap.add_argument("--no-step-sensitivity", action="store_true",
                    help="skip the FP64 run from an initial state perturbed at FP32 rounding level")
    ap.add_argument("--nsolves", type=int, default=64)
    ap.add_argument("--lattice", type=int, default=700)
    ap.add_argument("--plain-steps", type=int, default=50)
    ap.add_argument("--t-final", type=float, default=2.0, help="vortex time of the 980k L2 runs")
    ap.add_argument("--no-accuracy", action="store_true")
    ap.add_argument("--no-plain", action="store_true", help="skip the single-solve measurements")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--precision", default="all",
                    help="comma list of fp32, fp32c, fp64, or 'all'")
    ap.add_argument("--headline", default="fp32c", choices=["fp32", "fp32c"],
                    help="FP32 form whose batched rate is the line's value (fp32c: the form that "
                         "holds the vortex L2 error within 1.05x of FP64)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end C-ABI run")
    ap.add_argument("--no-serving", action="store_true", help="skip the serving sweep")
    ap.add_argument("--serve-requests", type=int, default=100, help="requests per arrival-rate point")
    ap.add_argument("--serve-loads", default="0.8",
                    help="arrival rates as fractions of the measured saturated request rate (the default run "
                         "keeps one; --workload serving --serve-loads 0.5,0.7,0.8,0.9 sweeps)")
    return ap.parse_args()


# ------------------------------------------------------------ distributed --
class Dist:
    """One process per GPU (torchrun env vars); NCCL on GPUs, gloo when the
    process has no GPU (the CPU tests of the multi-rank path)."""

    def __init__(self, backend: str | None = None):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend
        self.pg = False

    def init(self):
        import torch

        if self.backend is None:
            self.backend = "nccl" if torch.cuda.is_available() else "gloo"
        if self.backend == "nccl":
            torch.cuda.set_device(self.local if self.world > 1 else 0)
        if self.world > 1:
            import datetime

            import torch.distributed as dist

            dist.init_process_group(self.backend, timeout=datetime.timedelta(seconds=600))
            self.pg = True

    def barrier(self):
        if self.pg:
            import torch.distributed as dist

            dist.barrier()

    def _reduce(self, x, op):
        if not self.pg:
            return x
        import torch
        import torch.distributed as dist

        t = torch.tensor([x], dtype=torch.float64, device="cuda" if self.backend == "nccl" else "cpu")
        dist.all_reduce(t, op=op)
        return float(t.item())

    def max(self, x: float) -> float:
        import torch.distributed as dist

        return self._reduce(x, dist.ReduceOp.MAX) if self.pg else x

    def sum(self, x: float) -> float:
        import torch.distributed as dist

        return self._reduce(x, dist.ReduceOp.SUM) if self.pg else x

    def close(self):
        if self.pg:
            import torch.distributed as dist

            dist.destroy_process_group()


# ----------------------------------------------------------------- clocks --
class ClockSampler:
    """SM clocks and clock-event (throttle) reasons sampled during a region:
    NVML polled from a host thread every 2 ms (a timed region of a few tens
    of milliseconds still gets samples), the device found by its PCI bus id
    so that a remapped CUDA_VISIBLE_DEVICES still names the right GPU;
    nvidia-smi at 200 ms where the NVML binding is absent.  Read-only."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
               ("sw_power_cap", 0x4), ("hw_power_brake_slowdown", 0x80))

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.nvml = None
        self.out = []
        self.samples = []  # (sm MHz, max sm MHz, reason bits) from NVML
        self.stop = threading.Event()

    def _nvml_handle(self):
        import pynvml
        import torch

        pynvml.nvmlInit()
        try:
            pr = torch.cuda.get_device_properties(self.gpu)
            bus = f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0"
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.gpu)

    def _poll(self):
        nv, h = self.nvml
        mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        while True:
            try:
                self.samples.append((nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM), mx,
                                     nv.nvmlDeviceGetCurrentClocksEventReasons(h)))
            except Exception:
                pass
            if self.stop.wait(0.002):
                break

    def __enter__(self):
        try:
            self.nvml = self._nvml_handle()
            self.thread = threading.Thread(target=self._poll, daemon=True)
            self.thread.start()
            return self
        except Exception:
            self.nvml = None
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
        if self.nvml:
            self.stop.set()
            self.thread.join(timeout=5)
            try:
                self.nvml[0].nvmlShutdown()
            except Exception:
                pass
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        for clk, m, bits in self.samples:
            sm.append(float(clk))
            mx = float(m)
            reasons.update(n for n, b in self.REASONS if bits & b)
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
                "samples": len(sm), "source": "nvml, 2 ms" if self.samples else "nvidia-smi, 200 ms"}


# ------------------------------------------------------------ workloads --
def conservative(rho, u, v, p):
    return (rho, rho * u, rho * v, p / (GAMMA - 1) + 0.5 * rho * (u * u + v * v))


FAR_C2 = conservative(1.0, 1.0, 1.0, 1.0)


def batched_problems(n=64, seed=4):
    """The 64 uneven vortex solves: (meshes, orders, initial native states,
    far fields, (beta, uinf, vinf) per solve)."""
    from rkdg_heter_calculate_b200 import meshgen, vortex

    rng = np.random.default_rng(seed)
    betas = rng.uniform(1.0, 5.0, n)
    thetas = rng.uniform(0.0, 2 * math.pi, n)
    tris = np.exp(rng.uniform(math.log(5e3), math.log(2e5), n))
    orders = np.where(rng.random(n) < 0.5, 1, 2).astype(np.int32)
    mesh_seeds = rng.integers(0, 2 ** 31, n)
    meshes, states, fars, par = [], [], [], []
    for i in range(n):
        lat = max(4, int(round(math.sqrt(tris[i] / 2.0))))
        m = meshgen.periodic_delaunay(lat, L=10.0, jitter=0.3, seed=int(mesh_seeds[i]))
        ui, vi = math.sqrt(2) * math.cos(thetas[i]), math.sqrt(2) * math.sin(thetas[i])
        nb = 3 if orders[i] == 1 else 6
        b = float(betas[i])
        U = vortex.project_native(m, lambda X, Y, b=b, ui=ui, vi=vi: vortex.exact(X, Y, 0.0, b, GAMMA, ui, vi), nb, n=4)
        meshes.append(m)
        states.append(U)
        fars.append(conservative(1.0, ui, vi, 1.0))
        par.append((b, ui, vi))
    return meshes, orders, states, fars, par


def bytes_per_elem_stage(nb: int, prec: str, rk: int = 3) -> float:
    """Algorithmic HBM bytes of one element-stage: the stage input read and
    the output written (2), U^n read where the stage combines with it (mean
    r over the scheme's stages), 16-byte state rows (FP64 two per basis
    function, FP32 one, FP32C one plus the row of the cell means' low
    parts), and 56 B of geometry, edge codes and tile tables."""
    r = {3: 2.0 / 3.0, 2: 0.5}[rk]
    rows = {"fp64": 2 * nb, "fp32": nb, "fp32c": nb + 1}[prec]
    return 16 * rows * (2 + r) + 56


def precisions(args):
    sel = ["fp32", "fp32c", "fp64"] if args.precision == "all" else args.precision.split(",")
    return [p for p in ("fp32", "fp32c", "fp64") if p in sel]


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        try:
            return float(json.load(open(p))["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


@contextlib.contextmanager
def no_gc():
    """Python's cyclic collector paused over a timed region: a collection
    over the bench's large heap would otherwise be timed as the library's."""
    was = gc.isenabled()
    gc.disable()
    try:
        yield
    finally:
        if was:
            gc.enable()


def event_time(stream_ptr, fn, dist):
    import torch

    st = torch.cuda.ExternalStream(stream_ptr)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    dist.barrier()
    torch.cuda.synchronize()
    with no_gc():
        e0.record(st)
        fn()
        e1.record(st)
    torch.cuda.synchronize()
    dist.barrier()
    return dist.max(e0.elapsed_time(e1))


def measured_traffic(profile):
    """DRAM bytes per launch (mean over an SSP-RK3 step) that an ncu capture
    of the same workload recorded in profiles/<profile> (None if absent)."""
    p = os.path.join(ROOT, "profiles", profile)
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith("traffic_bytes_per_launch_mean:"):
            return float(line.split(":")[1])
    return None


def stage_times(obj, trials=3, reps=10):
    """Event-timed mean launch time of each RK stage (reps back-to-back
    launches on the solver's stream), the best of a few trials: the same
    best-of convention as the measured HBM peak it is divided into."""
    return [min(obj.time_stage(k, reps) for _ in range(trials)) for k in range(3)]


def roofline(t0, t1, t2, alg_bytes, peak, peak_kind, kernel, traffic=None):
    t_avg = (t0 + t1 + t2) / 3.0  # SSP-RK3: stage 1 without U^n, stages 2-3 with; 3 adds the epilogue
    achieved = alg_bytes / (t_avg * 1e-3) / 1e9
    return {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4), "traffic": traffic, "kernel": kernel,
            "peak_kind": peak_kind,
            "ms_per_launch": {"stage_without_U0": round(t0, 5), "stage_with_U0": round(t1, 5),
                              "last_stage": round(t2, 5)},
            "timing": "CUDA events: mean of 10 back-to-back launches per RK stage, best of 3 trials",
            "algorithmic_bytes_per_launch": alg_bytes}


def pinned_like(a):
    import torch

    t = torch.empty(a.shape, dtype=torch.float64, pin_memory=True)
    h = t.numpy()
    h[...] = a
    return t, h


# ------------------------------------------------------- batched (C4) --
def run_batched(args, dist, peak, peak_kind):
    from rkdg_heter_calculate_b200 import capi, vortex
    from rkdg_heter_calculate_b200.batch import Batch

    K, W = args.steps, args.warmup
    meshes, orders, states, fars, par = batched_problems(args.nsolves)
    nbs = [3 if o == 1 else 6 for o in orders]
    dofs = sum(m.ntri * 4 * nb for m, nb in zip(meshes, nbs))
    out = {}
    # the line's own form first, on the device as the run finds it; the
    # other forms after it
    order = sorted(precisions(args), key=lambda p: p != args.headline)
    for prec in order:
        b = Batch(meshes, orders, precision=prec, flux="hllc", rk=3, nq=6, cfl=0.2, farfields=fars)
        for i, U in enumerate(states):
            b.set_state(i, U)
        ctas, torder, tile = b.autotune()
        for i, U in enumerate(states):
            b.set_state(i, U)
            b.set_time(i, 0.0)
        b.advance(W)
        sp = b.stream()
        with ClockSampler(dist.local) as cs:
            ms = event_time(sp, lambda: b.advance(K), dist)
        clocks = cs.summary()
        value = dist.sum(dofs * 3 * K) / (ms * 1e-3)
        alg = sum(m.ntri * bytes_per_elem_stage(nb, prec) for m, nb in zip(meshes, nbs))
        label = ("tiled_stage_kernel (one RK stage: the P2 tiles and the P1 tiles as two concurrent launches; "
                 "time and bytes per stage)" if torder == 2 else
                 "tiled_stage_kernel (P1+P2 tiles, one launch per stage)")
        roof = roofline(*stage_times(b), alg, peak, peak_kind,
                        label, measured_traffic(f"tiled_stage_kernel_batched_{prec}.md")
                        if args.nsolves == 64 else None)
        e2e = None
        if not args.no_e2e:
            hosts = [pinned_like(U) for U in states]
            outs = [pinned_like(np.zeros_like(U)) for U in states]
            for i, (_, h) in enumerate(hosts):
                b.set_state(i, h)
            b.advance(2)
            dist.barrier()
            with no_gc():
                t = time.perf_counter()
                for i, (_, h) in enumerate(hosts):
                    capi.check(capi.lib().rkdg_batch_set_state(b.h, i, capi.dptr(h), h.shape[2]))
                    b.set_time(i, 0.0)
                b.advance(K)
                for i, (_, h) in enumerate(outs):
                    capi.check(capi.lib().rkdg_batch_get_state(b.h, i, capi.dptr(h), h.shape[2]))
                wall = time.perf_counter() - t
            wall = dist.max(wall)
            nbytes = sum(h.nbytes for _, h in hosts)
            e2e = {"value": dist.sum(dofs * 3 * K) / wall, "unit": UNIT,
                   "h2d_bytes_per_step": nbytes / K, "d2h_bytes_per_step": nbytes / K,
                   "timed": "per solve set_state (pinned host, native basis) + K steps + get_state"}
        acc = None
        if not args.no_accuracy:
            for i, U in enumerate(states):
                b.set_state(i, U)
                b.set_time(i, 0.0)
            t_end, _ = b.advance(200)
            acc = []
            for i, m in enumerate(meshes):
                beta, ui, vi = par[i]
                acc.append(vortex.l2_error(m, b.state(i), lambda X, Y: vortex.exact(X, Y, t_end[i], beta, GAMMA, ui, vi)))
        out[prec] = {"value": value, "ms_per_step": ms / K, "roofline": roof, "e2e": e2e,
                     "clocks": clocks, "shape": {"ctas": ctas, "tile_order": torder, "tile": tile},
                     "l2": acc, "tris": [int(m.ntri) for m in meshes], "orders": [int(o) for o in orders]}
        b.close()
    info = {"solves": len(meshes), "triangles": int(sum(m.ntri for m in meshes)),
            "p1_solves": int((orders == 1).sum()), "p2_solves": int((orders == 2).sum()),
            "dofs": int(dofs), "min_tris": int(min(m.ntri for m in meshes)),
            "max_tris": int(max(m.ntri for m in meshes))}
    return out, info


# ------------------------------------------------- single solve (C2) --
def solver_for(mesh, precision):
    from rkdg_heter_calculate_b200 import CUDARkdgSolver

    return CUDARkdgSolver(mesh, order=2, nq=6, ng=3, flux="hllc", rk=3, precision=precision,
                          gamma=GAMMA, cfl=0.2, farfield=FAR_C2, reorder=True)


def run_plain(args, dist, peak, peak_kind, K):
    from rkdg_heter_calculate_b200 import capi, meshgen, vortex

    mesh = meshgen.periodic_delaunay(args.lattice, L=10.0, jitter=0.3, seed=2)
    T = mesh.ntri
    U0 = vortex.project_native(mesh, lambda X, Y: vortex.exact(X, Y, 0.0), 6, n=4)
    out = {}
    for prec in precisions(args):
        s = solver_for(mesh, prec)
        s.setFreedom(U0, basis="native")
        s.advance(args.warmup)
        ms = event_time(s.stream(), lambda: s.advance(K), dist)
        value = dist.sum(T * 24 * 3 * K) / (ms * 1e-3)
        roof = roofline(*stage_times(s), T * bytes_per_elem_stage(6, prec),
                        peak, peak_kind, "tiled_stage_kernel (P2)")
        e2e = None
        if not args.no_e2e:
            s.setFreedom(U0, basis="native")
            Uref = s.copyFreedomToHost(basis="reference")
            _, host = pinned_like(Uref)
            _, res = pinned_like(np.zeros_like(Uref))
            s.setFreedom(host)
            s.advance(2)
            s.copyFreedomToHost()
            dist.barrier()
            with no_gc():
                t = time.perf_counter()
                s.setFreedom(host)  # reference basis and layout
                s.set_time(0.0)
                t1 = time.perf_counter()
                s.advance(K)
                t2 = time.perf_counter()
                capi.check(capi.lib().rkdg_get_state(s.h, capi.dptr(res), T, capi.BASIS_REFERENCE))
                t3 = time.perf_counter()
            wall = dist.max(t3 - t)
            e2e = {"value": dist.sum(T * 24 * 3 * K) / wall, "unit": UNIT,
                   "h2d_bytes_per_step": host.nbytes / K, "d2h_bytes_per_step": host.nbytes / K,
                   "timed": "set_state (pinned host, reference basis) + K steps + get_state",
                   "phases_ms": {"set_state": round((t1 - t) * 1e3, 2), "advance": round((t2 - t1) * 1e3, 2),
                                 "get_state": round((t3 - t2) * 1e3, 2)}}
        acc = None
        if not args.no_accuracy:
            s.setFreedom(U0, basis="native")
            s.set_time(0.0)
            t, n = s.advance(10 ** 7, t_final=args.t_final)
            acc = {"l2_rho": vortex.l2_error(mesh, s.copyFreedomToHost(basis="native"),
                                             lambda X, Y: vortex.exact(X, Y, t)),
                   "t": t, "steps": n}
        out[prec] = {"value": value, "ms_per_step": ms / K, "roofline": roof, "e2e": e2e, "l2": acc}
        s.close()
    return out, T


# ------------------------------------------------- domain decomposition --
def run_decomp(args, dist):
    """One mesh decomposed into parts (the unstructured vortex of the plain
    workload, P2, HLLC, SSP-RK3, CFL 0.2, the first form of --precision).
    At N = 1 the parts of each count in --decomp-parts share the GPU
    (LocalTransport: rows between the parts' buffers, events between their
    streams); under torchrun each rank holds one part of an N-way split and
    moves rows with NCCL (TorchTransport).  Each run: W warm-up steps, then
    K steps of DecomposedSolve.advance_device (halo transfers, the
    wave-speed all-reduce and the stages in stream order), timed from a CUDA
    event before the first enqueue to one after every part's stream has
    drained, max over ranks; the single context's advance on the same mesh
    beside it."""
    import torch

    from rkdg_heter_calculate_b200 import meshgen, vortex
    from rkdg_heter_calculate_b200.decomp import (DecomposedSolve, DevicePart, LocalTransport, Partition,
                                                  TorchTransport)

    prec = precisions(args)[0]
    K, W = args.steps, args.warmup
    mesh = meshgen.periodic_delaunay(args.lattice, L=10.0, jitter=0.3, seed=2)
    T = mesh.ntri
    U0 = vortex.project_native(mesh, lambda X, Y: vortex.exact(X, Y, 0.0), 6, n=4)
    kw = dict(order=2, nq=6, ng=3, flux="hllc", rk=3, precision=prec, gamma=GAMMA, cfl=0.2, farfield=FAR_C2)
    out = {"workload": f"unstructured isentropic vortex, periodic Delaunay of a {args.lattice}x{args.lattice} "
                       f"lattice jittered +-0.3h (seed 2), {T} triangles, P2, HLLC, SSP-RK3, CFL 0.2, {prec}",
           "triangles": T, "steps": K, "warmup": W, "runs": []}
    s = solver_for(mesh, prec)
    s.setFreedom(U0, basis="native")
    s.advance(W)
    ms1 = event_time(s.stream(), lambda: s.advance(K), dist)
    s.close()
    out["single_context"] = {"dof_stage_per_s": T * 72 * K / (ms1 * 1e-3), "ms_per_step": ms1 / K}
    counts = [dist.world] if dist.world > 1 else [int(x) for x in args.decomp_parts.split(",")]
    for k in counts:
        P = Partition(mesh, k)
        mine = [dist.rank] if dist.world > 1 else list(range(k))
        parts = {p: DevicePart(P, p, **kw) for p in mine}
        for p, part in parts.items():
            part.set_state(P.split(U0, p), basis="native")
        halo = int(sum(P.halo[p].size for p in range(k)))
        # the enqueued loop, and (parts in one process) the captured step
        # replayed, with each stage's transfers beside its interior tiles
        # (overlap) or before the whole stage
        shapes = ([(False, False), (True, False), (True, True)] if dist.world == 1 else
                  [(False, True), (False, False)])
        for graph, overlap in shapes:
            solve = DecomposedSolve(parts, TorchTransport() if dist.world > 1 else LocalTransport(), rk=3,
                                    overlap=overlap)
            solve.advance_device(W, graph=graph)
            dist.barrier()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for part in parts.values():
                part.stream().wait_event(e0)
            solve.advance_device(K, graph=graph)  # returns once every part's stream has drained
            e1.record()
            torch.cuda.synchronize()
            ms = dist.max(e0.elapsed_time(e1))
            out["runs"].append({"parts": k, "ranks": dist.world, "graph": graph, "overlap": overlap,
                                "dof_stage_per_s": T * 72 * K / (ms * 1e-3), "ms_per_step": ms / K,
                                "halo_copies": halo, "vs_single_context": ms1 / ms})
        for part in parts.values():
            part.close()
    return out


# ------------------------------------------------------ Mach-3 step (C3) --
def run_step(args, dist, peak, peak_kind):
    """Mach-3 wind-tunnel step: jittered Delaunay mesh, h = 1/400 (seed 3),
    P1, LLF, TVB limiter M = 50 on characteristic variables, SSP-RK3, CFL 0.3,
    uniform inflow (1.4, 3, 0, 1) to t = 0.5; FP32 and FP32C (FP64 geometry
    and dt) against FP64.  Reports the relative L1 difference of the
    cell-mean density, sum_e A_e |rho_x - rho64| / sum_e A_e |rho64|, at
    t = 0.05 and t = 0.5, the same difference for an FP64 run started from a
    state perturbed by 6e-8 relative (the control: how far FP64 moves under
    FP32-sized input noise), each precision's DOF-stage/s over the run (CUDA
    events), and the roofline of one stage (stage kernel + limiter)."""
    from rkdg_heter_calculate_b200 import CUDARkdgSolver, meshgen

    m = meshgen.forward_step(h=1.0 / args.step_h, seed=3)
    far = np.array(conservative(1.4, 3.0, 0.0, 1.0))
    U = np.zeros((4, 3, m.ntri))
    U[:, 0, :] = far[:, None]
    a = m.areas()
    kw = dict(order=1, nq=3, ng=2, flux="llf", rk=3, limiter="tvb", tvb_m=50.0, cfl=0.3, farfield=far)
    times = [float(x) for x in args.step_times.split(",")]
    runs = [(p, U) for p in precisions(args)]
    if "fp64" in precisions(args) and not args.no_step_sensitivity:
        rng = np.random.default_rng(7)
        Up = U.copy()
        Up[:, 0, :] *= 1.0 + 6e-8 * rng.uniform(-1.0, 1.0, (4, m.ntri))
        runs.append(("fp64_perturbed", Up))
    res = {}
    for name, U0 in runs:
        prec = name.split("_")[0]
        s = CUDARkdgSolver(m, precision=prec, **kw)
        s.setFreedom(U0, basis="native")
        out = {}
        steps = 0
        ms = 0.0
        for tt in times:
            box = {}
            ms += event_time(s.stream(), lambda: box.update(r=s.advance(10 ** 8, t_final=tt)), dist)
            steps += box["r"][1]
            out[tt] = s.copyFreedomToHost(basis="native")[0, 0]
        stage_ms = stage_times(s) if name in ("fp32", "fp32c", "fp64") else None
        s.close()
        res[name] = {"rho": out, "steps": steps, "ms": ms, "stage_ms": stage_ms}

    def rel(x, y):
        return float(np.sum(a * np.abs(x - y)) / np.sum(a * np.abs(y)))

    line = {"workload": "Mach-3 step, jittered Delaunay h = 1/%d (seed 3), %d triangles, P1, LLF, TVB M = 50, "
                        "SSP-RK3, CFL 0.3, to t = %g" % (args.step_h, m.ntri, times[-1]),
            "triangles": int(m.ntri),
            "definition": "sum_e A_e |rho_x - rho64| / sum_e A_e |rho64| over cell means"}
    for p in ("fp32", "fp32c"):
        if p in res and "fp64" in res:
            line[f"rel_L1_rho_{p}_vs_fp64"] = {str(t): rel(res[p]["rho"][t], res["fp64"]["rho"][t]) for t in times}
    for name in res:
        r = res[name]
        per_stage_ms = r["ms"] / (3 * r["steps"])
        d = {"steps": r["steps"], "ms": round(r["ms"], 1),
             "dof_stage_per_s": dist.sum(r["steps"] * 3 * 12 * m.ntri / (r["ms"] * 1e-3))}
        if r["stage_ms"]:
            prec = name
            alg = m.ntri * bytes_per_elem_stage(3, prec)
            # the whole stage (fused stage kernel, TVB limiter, the step's dt
            # kernel shared out) as it runs in the time loop, and the stage
            # kernel alone (event-timed launches, epilogue included)
            d["roofline"] = {"bound": "hbm", "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                             "algorithmic_bytes_per_stage": alg,
                             "stage_with_limiter": {"ms": round(per_stage_ms, 5),
                                                    "achieved": round(alg / (per_stage_ms * 1e-3) / 1e9, 1),
                                                    "frac": round(alg / (per_stage_ms * 1e-3) / 1e9 / peak, 4)},
                             "stage_kernel_only": roofline(*r["stage_ms"], alg, peak, peak_kind,
                                                           "tiled_stage_kernel (P1, LLF)")}
        line[name] = d
    if "fp64_perturbed" in res:
        line["rel_L1_rho_fp64_perturbed_vs_fp64"] = {
            str(t): rel(res["fp64_perturbed"]["rho"][t], res["fp64"]["rho"][t]) for t in times}
    return line


# ------------------------------------------------------------ serving (C5) --
SERVE_LEVELS = 8   # mesh sizes per request kind, log-spaced over [2k, 500k] triangles


def serving_catalogue(seed=5):
    """Meshes and initial states the serving requests draw from: per kind
    (isentropic vortex on a periodic Delaunay mesh, Mach-3 wind-tunnel step)
    SERVE_LEVELS meshes with triangle counts log-spaced over [2k, 500k]."""
    from rkdg_heter_calculate_b200 import meshgen, vortex

    rng = np.random.default_rng(seed)
    sizes = np.exp(np.linspace(math.log(2e3), math.log(5e5), SERVE_LEVELS))
    cat = {"vortex": [], "step": []}
    for k, T in enumerate(sizes):
        lat = max(8, int(round(math.sqrt(T / 2.0))))
        m = meshgen.periodic_delaunay(lat, L=10.0, jitter=0.3, seed=int(rng.integers(0, 2 ** 31)))
        b, th = float(rng.uniform(1.0, 5.0)), float(rng.uniform(0.0, 2 * math.pi))
        ui, vi = math.sqrt(2) * math.cos(th), math.sqrt(2) * math.sin(th)
        U2 = vortex.project_native(m, lambda X, Y: vortex.exact(X, Y, 0.0, b, GAMMA, ui, vi), 6, n=4)
        # the native basis is orthonormal and hierarchical: the P1 projection
        # is the first three coefficients of the P2 one
        cat["vortex"].append((m, U2, np.ascontiguousarray(U2[:, :3]), conservative(1.0, ui, vi, 1.0)))
        k = max(10, 5 * int(round(math.sqrt(T / 5.04) / 5)))  # 1/h: the step corner on the lattice
        st = meshgen.forward_step(h=1.0 / k, seed=int(rng.integers(0, 2 ** 31)))
        far = conservative(1.4, 3.0, 0.0, 1.0)
        U1 = np.zeros((4, 3, st.ntri))
        U1[:, 0, :] = np.array(far)[:, None]
        cat["step"].append((st, U1, far))
    return cat, sizes


def serving_requests(cat, sizes, n, rng):
    """n requests: kind 50/50, triangle count log-uniform in [2k, 500k]
    (snapped to the nearest catalogue size), vortex P1/P2 50/50 with HLLC and
    no limiter, step P1 with LLF and the TVB limiter (the limited-flow
    configuration's method; with Davis wave-speed bounds the HLLC flux goes
    non-physical at the step corner under P1 + TVB), final time U[0.1, 1.0].
    Each: (mesh, order, U0, t_final, far field, limiter, flux)."""
    out = []
    lo, hi = math.log(sizes[0]), math.log(sizes[-1])
    for _ in range(n):
        kind = "vortex" if rng.random() < 0.5 else "step"
        lvl = int(round((rng.uniform(lo, hi) - lo) / (hi - lo) * (SERVE_LEVELS - 1)))
        tf = float(rng.uniform(0.1, 1.0))
        if kind == "vortex":
            m, U2, U1, far = cat["vortex"][lvl]
            order = 2 if rng.random() < 0.5 else 1
            out.append((m, order, U2 if order == 2 else U1, tf, far, False, "hllc"))
        else:
            m, U1, far = cat["step"][lvl]
            out.append((m, 1, U1, tf, far, True, "llf"))
    return out


def serve_point(srv, reqs, rate):
    """Submits reqs with Poisson arrivals at `rate` requests/s (inf: all at
    once) from a pool of submitter threads; returns per-request latencies
    (completion - arrival, seconds), DOF-stage/s over the point, the split of
    DOF-stage updates by request kind and where the loop's time went."""
    import concurrent.futures as cf

    from rkdg_heter_calculate_b200 import capi
    from rkdg_heter_calculate_b200.serve import clock

    rng = np.random.default_rng(6)
    gaps = rng.exponential(1.0 / rate, len(reqs)) if math.isfinite(rate) else np.zeros(len(reqs))
    gaps[0] = 0.0
    arrive = np.cumsum(gaps)
    st0, tm0 = srv.stats(), srv.timing()
    pool = cf.ThreadPoolExecutor(8)
    t0 = clock()
    futs = []
    for (m, order, U, tf, far, lim, flux), at in zip(reqs, arrive):
        d = t0 + at - clock()
        if d > 0:
            time.sleep(d)
        futs.append(pool.submit(srv.submit, m, order, U, tf, far, lim, flux))
    lat, queue_wait, failed, t_end = [], [], 0, t0
    kind_dofs = {"vortex": 0.0, "step": 0.0}
    for f, at, (m, order, U, tf, far, lim, flux) in zip(futs, arrive, reqs):
        try:
            r = srv.wait(f.result())
            lat.append(r.completed - (t0 + at))
            queue_wait.append(r.admitted - r.submitted)
            t_end = max(t_end, r.completed)
            kind_dofs["step" if lim else "vortex"] += r.steps * 3 * 4 * (3 if order == 1 else 6) * m.ntri
        except capi.RkdgError:
            failed += 1
    pool.shutdown()
    st1, tm1 = srv.stats(), srv.timing()
    wall = t_end - t0
    return {"latency": np.array(lat), "queue_wait": np.array(queue_wait),
            "dof_per_s": (st1["dof_stage_updates"] - st0["dof_stage_updates"]) / wall,
            "wall_s": wall, "failed": failed, "busy_frac": (st1["busy_seconds"] - st0["busy_seconds"]) / wall,
            "peak_in_flight": st1["peak_in_flight"],
            "loop_s": {k: tm1[k] - tm0[k] for k in ("admit_s", "retire_s", "step_s")},
            "chunks": tm1["chunks"] - tm0["chunks"], "kind_dofs": kind_dofs}


def run_serving(args, dist):
    from rkdg_heter_calculate_b200.serve import Server

    cat, sizes = serving_catalogue()
    rng = np.random.default_rng(5 + dist.rank)
    n = args.serve_requests
    with Server(8 << 30, max_slots=64, precision="fp32", flux="llf", rk=3, gamma=GAMMA, cfl=0.2,
                tvb_m=50.0) as srv:
        # warm-up: one small request of each kind
        for r in (serving_requests(cat, sizes, 4, np.random.default_rng(99))):
            m, order, U, tf, far, lim, flux = r
            try:
                srv.wait(srv.submit(m, order, U, min(tf, 0.05), far, lim, flux))
            except Exception:
                pass
        # one request set, offered all at once and then at Poisson rates that
        # are fractions of the saturated completion rate
        reqs = serving_requests(cat, sizes, n, rng)
        sat = serve_point(srv, reqs, math.inf)
        cap_rate = n / sat["wall_s"]
        points = [("saturated", math.inf, sat)]
        for f in [float(x) for x in args.serve_loads.split(",") if x]:
            points.append((f, f * cap_rate, serve_point(srv, reqs, f * cap_rate)))
    out = []
    for f, rate, p in points:
        lat = p["latency"]
        pc = {q: dist.max(float(np.percentile(lat, q))) if len(lat) else None for q in (50, 90, 99)}
        kd = p["kind_dofs"]
        tot = max(1.0, kd["vortex"] + kd["step"])
        out.append({"load": f, "lambda_req_per_s": None if not math.isfinite(rate) else round(rate, 3),
                    "p50_s": pc[50], "p90_s": pc[90], "p99_s": pc[99],
                    "mean_s": float(lat.mean()) if len(lat) else None,
                    "max_s": float(lat.max()) if len(lat) else None,
                    "queue_wait_p50_s": float(np.percentile(p["queue_wait"], 50)) if len(lat) else None,
                    "dof_stage_per_s": dist.sum(p["dof_per_s"]), "wall_s": round(p["wall_s"], 3),
                    "completed": int(len(lat)), "failed": p["failed"],
                    "busy_frac": round(p["busy_frac"], 3), "peak_in_flight": p["peak_in_flight"],
                    "loop_time_frac": {k: round(v / p["wall_s"], 4) for k, v in p["loop_s"].items()},
                    "step_chunks": p["chunks"],
                    "dof_share_step_requests": round(kd["step"] / tot, 4)})
    return {"workload": f"Poisson arrivals (default_rng(5)) of isentropic-vortex and Mach-3-step requests "
                        f"50/50, triangles log-uniform in [2k, 500k] snapped to {SERVE_LEVELS} mesh sizes "
                        "per kind, vortex P1/P2 50/50 with HLLC, step P1 with LLF and TVB (M=50), final time "
                        "U[0.1, 1.0]; FP32, SSP-RK3, CFL 0.2; 8 GiB pool, 64 slots",
            "step_flux": "LLF: with Davis wave-speed bounds the HLLC flux goes non-physical at the step corner "
                         "under P1 + TVB, in FP64 and FP32 alike, so step requests run the limited-flow "
                         "configuration's LLF",
            "requests_per_point": n, "saturated_req_per_s": round(cap_rate, 3),
            "latency": "completion - arrival, host preprocessing and result read-back included",
            "loop_time": "fractions of each point's wall time the serving loop spent uploading admitted "
                         "requests, retiring finished ones, and running step chunks (graph launches and the "
                         "control-block read that ends each chunk of 4 steps)",
            "points": out}


# --------------------------------------------------------- CPU baselines --
def host_cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip() + f" ({os.cpu_count()} logical CPUs)"
    except OSError:
        pass
    return f"{os.cpu_count()} logical CPUs"


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
        c = ref.RefCase(mesh, gamma=GAMMA, alpha_deg=45.0, mach=math.sqrt(2.0 / GAMMA), cfl=0.2,
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
        o = oracle.Oracle(mesh, order=2, nq=6, ng=3, flux=oracle.HLLC, rk=3, cfl=0.2, farfield=FAR_C2)
        U = np.zeros((4, 6, T))
        U[:, 0, :] = np.array(FAR_C2)[:, None]
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
            "config": {"workload": "isentropic vortex on periodic Delaunay meshes (bounded CPU sample)"},
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

    if dist.world > 1 and args.workload == "batched":
        # a scaling run times the headline pack per rank (replicas); the
        # single-GPU legs (plain, Mach-3 step, serving, CPU) run at N = 1
        args.no_plain = args.no_step = args.no_serving = args.no_cpu = True

    peak, peak_kind = measured_peak()
    line = None
    if args.workload == "batched":
        res, info = run_batched(args, dist, peak, peak_kind)
        plain = None
        if not args.no_plain:
            plain, T2 = run_plain(args, dist, peak, peak_kind, args.plain_steps)
        head = next((p for p in (args.headline, "fp32", "fp32c", "fp64") if p in res))
        r = res[head]
        serving = None if args.no_serving else run_serving(args, dist)
        step = None if (args.no_step or args.no_accuracy) else run_step(args, dist, peak, peak_kind)
        cpu = None
        if dist.rank == 0 and not args.no_cpu:
            _, cpu = cpu_reference_sample(args.cpu_seconds)
            v1, d1 = cpu_reference_sample(args.cpu_seconds / 3.0, threads=1)
            cpu["single_core"] = {"value": v1, "sample": d1["sample"]}
            cpu["host_cpu"] = host_cpu_model()
        if dist.rank == 0:
            def l2_summary(prec):
                if res.get(prec, {}).get("l2") is None or res.get("fp64", {}).get("l2") is None:
                    return None
                x, ref = np.array(res[prec]["l2"]), np.array(res["fp64"]["l2"])
                ratio = x / ref
                w = int(np.argmax(ratio))
                return {"over_fp64_max": float(ratio.max()), "over_fp64_median": float(np.median(ratio)),
                        "solves_over_1.05": int((ratio > 1.05).sum()),
                        "worst": {"triangles": r["tris"][w], "order": r["orders"][w],
                                  "fp64_l2_rho": float(ref[w]), "l2_rho": float(x[w])}}
            l2 = None
            if "fp64" in res and res["fp64"].get("l2") is not None:
                l2 = {"steps": 200, "batched_fp64_l2_rho_median": float(np.median(res["fp64"]["l2"]))}
                for p in ("fp32", "fp32c"):
                    if l2_summary(p):
                        l2["batched_" + p] = l2_summary(p)
            if plain and plain.get("fp64", {}).get("l2"):
                l2 = dict(l2 or {})
                for p in plain:
                    if plain[p].get("l2"):
                        l2["plain_980k_" + p] = plain[p]["l2"]
            pf64 = plain["fp64"]["value"] if plain and "fp64" in plain else None
            line = {
                "metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": dist.world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["ms_per_step"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32" if head != "fp64" else "f64", "data": "synthetic",
                "config": {"workload": f"batched uneven solves: {info['solves']} isentropic vortices "
                                       f"(strength U[1,5], angle U[0,2pi), seed 4) on periodic jittered "
                                       f"Delaunay meshes, {info['min_tris']}-{info['max_tris']} triangles "
                                       f"(log-uniform 5k-200k), {info['p1_solves']} P1 + {info['p2_solves']} P2, "
                                       + {"fp32": "FP32 state (FP64 geometry, dt)",
                                          "fp32c": "FP32 arithmetic, FP32 state with cell means as high + low "
                                                   "float pairs updated in FP64 (FP64 geometry, dt)",
                                          "fp64": "FP64"}[head]
                                       + ", HLLC, SSP-RK3, CFL 0.2, one launch per RK stage for all solves, "
                                       "CUDA graph, autotuned shape",
                           "precision_form": head, **info, "launch_shape": r["shape"],
                           "parallelism": f"{dist.world} independent replica(s), no collective",
                           "l2_flush": "inputs larger than L2 (3 state buffers of the packed solves)"},
                "roofline": r["roofline"], "e2e": r["e2e"],
                "batched_forms": {p: {k: res[p][k] for k in ("value", "ms_per_step", "roofline", "clocks", "shape")}
                                  for p in res},
                "plain_fp64": pf64,
                "batched_over_plain_fp64": ({p: res[p]["value"] / pf64 for p in res if p != "fp64"}
                                            if pf64 else None),
                "plain": ({p: {k: v for k, v in plain[p].items() if k != "l2"} for p in plain}
                          if plain else None),
                "cpu_baseline": cpu, "clocks": r["clocks"], "gpu_launches": 4 * args.steps,
                "l2": l2, "serving": serving, "step_fp32_vs_fp64": step,
            }
    elif args.workload == "step":
        step = run_step(args, dist, *measured_peak())
        if dist.rank == 0:
            print(json.dumps({"workload": "step", "n_gpus": dist.world, "step_fp32_vs_fp64": step}), flush=True)
    elif args.workload == "decomp":
        dec = run_decomp(args, dist)
        if dist.rank == 0:
            print(json.dumps({"workload": "decomp", "n_gpus": dist.world, "decomp": dec}), flush=True)
    elif args.workload == "serving":
        serving = run_serving(args, dist)
        if dist.rank == 0:
            print(json.dumps({"workload": "serving", "n_gpus": dist.world, "serving": serving}), flush=True)
    else:
        res, T = run_plain(args, dist, peak, peak_kind, args.steps)
        head = next((p for p in (args.headline, "fp32", "fp32c", "fp64") if p in res))
        r = res[head]
        cpu = None
        if dist.rank == 0 and not args.no_cpu:
            _, cpu = cpu_reference_sample(args.cpu_seconds)
        if dist.rank == 0:
            line = {
                "metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": dist.world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["ms_per_step"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32" if head != "fp64" else "f64", "data": "synthetic",
                "config": {"workload": "unstructured isentropic vortex: periodic Delaunay of a "
                                       f"{args.lattice}x{args.lattice} lattice jittered +-0.3h (seed 2), "
                                       f"{T} triangles, P2, 6-pt volume / 3-pt edge, HLLC, SSP-RK3, CFL 0.2",
                           "triangles": T, "parallelism": f"{dist.world} independent replica(s)",
                           "l2_flush": "inputs larger than L2"},
                "roofline": r["roofline"], "e2e": r["e2e"],
                "forms": {p: res[p] for p in res if p != head},
                "cpu_baseline": cpu, "gpu_launches": 4 * args.steps,
                "l2": {p: res[p]["l2"] for p in res},
            }
    if line is not None:
        print(json.dumps(line), flush=True)
    dist.close()


if __name__ == "__main__":
    main()
