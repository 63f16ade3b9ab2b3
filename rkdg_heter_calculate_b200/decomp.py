"""Domain decomposition of one mesh over several devices.

The reference splits a mesh over MPI ranks: each rank reads a partition
file, finds its interface elements and builds inner-boundary ghost cells
(multi_gpuRkdg/src/unstructuredgrid.cpp:290-318, 502-526), exchanges the
interface indices once (src/sendboundaryindex.cpp:8-37), and before every
stage copies its whole state to the host, packs the interface rows and sends
them with MPI_Isend/MPI_Irecv (RkdgAdvance::commuInfo,
src/rkdgadvance.cpp:287-409); its dt reduction over ranks is commented out
(src/rkdgadvance.cpp:226-234).

Here one process drives one device.  `Partition` splits the mesh into
contiguous ranges of its locality (Morton) order and lists, per part, the
halo copies it needs and, per pair of parts, the rows that cross.
`DecomposedSolve` advances the parts held by this process: before every
stage the halo rows are gathered on the owner's device (rkdg_gather_rows),
moved device to device, and scattered into the receiver's halo rows
(rkdg_scatter_rows); each step's dt is the minimum over all parts; with the
TVB limiter the halo means of each stage output are refreshed before
rkdg_limit.  The transport is pluggable: `TorchTransport` uses
torch.distributed point-to-point operations (NCCL between GPUs, gloo on the
host), `LocalTransport` moves rows between parts held by one process.

`DecomposedSolve.step` is the host-driven loop (each stage call and dt
returns to the host; any part object with the DevicePart methods, the
oracle's included).  `DecomposedSolve.advance_device` runs whole steps in
stream order on the device parts: the halo transfers, an all-reduce of the
CFL wave-speed maximum and the stages are enqueued on the parts' streams
with no host round trip until the end (rkdg_part_wave, rkdg_part_begin_step,
rkdg_part_stage, rkdg_part_limit).
"""
from __future__ import annotations

import numpy as np

import ctypes as C

from . import capi, meshgen


class Partition:
    """k parts of a mesh: contiguous, equal-sized ranges of its locality
    order.  For part p: `owned[p]` (caller element ids, in locality order),
    `halo[p]` (caller ids of the other parts' elements that share an edge
    with an owned one, grouped by owner and in the owner's order),
    `local_mesh(p)` (owned elements first, then the halo copies), and for
    each pair of parts the local indices that cross: `send[p][q]` (p-local
    rows q needs, in q's halo order) and `recv[p][q]` (where they land in
    p's halo)."""

    def __init__(self, mesh: meshgen.Mesh, nparts: int):
        if nparts < 1 or nparts > mesh.ntri:
            raise ValueError("nparts must be in [1, ntri]")
        T = mesh.ntri
        order = capi.locality_order(mesh.vertices, mesh.tris, mesh.neighbours)  # new -> caller
        bounds = np.rint(np.linspace(0, T, nparts + 1)).astype(np.int64)
        owner = np.empty(T, dtype=np.int64)
        pos = np.empty(T, dtype=np.int64)  # position in the owner's owned list
        self.mesh = mesh
        self.nparts = nparts
        self.owned = []
        for p in range(nparts):
            ids = order[bounds[p]:bounds[p + 1]].astype(np.int64)
            owner[ids] = p
            pos[ids] = np.arange(ids.size)
            self.owned.append(ids)
        self.owner = owner
        self.halo = []
        for p in range(nparts):
            nb = mesh.neighbours[self.owned[p]].ravel()
            nb = np.unique(nb[nb >= 0])
            nb = nb[owner[nb] != p]
            key = owner[nb] * (T + 1) + pos[nb]
            self.halo.append(nb[np.argsort(key, kind="stable")])
        # rows crossing between parts: q's halo entries owned by p, in q's order
        self.send = [dict() for _ in range(nparts)]
        self.recv = [dict() for _ in range(nparts)]
        for q in range(nparts):
            h = self.halo[q]
            n_own_q = self.owned[q].size
            for p in np.unique(owner[h]):
                sel = np.nonzero(owner[h] == p)[0]
                self.send[int(p)][q] = pos[h[sel]].astype(np.int32)
                self.recv[q][int(p)] = (n_own_q + sel).astype(np.int32)

    def n_owned(self, p: int) -> int:
        return int(self.owned[p].size)

    def local_ids(self, p: int) -> np.ndarray:
        """Caller ids of part p's local elements: owned, then halo copies."""
        return np.concatenate([self.owned[p], self.halo[p]])

    def local_mesh(self, p: int) -> meshgen.Mesh:
        """Part p as a mesh: its owned elements and halo copies, neighbours
        renumbered; a halo copy's edges to elements outside the part are
        open (tagged outflow; the library never updates a halo copy)."""
        m = self.mesh
        ids = self.local_ids(p)
        g2l = np.full(m.ntri, -1, dtype=np.int64)
        g2l[ids] = np.arange(ids.size)
        nb_g = m.neighbours[ids]
        nb = np.where(nb_g >= 0, g2l[np.maximum(nb_g, 0)], -1).astype(np.int32)
        bc = m.bc[ids].copy()
        opened = (nb < 0) & (nb_g >= 0)  # edges of halo copies leaving the part
        assert not opened[: self.n_owned(p)].any()
        bc[opened] = capi.BC_OUTFLOW
        return meshgen.Mesh(vertices=m.vertices, tris=np.ascontiguousarray(m.tris[ids]), neighbours=nb,
                            bc=bc.astype(np.int8), periodic=m.periodic, name=f"{m.name}_part{p}", extent=m.extent)

    def split(self, U: np.ndarray, p: int) -> np.ndarray:
        """Part p's local state [4][nb][local] from a whole-mesh state."""
        return np.ascontiguousarray(U[:, :, self.local_ids(p)])

    def join(self, parts: dict) -> np.ndarray:
        """A whole-mesh state from the parts' owned rows {p: [4][nb][local]}."""
        first = next(iter(parts.values()))
        out = np.zeros(first.shape[:2] + (self.mesh.ntri,))
        for p, U in parts.items():
            out[:, :, self.owned[p]] = U[:, :, : self.n_owned(p)]
        return out


class DevicePart:
    """One part on the current device: a partition context (rkdg_create_part)
    and the device index lists of its halo exchange."""

    def __init__(self, partition: Partition, p: int, **solver_kw):
        import torch

        from .solver import CUDARkdgSolver

        self.p = p
        self.s = CUDARkdgSolver(partition.local_mesh(p), n_owned=partition.n_owned(p), **solver_kw)
        self.limiter = solver_kw.get("limiter") is not None
        rows, mean_rows = self.s.part_rows()
        self.rows = {False: rows, True: mean_rows}
        dev = torch.device("cuda", torch.cuda.current_device())
        self.send = {q: torch.tensor(v, device=dev) for q, v in partition.send[p].items()}
        self.recv = {q: torch.tensor(v, device=dev) for q, v in partition.recv[p].items()}
        self._bufs = {}  # (q, incoming, means_only) -> exchange buffer, allocated once
        self._stream = torch.cuda.ExternalStream(self.s.stream())

    def stream(self):
        return self._stream

    def set_state(self, U, basis="reference"):
        self.s.setFreedom(U, basis=basis)

    def state(self, basis="reference"):
        return self.s.copyFreedomToHost(basis=basis)

    def time_step(self) -> float:
        return self.s.getTimeStep()

    def save_old(self):
        self.s.saveOld()

    def stage(self, st: int, dt: float):
        self.s.stage(st, dt)

    def limit(self):
        self.s.limit()

    def buffer(self, q: int, incoming: bool, means_only: bool):
        """The exchange buffer for rows to (or from) part q: allocated on
        first use and reused by every later exchange, so a captured step
        replays on the same memory (the transports order the reuse)."""
        import torch

        key = (q, incoming, means_only)
        if key not in self._bufs:
            n = (self.recv if incoming else self.send)[q].numel()
            self._bufs[key] = torch.empty((n, self.rows[means_only], 16), dtype=torch.uint8,
                                          device=self.send_device())
        return self._bufs[key]

    def send_device(self):
        import torch

        return torch.device("cuda", torch.cuda.current_device())

    def pack(self, q: int, means_only: bool):
        buf = self.buffer(q, False, means_only)
        idx = self.send[q]
        capi.check(capi.lib().rkdg_gather_rows(self.s.h, idx.data_ptr(), idx.numel(), self.rows[means_only],
                                               buf.data_ptr()))
        return buf

    def unpack(self, q: int, means_only: bool, buf):
        idx = self.recv[q]
        capi.check(capi.lib().rkdg_scatter_rows(self.s.h, idx.data_ptr(), idx.numel(), self.rows[means_only],
                                                buf.data_ptr()))

    def sync(self):
        capi.check(capi.lib().rkdg_sync(self.s.h))

    # -- stream-ordered steps (advance_device)
    def set_final_time(self, t_final: float):
        capi.check(capi.lib().rkdg_part_set_final_time(self.s.h, float(t_final)))

    def wave_out(self, buf):
        """The part's CFL wave-speed maximum into buf (a one-element float64
        device tensor), in stream order."""
        capi.check(capi.lib().rkdg_part_wave(self.s.h, buf.data_ptr(), 0))

    def wave_in(self, buf):
        capi.check(capi.lib().rkdg_part_wave(self.s.h, buf.data_ptr(), 1))

    def begin_step(self):
        capi.check(capi.lib().rkdg_part_begin_step(self.s.h))

    def stage_async(self, st: int):
        capi.check(capi.lib().rkdg_part_stage(self.s.h, st))

    def stage_begin(self, st: int):
        """The tiles that read no halo copy (may run while the copies are
        being refreshed)."""
        capi.check(capi.lib().rkdg_part_stage_begin(self.s.h, st))

    def stage_end(self, st: int):
        capi.check(capi.lib().rkdg_part_stage_end(self.s.h, st))

    def limit_async(self):
        capi.check(capi.lib().rkdg_part_limit(self.s.h))

    def time(self):
        """(time, steps, done) after waiting for the part's stream."""
        t, n, d = C.c_double(), C.c_int32(), C.c_int32()
        capi.check(capi.lib().rkdg_part_time(self.s.h, C.byref(t), C.byref(n), C.byref(d)))
        return t.value, n.value, bool(d.value)

    def close(self):
        self.s.close()


class LocalTransport:
    """Every part held by this process: rows move between the parts'
    buffers on one device, dt is the minimum over them.  With sync=False
    the parts' streams are ordered by events instead of host waits."""

    def __init__(self):
        self._read = {}  # part -> event after its last unpacks (the senders' buffers are free again)

    def exchange(self, parts: dict, means_only: bool, sync: bool = True):
        """Rows between the parts' buffers.  With sync=False no host waits:
        each part packs on its stream once every receiver has read the
        previous exchange's buffers, and unpacks once its senders have
        packed (events between the streams)."""
        self.exchange_end(parts, means_only, self.exchange_begin(parts, means_only, sync), sync)

    def exchange_begin(self, parts: dict, means_only: bool, sync: bool = False):
        """The packing half of an exchange; returns what exchange_end takes."""
        dev = not sync and all(hasattr(part, "stream") for part in parts.values())
        bufs = {}
        done = {}
        for p, part in parts.items():
            if dev:
                for q in part.send:
                    if q in self._read:
                        part.stream().wait_event(self._read[q])
            for q in part.send:
                bufs[(p, q)] = part.pack(q, means_only)
            if dev:
                done[p] = _record(part.stream())
            elif sync:
                part.sync()
        return bufs, done, dev

    def exchange_end(self, parts: dict, means_only: bool, pending, sync: bool = False):
        """The unpacking half: every part's halo rows written."""
        bufs, done, dev = pending
        for p, part in parts.items():
            for q in part.recv:
                if dev:
                    part.stream().wait_event(done[q])
                part.unpack(q, means_only, bufs[(q, p)])
            if dev:
                self._read[p] = _record(part.stream())
            elif sync:
                part.sync()

    def min(self, x: float) -> float:
        return x

    def max_device(self, parts: dict, bufs: dict):
        """bufs[p] (one float64 each, written on part p's stream) all become
        their maximum, in stream order (on the first part's stream)."""
        import torch

        first = next(iter(parts.values())).stream()
        for part in parts.values():
            first.wait_event(_record(part.stream()))
        with torch.cuda.stream(first):
            m = bufs[next(iter(parts))]
            for p in parts:
                torch.maximum(m, bufs[p], out=m)
            for p in parts:
                bufs[p].copy_(m)
        ev = _record(first)
        for part in parts.values():
            part.stream().wait_event(ev)


def _record(stream):
    import torch

    ev = torch.cuda.Event()
    ev.record(stream)
    return ev


class TorchTransport:
    """One part per rank of a torch.distributed process group: the rows of
    every neighbouring pair cross in one batch of point-to-point operations
    (NCCL between GPUs: device to device, ordered on the part's stream; gloo
    between host processes), and dt is an all-reduce minimum."""

    def __init__(self, group=None):
        import torch.distributed as dist

        self.dist = dist
        self.group = group

    def exchange(self, parts: dict, means_only: bool, sync: bool = True):
        self.exchange_end(parts, means_only, self.exchange_begin(parts, means_only, sync), sync)

    def _stream_ctx(self, part):
        import contextlib

        import torch

        return torch.cuda.stream(part.stream()) if hasattr(part, "stream") else contextlib.nullcontext()

    def exchange_begin(self, parts: dict, means_only: bool, sync: bool = False):
        """Packs this rank's rows and starts the batch of sends and receives
        (on the part's stream: NCCL runs them beside what the stream does
        next); returns what exchange_end takes."""
        (p, part), = parts.items()
        with self._stream_ctx(part):
            ops, incoming = [], {}
            for q in sorted(set(part.send) | set(part.recv)):
                if q in part.send:
                    ops.append(self.dist.P2POp(self.dist.isend, part.pack(q, means_only), q, self.group))
                if q in part.recv:
                    incoming[q] = part.buffer(q, True, means_only)
                    ops.append(self.dist.P2POp(self.dist.irecv, incoming[q], q, self.group))
            works = self.dist.batch_isend_irecv(ops) if ops else []
        return works, incoming

    def exchange_end(self, parts: dict, means_only: bool, pending, sync: bool = False):
        """Waits for the transfers (the part's stream waits, not the host)
        and writes the received rows into the halo copies."""
        (p, part), = parts.items()
        works, incoming = pending
        with self._stream_ctx(part):
            for w in works:
                w.wait()
            for q, buf in incoming.items():
                part.unpack(q, means_only, buf)
        if sync:
            part.sync()

    def max_device(self, parts: dict, bufs: dict):
        """The one part's bufs[p] becomes the maximum over all ranks: an
        all-reduce on the part's stream (NCCL keeps it in stream order)."""
        import torch

        (p, part), = parts.items()
        with torch.cuda.stream(part.stream()):
            self.dist.all_reduce(bufs[p], op=self.dist.ReduceOp.MAX, group=self.group)

    def min(self, x: float) -> float:
        import torch

        dev = "cuda" if self.dist.get_backend(self.group) == "nccl" else "cpu"
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MIN, group=self.group)
        return float(t.item())


class DecomposedSolve:
    """The time loop over the parts this process holds ({part: DevicePart}
    or any object with the same methods), with halo exchanges through
    `transport`.  Every process takes the same exchange and reduction steps
    in the same order.  overlap (the device loop): run each stage's halo
    transfers beside the tiles that need no halo copy; by default on for
    transfers between devices (TorchTransport), off for parts that share a
    device, where the rows move by kernels on that device and the second
    launch per stage costs more than it hides (measured on one B200: 0.357
    against 0.342 ms per step with two parts of a 980,000-triangle mesh)."""

    def __init__(self, parts: dict, transport, rk: int = 3, limiter: bool = False, overlap=None):
        self.parts = parts
        self.transport = transport
        self.rk = rk
        self.limiter = limiter
        self.overlap = isinstance(transport, TorchTransport) if overlap is None else bool(overlap)

    def step(self) -> float:
        # halo copies current (so every part's dt sees true neighbour
        # states), then dt as the minimum over all parts
        self.transport.exchange(self.parts, False)
        dt = self.transport.min(min(part.time_step() for part in self.parts.values()))
        for part in self.parts.values():
            part.save_old()
        for st in range(self.rk):
            if st > 0:
                self.transport.exchange(self.parts, False)
            for part in self.parts.values():
                part.stage(st, dt)
            if self.limiter:
                self.transport.exchange(self.parts, True)
                for part in self.parts.values():
                    part.limit()
        return dt

    def advance(self, nsteps: int) -> float:
        t = 0.0
        for _ in range(nsteps):
            t += self.step()
        return t

    def _enqueue_device_step(self, bufs):
        """One step in stream order.  With overlap, each stage's halo
        refresh runs beside the tiles that read no halo copy: start the
        transfers, launch those tiles, finish the transfers, launch the
        rest (two launches per stage instead of one)."""
        parts, tr = self.parts, self.transport
        if not self.overlap:
            tr.exchange(parts, False, sync=False)
            for p, part in parts.items():
                part.wave_out(bufs[p])
            tr.max_device(parts, bufs)
            for p, part in parts.items():
                part.wave_in(bufs[p])
                part.begin_step()
            for st in range(self.rk):
                if st > 0:
                    tr.exchange(parts, False, sync=False)
                for part in parts.values():
                    part.stage_async(st)
                if self.limiter:
                    tr.exchange(parts, True, sync=False)
                    for part in parts.values():
                        part.limit_async()
            return
        for st in range(self.rk):
            pending = tr.exchange_begin(parts, False)
            if st == 0:  # the step's dt from the state at its start (owned elements)
                for p, part in parts.items():
                    part.wave_out(bufs[p])
                tr.max_device(parts, bufs)
                for p, part in parts.items():
                    part.wave_in(bufs[p])
                    part.begin_step()
            for part in parts.values():
                part.stage_begin(st)
            tr.exchange_end(parts, False, pending)
            for part in parts.values():
                part.stage_end(st)
            if self.limiter:
                tr.exchange(parts, True, sync=False)
                for part in parts.values():
                    part.limit_async()

    def advance_device(self, nsteps: int, t_final: float = 0.0, graph: bool = False):
        """nsteps steps (fewer once t_final > 0 is reached) in stream order
        on device parts; returns (time, steps) of the solve.  Every part
        forms dt = cfl / (the maximum of the parts' wave speeds), equal to
        the minimum of their own CFL steps that `step` takes.  With graph
        (parts held by this process, LocalTransport), one step is captured
        as a CUDA graph (the parts' streams forked from and joined to the
        capturing stream) and replayed: one host call per step.  A whole
        step returns the parts' buffer rotation to its start, so every
        replay is the next step."""
        import torch

        parts = self.parts
        if graph and not isinstance(self.transport, LocalTransport):
            raise ValueError("graph replay needs every part in this process (LocalTransport)")
        if getattr(self, "_wave_bufs", None) is None:
            self._wave_bufs = {p: torch.zeros(1, dtype=torch.float64, device=part.send_device())
                               for p, part in parts.items()}
        bufs = self._wave_bufs
        for part in parts.values():
            part.set_final_time(t_final)
        cur = torch.cuda.current_stream()

        def join_parts():  # the parts' streams wait for the replays so far
            ev = _record(cur)
            for part in parts.values():
                part.stream().wait_event(ev)

        g = None
        for n in range(nsteps):
            # with a final time, every 16 steps one host read of the
            # device-resident time ends the loop once the solve is done
            # (every part has the same time)
            if t_final > 0 and n > 0 and n % 16 == 0:
                if g is not None:
                    join_parts()
                if next(iter(parts.values())).time()[2]:
                    break
            if graph and n >= 1:  # the first step runs eagerly: buffers and the wave maximum exist
                if g is None:
                    g = self._capture(bufs)
                    for part in parts.values():
                        cur.wait_event(_record(part.stream()))
                g.replay()
            else:
                self._enqueue_device_step(bufs)
        if g is not None:
            join_parts()
        out = [part.time() for part in parts.values()]
        for part in parts.values():
            part.sync()
        return out[0][0], out[0][1]

    def _capture(self, bufs):
        """One device step as a CUDA graph.  The parts' streams join the
        capture through events from the capturing stream and rejoin it at
        the end; the exchange buffers are the parts' persistent ones."""
        import torch

        parts = self.parts
        if getattr(self, "_graph", None) is not None:
            return self._graph
        torch.cuda.synchronize()  # nothing in flight on the parts' streams while they join the capture
        if isinstance(self.transport, LocalTransport):
            self.transport._read = {}  # a capture may wait only on events recorded inside it
        cap = torch.cuda.Stream()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=cap, capture_error_mode="thread_local"):
            fork = _record(cap)
            for part in parts.values():
                part.stream().wait_event(fork)
            self._enqueue_device_step(bufs)
            for part in parts.values():
                cap.wait_event(_record(part.stream()))
        # events recorded inside the capture order only the graph's own work
        if isinstance(self.transport, LocalTransport):
            self.transport._read = {}
        self._graph = g
        return g
