"""Domain decomposition of one mesh over partitions (tg_part_* of the C ABI).

The reference splits a mesh into METIS partitions, one MPI process each, and
sums the partial residuals, gradients and local time steps of the vertices the
partitions share (src/reduce_residual.cc:14-104, src/fv.cc:827-1030,
src/reduce_dt.cc), with an MPI minimum for dt (src/fv.cc:1602) and a sum for the
residual norms (src/reduce_res_norm.cc:25).  Here partition q owns a contiguous
range of the solver's Hilbert-ordered vertices and keeps every vertex its owned
vertices' gather lists reach as a ghost; the owner alone computes a vertex, in
the one-partition summation order, so any partition count reproduces the
one-partition solve bit for bit.  A step is

    begin;  per stage r: gradients(r), halo(GRAD), flux(r), halo(STATE);  scalars

where halo(field) packs 8 doubles per shared vertex, moves them with an
all-to-all and unpacks them into the ghost slots, and scalars all-gathers each
partition's dt minimum and norm sums so every partition forms the same dt and
norms.  With overlap (the default) every phase runs as two launches, the interior
tiles (no ghost among their vertices) while an exchange is in flight and the
frontier tiles after it landed (run_step).  Two transports implement the exchange:

* :class:`LocalExchange` -- all partitions in this process, device copies
  ordered by CUDA events (one GPU, or several GPUs driven by one process);
* :class:`DistExchange` -- one partition per rank over ``torch.distributed``
  (NCCL over NVLink between GPUs), the layout of one process per GPU.

Every call is enqueued on the partition handle's CUDA stream; nothing waits on
the host inside a step.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi, gpu

HALO_STATE, HALO_GRAD = 0, 1
TILES_ALL, TILES_FRONTIER, TILES_INTERIOR = 0, 1, 2
WIDTH = 8        # doubles per vertex in a halo record
REC = 5          # 8-byte words per partition in the scalar exchange
_ip = C.POINTER(C.c_int)


def _i(a: np.ndarray):
    return a.ctypes.data_as(_ip)


def plan(problem: abi.Problem, n_parts: int, part: int) -> dict:
    """Host-only plan of one partition (tg_part_plan): owned and ghost vertices
    (caller indices, owned first), per-peer counts and the local positions of the
    send and receive entries."""
    L = gpu.load()
    out4 = np.zeros(4, np.int32)
    st = L.tg_part_plan(C.byref(problem.mesh), C.byref(problem.bc), n_parts, part, _i(out4), None, None, None,
                        None, None)
    if st != 0:
        raise gpu.TensumError(st, L.tg_last_error(None).decode())
    n_own, n_ghost, n_send, n_recv = (int(x) for x in out4)
    local = np.zeros(n_own + n_ghost, np.int32)
    sc, rc = np.zeros(n_parts, np.int32), np.zeros(n_parts, np.int32)
    si, ri = np.zeros(max(1, n_send), np.int32), np.zeros(max(1, n_recv), np.int32)
    st = L.tg_part_plan(C.byref(problem.mesh), C.byref(problem.bc), n_parts, part, _i(out4), _i(local), _i(sc),
                        _i(rc), _i(si), _i(ri))
    if st != 0:
        raise gpu.TensumError(st, L.tg_last_error(None).decode())
    return dict(n_owned=n_own, n_ghost=n_ghost, local=local, send_counts=sc, recv_counts=rc, send_idx=si[:n_send],
                recv_idx=ri[:n_recv])


def needs_gradients(problem: abi.Problem) -> bool:
    """Whether the stages form reconstruction gradients (TeCNO fluxes above first order)."""
    m = problem.material
    return m.flux_scheme in (abi.FLUX["kepes_tecno_roe"], abi.FLUX["kepes_tecno_rusanov"]) and \
        m.reconstruct_scheme != abi.RECON["first"]


class Partition:
    """One partition handle on one device with its exchange buffers (torch tensors)."""

    def __init__(self, problem: abi.Problem, n_parts: int, part: int, device: int = 0):
        import torch
        self.L = gpu.load()
        self.problem = problem
        self.device = torch.device("cuda", device)
        self.nv = problem.geom.n_vertex
        h = C.c_void_p()
        with torch.cuda.device(self.device):
            st = self.L.tg_part_create(C.byref(problem.mesh), C.byref(problem.material), C.byref(problem.bc),
                                       C.byref(problem.options), n_parts, part, C.byref(h))
            if st != 0:
                raise gpu.TensumError(st, self.L.tg_last_error(None).decode())
            self.h = h
            info = np.zeros(8, np.int32)
            self.send_counts = np.zeros(n_parts, np.int32)
            self.recv_counts = np.zeros(n_parts, np.int32)
            self._chk(self.L.tg_part_info(self.h, _i(info), _i(self.send_counts), _i(self.recv_counts)))
            (self.n_parts, self.part, self.n_owned, self.n_ghost, self.n_send, self.n_recv, self.n_tiles,
             self.n_frontier) = (int(x) for x in info)
            self.send_off = np.concatenate([[0], np.cumsum(self.send_counts)]) * WIDTH
            self.recv_off = np.concatenate([[0], np.cumsum(self.recv_counts)]) * WIDTH
            f64 = dict(dtype=torch.float64, device=self.device)
            self.send = torch.zeros(max(1, self.n_send * WIDTH), **f64)
            self.recv = torch.zeros(max(1, self.n_recv * WIDTH), **f64)
            self.sc_out = torch.zeros(REC, dtype=torch.int64, device=self.device)
            self.sc_all = torch.zeros(n_parts * REC, dtype=torch.int64, device=self.device)
            sp = C.c_void_p()
            self._chk(self.L.tg_stream(self.h, C.byref(sp)))
            self.stream = torch.cuda.ExternalStream(sp.value, device=self.device)
            self.done = torch.cuda.Event()      # the exchange buffers of this partition are free again
            self.cstream = torch.cuda.Stream(device=self.device)   # copies of the local exchange
            self.copied = torch.cuda.Event()    # this partition's receive buffer is filled
        self.n_rks = 4 if problem.options.time_scheme == 1 else 3
        self.grads = needs_gradients(problem)

    def _chk(self, st):
        if st != 0:
            raise gpu.TensumError(st, self.L.tg_last_error(self.h).decode())

    def _call(self, name, *args):
        import torch
        with torch.cuda.device(self.device):
            self._chk(getattr(self.L, name)(self.h, *args))

    def close(self):
        if getattr(self, "h", None):
            self.L.tg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def query(self, key: str) -> float:
        out = C.c_double()
        self._call("tg_query", gpu.QUERY[key], C.byref(out))
        return out.value

    # ---- state: the whole mesh's PrimVar records in the caller's order
    def set_state(self, prim: np.ndarray, t0: float = 0.0):
        prim = np.ascontiguousarray(prim, np.float64)
        self._call("tg_set_state", gpu._d(prim), self.nv, t0)

    def get_state(self, out: np.ndarray) -> np.ndarray:
        """Writes the records of the vertices this partition owns into `out` (n_vertex, 5)."""
        if out.shape != (self.nv, 5) or out.dtype != np.float64 or not out.flags.c_contiguous:
            raise ValueError("out must be a C-contiguous float64 array of shape (n_vertex, 5)")
        self._call("tg_get_state", gpu._d(out), self.nv)
        return out

    # ---- one step's phases
    def prime(self):
        self._call("tg_part_prime")

    def begin(self):
        self._call("tg_part_begin")

    def gradients(self, r: int, tiles: int = TILES_ALL):
        self._call("tg_part_gradients", r, tiles)

    def flux(self, r: int, tiles: int = TILES_ALL):
        self._call("tg_part_flux", r, tiles)

    def pack(self, field: int):
        self._call("tg_part_pack", field, C.c_void_p(self.send.data_ptr()))

    def unpack(self, field: int):
        self._call("tg_part_unpack", field, C.c_void_p(self.recv.data_ptr()))

    def export(self):
        self._call("tg_part_export", C.c_void_p(self.sc_out.data_ptr()))

    def import_(self):
        self._call("tg_part_import", C.c_void_p(self.sc_all.data_ptr()))

    def scalars(self) -> np.ndarray:
        """Waits for the stream: elapsed time, dt, relative residual, iterations."""
        info = np.empty(4)
        self._call("tg_part_scalars", gpu._d(info))
        return info


class LocalExchange:
    """All partitions in this process.  start(): each sender packs on its stream; each
    receiver's copy stream waits for the senders' packs and copies their segments into
    its receive buffer.  finish(): the receiver's stream waits for its copies and
    unpacks.  Work enqueued between the two (interior tiles) overlaps the copies.  A
    sender packs again only after every receiver has copied, and a receive buffer is
    refilled only after its unpack."""

    def __init__(self, parts):
        self.parts = parts

    def start(self, field: int):
        import torch
        evs = []
        for p in self.parts:
            for q in self.parts:
                if q is not p:
                    p.stream.wait_event(q.copied)
            p.pack(field)
            ev = torch.cuda.Event()
            ev.record(p.stream)
            evs.append(ev)
        for q, own in zip(self.parts, evs):
            q.cstream.wait_event(own)          # joins the copy stream to q's work (and to a capture)
            q.cstream.wait_event(q.done)
            with torch.cuda.stream(q.cstream):
                for p, ev in zip(self.parts, evs):
                    n = int(q.recv_counts[p.part]) * WIDTH
                    if p is q or n == 0:
                        continue
                    q.cstream.wait_event(ev)
                    a, b = int(p.send_off[q.part]), int(q.recv_off[p.part])
                    q.recv[b:b + n].copy_(p.send[a:a + n], non_blocking=True)
            q.copied.record(q.cstream)

    def finish(self, field: int):
        for q in self.parts:
            q.stream.wait_event(q.copied)
            q.unpack(field)
            q.done.record(q.stream)

    def halo(self, field: int):
        self.start(field)
        self.finish(field)

    def scalars(self):
        import torch
        evs = []
        for p in self.parts:
            p.export()
            ev = torch.cuda.Event()
            ev.record(p.stream)
            evs.append(ev)
        for q in self.parts:
            with torch.cuda.stream(q.stream):
                for p, ev in zip(self.parts, evs):
                    q.stream.wait_event(ev)
                    q.sc_all[p.part * REC:(p.part + 1) * REC].copy_(p.sc_out, non_blocking=True)
            q.import_()
        for p in self.parts:                  # sc_out is written again only after every copy
            for q in self.parts:
                if q is not p:
                    ev = torch.cuda.Event()
                    ev.record(q.stream)
                    p.stream.wait_event(ev)


class DistTransport:
    """The two collectives of the exchange over a torch.distributed group (any
    backend: NCCL for device tensors, gloo for host tensors)."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group

    def alltoall(self, send, recv, send_counts, recv_counts, width: int = WIDTH, async_op: bool = False):
        return self.dist.all_to_all_single(recv[:int(np.sum(recv_counts)) * width] if recv.numel() else recv,
                                           send[:int(np.sum(send_counts)) * width] if send.numel() else send,
                                           [int(c) * width for c in recv_counts],
                                           [int(c) * width for c in send_counts], group=self.group,
                                           async_op=async_op)

    def allgather(self, mine, everyone):
        self.dist.all_gather_into_tensor(everyone, mine, group=self.group)


class DistExchange:
    """One partition per rank: the collectives run on the partition's stream."""

    def __init__(self, part: Partition, group=None):
        self.p = part
        self.t = DistTransport(group)

    def start(self, field: int):
        """Pack and launch the all-to-all; work enqueued before finish() overlaps it."""
        import torch
        p = self.p
        p.pack(field)
        with torch.cuda.stream(p.stream):
            self.work = self.t.alltoall(p.send, p.recv, p.send_counts, p.recv_counts, async_op=True)

    def finish(self, field: int):
        import torch
        with torch.cuda.stream(self.p.stream):
            self.work.wait()
        self.work = None
        self.p.unpack(field)

    def halo(self, field: int):
        self.start(field)
        self.finish(field)

    def scalars(self):
        import torch
        p = self.p
        p.export()
        with torch.cuda.stream(p.stream):
            self.t.allgather(p.sc_out, p.sc_all)
        p.import_()


def run_step(parts, exchange, overlap: bool = True):
    """One time step of every partition in `parts` with `exchange` as transport.  With
    overlap, each exchange runs while the interior tiles (no ghost among their
    vertices) compute: gradients(I) | finish STATE | gradients(F) | start GRAD |
    flux(I) | finish GRAD | flux(F) | start STATE (the first stage finds no exchange
    in flight; the last stage's completes before the scalar exchange)."""
    n_rks, grads = parts[0].n_rks, parts[0].grads
    for p in parts:
        p.begin()
    if not overlap:
        for r in range(n_rks):
            if grads:
                for p in parts:
                    p.gradients(r)
                exchange.halo(HALO_GRAD)
            for p in parts:
                p.flux(r)
            exchange.halo(HALO_STATE)
        exchange.scalars()
        return
    pending = False
    for r in range(n_rks):
        if grads:
            for p in parts:
                p.gradients(r, TILES_INTERIOR)
            if pending:
                exchange.finish(HALO_STATE)
            for p in parts:
                p.gradients(r, TILES_FRONTIER)
            exchange.start(HALO_GRAD)
            for p in parts:
                p.flux(r, TILES_INTERIOR)
            exchange.finish(HALO_GRAD)
        else:
            for p in parts:
                p.flux(r, TILES_INTERIOR)
            if pending:
                exchange.finish(HALO_STATE)
        for p in parts:
            p.flux(r, TILES_FRONTIER)
        exchange.start(HALO_STATE)
        pending = True
    exchange.finish(HALO_STATE)
    exchange.scalars()


class PartitionedSolver:
    """One mesh in n_parts partitions, all driven by this process (devices[q]
    holds partition q; by default all on cuda:0).  With every partition on one
    device the step -- phases, halo copies and scalar exchange of all partitions
    -- is captured once as a CUDA graph and replayed (graph=True), so issuing a
    step costs one launch however many partitions there are.  overlap: the copies
    run on side streams while the interior tiles compute (run_step)."""

    def __init__(self, problem: abi.Problem, n_parts: int, devices=None, graph: bool = True, overlap: bool = True):
        devices = devices or [0] * n_parts
        self.overlap = overlap
        self.nv = problem.geom.n_vertex
        self.parts = [Partition(problem, n_parts, q, devices[q]) for q in range(n_parts)]
        self.exchange = LocalExchange(self.parts)
        self.graph = graph and len(set(devices)) == 1
        self._graph = None

    def set_state(self, prim: np.ndarray, t0: float = 0.0):
        for p in self.parts:
            p.set_state(prim, t0)
        for p in self.parts:
            p.prime()
        self.exchange.scalars()

    def _fresh_events(self):
        import torch
        for p in self.parts:
            p.done = torch.cuda.Event()
            p.copied = torch.cuda.Event()

    def _capture(self):
        """Record one step: the partitions' streams fork from the capture stream
        and join it again, so the graph orders every partition's work."""
        import torch
        dev = self.parts[0].device
        cap = torch.cuda.Stream(device=dev)
        g = torch.cuda.CUDAGraph()
        torch.cuda.synchronize(dev)
        self._fresh_events()          # no wait on events recorded outside the capture
        with torch.cuda.graph(g, stream=cap):
            fork = torch.cuda.Event()
            fork.record(cap)
            for p in self.parts:
                p.stream.wait_event(fork)
            run_step(self.parts, self.exchange, self.overlap)
            for p in self.parts:
                ev = torch.cuda.Event()
                ev.record(p.stream)
                cap.wait_event(ev)
        self._fresh_events()
        self._graph, self._cap = g, cap

    def step(self, n: int) -> np.ndarray:
        if self.graph:
            import torch
            dev = self.parts[0].device
            if self._graph is None:
                self._capture()
            torch.cuda.synchronize(dev)            # the partitions' streams hold set_state / prime
            with torch.cuda.stream(self._cap):
                for _ in range(n):
                    self._graph.replay()
            torch.cuda.synchronize(dev)
        else:
            for _ in range(n):
                run_step(self.parts, self.exchange, self.overlap)
        info = [p.scalars() for p in self.parts]
        return info[0]

    def time_steps(self, n: int) -> float:
        """Device time of n replayed steps (CUDA events on the graph's stream), ms per step."""
        import torch
        if not self.graph:
            raise ValueError("time_steps replays the captured step (graph=True, one device)")
        dev = self.parts[0].device
        if self._graph is None:
            self._capture()
        torch.cuda.synchronize(dev)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(self._cap)
        with torch.cuda.stream(self._cap):
            for _ in range(n):
                self._graph.replay()
        b.record(self._cap)
        b.synchronize()
        return a.elapsed_time(b) / n

    def get_state(self) -> np.ndarray:
        out = np.zeros((self.nv, 5))
        for p in self.parts:
            p.get_state(out)
        return out

    def close(self):
        """Releases the captured graph (it names the handles' memory), then the handles."""
        self._graph = None
        for p in self.parts:
            p.close()


class DistPartitionedSolver:
    """This rank's partition of one mesh (rank r of the group holds partition r).
    With graph=True (NCCL groups) the step -- phases and collectives -- is captured
    once as a CUDA graph on the partition's stream and replayed; every rank captures
    and replays the same sequence."""

    def __init__(self, problem: abi.Problem, group=None, device: int | None = None, graph: bool = False,
                 overlap: bool = True):
        import torch
        import torch.distributed as dist
        n_parts, part = dist.get_world_size(group), dist.get_rank(group)
        self.part = Partition(problem, n_parts, part, torch.cuda.current_device() if device is None else device)
        self.exchange = DistExchange(self.part, group)
        self.nv = problem.geom.n_vertex
        self.graph = graph
        self.overlap = overlap
        self._graph = None

    def set_state(self, prim: np.ndarray, t0: float = 0.0):
        self.part.set_state(prim, t0)
        self.part.prime()
        self.exchange.scalars()

    def _capture(self):
        import torch
        p = self.part
        torch.cuda.synchronize(p.device)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=p.stream):
            run_step([p], self.exchange, self.overlap)
        self._graph = g

    def step(self, n: int) -> np.ndarray:
        if self.graph:
            import torch
            if self._graph is None:
                self._capture()
            with torch.cuda.stream(self.part.stream):
                for _ in range(n):
                    self._graph.replay()
        else:
            for _ in range(n):
                run_step([self.part], self.exchange, self.overlap)
        return self.part.scalars()

    def close(self):
        """Releases the captured graph (it holds the collectives) before the handle."""
        self._graph = None
        self.part.close()

    def get_state(self, out: np.ndarray | None = None) -> np.ndarray:
        """The records this rank owns, written into `out` (others left as they are)."""
        out = np.zeros((self.nv, 5)) if out is None else out
        return self.part.get_state(out)
