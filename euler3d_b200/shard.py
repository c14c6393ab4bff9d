"""Block sharding: one case split over several processes, one GPU each.

The reference's MPI mode (MPI/src/BlockCommunicator.cpp) gives every rank a
contiguous range of blocks (:29-38, getMyBlocks :284-294), sends the state of
the connexion cells that cross ranks once per outer iteration
(updateBoundaries :66-211) and sums every block's norms and forces for the
output and the stop test (getGlobal :299-339).  Here the library does the
device side (include/e3d.h, e3d_shard_*: a solver over the rank's blocks, and
kernels that pack the halo entries its peers need and unpack what arrives);
this module moves the buffers with torch.distributed:

* ``transport="nccl"``: device buffers, one ``all_to_all_single`` per outer
  iteration, queued on the solver's stream (NVLink / NVSwitch between the
  GPUs of a node);
* ``transport="host"``: the same buffers staged through pinned host memory
  and exchanged on a gloo group (no peer access needed).

Norms and forces travel as the raw per-block sums over a gloo group and are
combined in block order on every rank, so the history of a sharded run is the
single-GPU history bit for bit (the reference's MPI build sums per-rank
partials with MPI_Allreduce, whose order the MPI library chooses).

``LocalShards`` runs every rank's solver in one process on one GPU, moving the
buffers with device copies: the same plan and kernels without a transport.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from .api import Case, Solver


def first_blocks(n_blocks: int, n_ranks: int) -> np.ndarray:
    """The reference's block ranges: n_blocks // n_ranks blocks per rank, one
    more for the first n_blocks % n_ranks ranks (BlockCommunicator.cpp:29-38)."""
    out = np.empty(n_ranks + 1, dtype=np.int32)
    L.check(L.lib().e3d_shard_first_blocks(n_blocks, n_ranks, L.ptr(out)))
    return out


def _ranges(case: Case, n_ranks: int, first_block) -> np.ndarray:
    if first_block is None:
        return first_blocks(case.n_blocks, n_ranks)
    fb = np.ascontiguousarray(first_block, dtype=np.int32)
    if fb.shape != (n_ranks + 1,):
        raise ValueError(f"first_block needs {n_ranks + 1} entries")
    return fb


def plan(case: Case, n_ranks: int, rank: int, first_block=None) -> dict:
    """The halo entries of one rank (host only): per-peer counts, and the
    (block, block-local cell) of each entry in transport order."""
    fb = _ranges(case, n_ranks, first_block)
    sc = np.zeros(n_ranks, dtype=np.int64)
    rc = np.zeros(n_ranks, dtype=np.int64)
    lib = L.lib()
    L.check(lib.e3d_case_shard_plan(case._h, L.ptr(fb), n_ranks, rank, L.ptr(sc), L.ptr(rc), None, None))
    send = np.zeros((int(sc.sum()), 2), dtype=np.int32)
    recv = np.zeros((int(rc.sum()), 2), dtype=np.int32)
    L.check(lib.e3d_case_shard_plan(case._h, L.ptr(fb), n_ranks, rank, L.ptr(sc), L.ptr(rc), L.ptr(send),
                                    L.ptr(recv)))
    return {"first_block": fb, "send_counts": sc, "recv_counts": rc, "send_cells": send, "recv_cells": recv}


class ShardSolver(Solver):
    """The solver of one rank: the case blocks [first_block[rank],
    first_block[rank+1]), block indices local to that range."""

    def __init__(self, case: Case, n_ranks: int, rank: int, first_block=None, precision: str = "fp64",
                 carry_w0: int = -1, use_graph: bool = True, device: int = -1, stream: int | None = None,
                 hist_capacity: int = 4096, renumber: str = "none+boundary_last"):
        lib = L.lib()
        fb = _ranges(case, n_ranks, first_block)
        o = L.Options()
        lib.e3d_default_options(C.byref(o))
        o.precision = L.FP32 if precision == "fp32" else L.FP64
        o.carry_w0 = carry_w0
        o.use_graph = 1 if use_graph else 0
        o.device = device
        o.stream = stream
        o.hist_capacity = hist_capacity
        o.renumber = L.RENUMBER[renumber]
        h = C.c_void_p()
        L.check(lib.e3d_shard_create(case._h, L.ptr(fb), n_ranks, rank, C.byref(o), C.byref(h)))
        self._h = h
        self.case = case
        self.precision = precision
        self.rank, self.n_ranks = rank, n_ranks
        self.first_block = fb
        self.b0, self.b1 = int(fb[rank]), int(fb[rank + 1])
        self.n_blocks = self.b1 - self.b0
        self._info = [case.block_info(b) for b in range(self.b0, self.b1)]
        self.send_counts = np.zeros(n_ranks, dtype=np.int64)
        self.recv_counts = np.zeros(n_ranks, dtype=np.int64)
        L.check(lib.e3d_shard_halo_counts(h, L.ptr(self.send_counts), L.ptr(self.recv_counts)))

    def solve(self, max_iter: int, criterion: float, check_every: int = 1) -> int:
        raise NotImplementedError("a shard's stop test needs every rank's norms: use Sharded.solve")

    def pack(self, send_ptr: int) -> None:
        L.check(L.lib().e3d_shard_pack(self._h, C.c_void_p(send_ptr)))

    def unpack(self, recv_ptr: int) -> None:
        L.check(L.lib().e3d_shard_unpack(self._h, C.c_void_p(recv_ptr)))

    def take_flow_data(self) -> np.ndarray:
        """Raw per-block norms and forces [n][local blocks][10] of the
        iterations run since the last call."""
        lib = L.lib()
        n = C.c_int()
        L.check(lib.e3d_shard_flow_data(self._h, None, 0, C.byref(n)))
        out = np.zeros((n.value, self.n_blocks, 10))
        L.check(lib.e3d_shard_flow_data(self._h, L.ptr(out), out.size, C.byref(n)))
        return out

    def push_flow_data(self, all_blocks: np.ndarray) -> None:
        a = np.ascontiguousarray(all_blocks, dtype=np.float64)
        if a.ndim != 3 or a.shape[1:] != (self.case.n_blocks, 10):
            raise ValueError("flow data must be [iterations][all blocks][10]")
        L.check(L.lib().e3d_shard_push_flow_data(self._h, L.ptr(a), a.shape[0]))


def _stops(h: dict, first: int, max_iter: int, criterion: float) -> int | None:
    # PostProcessing::checkStopSolver (PostProcessing.cpp:77), as e3d_solve applies it
    for i in range(first, len(h["iter"])):
        if h["iter"][i] + 1 == max_iter or h["conv"][i, 0] <= criterion:
            return int(h["iter"][i]) + 1
    return None


class Sharded:
    """One rank of a block-sharded run (call on every rank of ``group``).

    ``transport``: "nccl" (device buffers, all-to-all on the solver stream;
    the default when the group's backend is NCCL) or "host" (pinned host
    buffers over gloo).  Every rank takes the same collective steps in the
    same order, errors included: a rank whose solver fails keeps taking part
    in the exchanges and the status reduction, and then every rank raises.
    """

    def __init__(self, case: Case, group=None, precision: str = "fp64", transport: str | None = None,
                 first_block=None, device: int | None = None, **solver_kw):
        import torch
        import torch.distributed as dist

        self._torch, self._dist = torch, dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        backend = dist.get_backend(group)
        # host-side messages (norms, status) always go through gloo
        self.ctrl = group if backend == "gloo" else dist.new_group(backend="gloo")
        self.transport = transport or ("nccl" if backend == "nccl" else "host")
        if self.transport not in ("nccl", "host"):
            raise ValueError(f"unknown transport {self.transport!r}")
        if self.transport == "nccl" and backend != "nccl":
            raise ValueError("transport 'nccl' needs a process group with the NCCL backend")
        self.device = torch.cuda.current_device() if device is None else device
        torch.cuda.set_device(self.device)
        self.stream = torch.cuda.Stream(self.device)
        self.solver = ShardSolver(case, self.world, self.rank, first_block, precision=precision, device=self.device,
                                  stream=self.stream.cuda_stream, **solver_kw)
        self.case = case
        dt = torch.float64 if precision == "fp64" else torch.float32
        s = self.solver
        self.send_splits = [int(x) * 5 for x in s.send_counts]
        self.recv_splits = [int(x) * 5 for x in s.recv_counts]
        dev = torch.device("cuda", self.device)
        self.send_dev = torch.empty(max(1, sum(self.send_splits)), dtype=dt, device=dev)
        self.recv_dev = torch.empty(max(1, sum(self.recv_splits)), dtype=dt, device=dev)
        if self.transport == "host":
            self.send_host = torch.empty(sum(self.send_splits), dtype=dt).pin_memory()
            self.recv_host = torch.empty(sum(self.recv_splits), dtype=dt).pin_memory()
        self._max_blocks = int(np.max(np.diff(s.first_block)))
        self._error = None
        self._exchange()  # Solver.cpp:48: the halo before the first iteration

    # ---- one halo exchange
    def _exchange(self) -> None:
        torch, dist = self._torch, self._dist
        ok = self._error is None
        if ok:
            try:
                self.solver.pack(self.send_dev.data_ptr())
            except L.E3DError as e:
                self._error, ok = e, False
        n_send, n_recv = sum(self.send_splits), sum(self.recv_splits)
        if self.world == 1:
            pass  # no peers: every connexion is a device copy inside the iteration
        elif self.transport == "nccl":
            with torch.cuda.stream(self.stream):
                dist.all_to_all_single(self.recv_dev[:n_recv], self.send_dev[:n_send], self.recv_splits,
                                       self.send_splits, group=self.group)
        else:
            if ok:
                with torch.cuda.stream(self.stream):
                    self.send_host.copy_(self.send_dev[:n_send], non_blocking=True)
                self.stream.synchronize()
            dist.all_to_all_single(self.recv_host, self.send_host, self.recv_splits, self.send_splits,
                                   group=self.ctrl)
            if ok:
                with torch.cuda.stream(self.stream):
                    self.recv_dev[:n_recv].copy_(self.recv_host, non_blocking=True)
        if ok:
            try:
                self.solver.unpack(self.recv_dev.data_ptr())
            except L.E3DError as e:
                self._error = e

    # ---- norms and forces of every block, in block order, on every rank
    def _gather(self) -> None:
        torch, dist = self._torch, self._dist
        raw = None
        if self._error is None:
            try:
                raw = self.solver.take_flow_data()
            except L.E3DError as e:
                self._error = e
        flag = torch.tensor([0 if self._error is None else 1], dtype=torch.int32)
        dist.all_reduce(flag, op=dist.ReduceOp.MAX, group=self.ctrl)
        if int(flag.item()):
            err, self._error = self._error, None
            raise err if err is not None else L.E3DError(-6, "a solver on another rank failed")
        n = raw.shape[0]
        pad = np.zeros((n, self._max_blocks, 10))
        pad[:, :raw.shape[1]] = raw
        parts = [torch.zeros(pad.shape, dtype=torch.float64) for _ in range(self.world)]
        dist.all_gather(parts, torch.from_numpy(pad), group=self.ctrl)
        fb = self.solver.first_block
        blocks = [p.numpy()[:, :fb[r + 1] - fb[r]] for r, p in enumerate(parts)]
        self.solver.push_flow_data(np.concatenate(blocks, axis=1))

    # ---- the reference's loop (Solver.cpp:83-96), one iteration per exchange
    def step(self, n: int) -> None:
        """n outer iterations with their halo exchanges, queued without
        waiting; the norms stay on the device until ``iterate`` or ``gather``."""
        for _ in range(n):
            if self._error is None:
                try:
                    self.solver.iterate(1)
                except L.E3DError as e:
                    self._error = e
            self._exchange()

    def iterate(self, n: int) -> None:
        self.step(n)
        self._gather()

    def gather(self) -> None:
        """Brings every rank's norms and forces of the iterations since the
        last gather into this rank's history (all ranks call it together)."""
        self._gather()

    def solve(self, max_iter: int, criterion: float, check_every: int = 1) -> int:
        """Iterate until PostProcessing::checkStopSolver fires (max_iter or the
        density criterion, PostProcessing.cpp:77); every rank stops together."""
        check_every = max(1, check_every)
        while True:
            before = len(self.history()["iter"])
            done = before
            self.iterate(min(check_every, max(1, max_iter - done)))
            stop = _stops(self.history(), before, max_iter, criterion)
            if stop is not None:
                return stop
            if len(self.history()["iter"]) >= max_iter:
                return len(self.history()["iter"])

    def history(self) -> dict:
        return self.solver.history()

    def get(self, b: int, name: str) -> np.ndarray:
        """Array of case block b (this rank's blocks only)."""
        if not self.solver.b0 <= b < self.solver.b1:
            raise IndexError(f"block {b} is on another rank")
        return self.solver.get(b - self.solver.b0, name)

    def close(self) -> None:
        self.solver.close()


class LocalShards:
    """Every rank's shard solver in one process on one GPU; the halo moves by
    device-to-device copies on one stream.  Same plan, kernels and history
    combination as ``Sharded``, without a transport."""

    def __init__(self, case: Case, n_ranks: int, precision: str = "fp64", first_block=None, **solver_kw):
        import torch

        self._torch = torch
        self.stream = torch.cuda.Stream()
        self.shards = [ShardSolver(case, n_ranks, r, first_block, precision=precision,
                                   stream=self.stream.cuda_stream, **solver_kw) for r in range(n_ranks)]
        self.case = case
        dt = torch.float64 if precision == "fp64" else torch.float32
        self.send = [torch.empty(max(1, int(s.send_counts.sum()) * 5), dtype=dt, device="cuda") for s in self.shards]
        self.recv = [torch.empty(max(1, int(s.recv_counts.sum()) * 5), dtype=dt, device="cuda") for s in self.shards]
        self._exchange()

    def _exchange(self) -> None:
        torch = self._torch
        for s, b in zip(self.shards, self.send):
            s.pack(b.data_ptr())
        soff = [np.concatenate([[0], np.cumsum(s.send_counts)]) * 5 for s in self.shards]
        roff = [np.concatenate([[0], np.cumsum(s.recv_counts)]) * 5 for s in self.shards]
        with torch.cuda.stream(self.stream):
            for a, sa in enumerate(self.shards):
                for b in range(len(self.shards)):
                    n = int(sa.send_counts[b]) * 5
                    if n:
                        self.recv[b][roff[b][a]:roff[b][a] + n].copy_(self.send[a][soff[a][b]:soff[a][b] + n])
        for s, b in zip(self.shards, self.recv):
            s.unpack(b.data_ptr())

    def iterate(self, n: int) -> None:
        for _ in range(n):
            for s in self.shards:
                s.iterate(1)
            self._exchange()
        raw = [s.take_flow_data() for s in self.shards]
        all_blocks = np.concatenate(raw, axis=1)
        for s in self.shards:
            s.push_flow_data(all_blocks)

    def history(self) -> dict:
        return self.shards[0].history()

    def get(self, b: int, name: str) -> np.ndarray:
        for s in self.shards:
            if s.b0 <= b < s.b1:
                return s.get(b - s.b0, name)
        raise IndexError(b)

    def close(self) -> None:
        for s in self.shards:
            s.close()
