"""Uneven multi-grid batches: several grids' scenario sets solved together on
one GPU.

Each grid has its own engine (symbolic plan, Ybus, workspace), so instances of
different grids cannot share one kernel launch of this engine.  They share
the device instead: every grid's batched Newton solve runs on its own CUDA
stream, driven by its own host thread (the ctypes calls into the engine
release the GIL, and each solve synchronises only its own stream once per
Newton iteration), so the grids' kernels overlap on the GPU and the small
grids' latency-bound launches fill the SMs the large grid leaves idle.

The largest grid sets the pace (its Newton loop is the longest chain of
dependent launches), so with ``prioritize`` the streams get CUDA stream
priorities by grid size: the largest grid's kernels are scheduled first
whenever blocks of several grids wait for free SMs, and the smaller grids
fill in around them.
"""
from __future__ import annotations

import threading

from . import BackendKind, ComputePolicy, NewtonOptions, NewtonSolver, NRConfig


class UnevenBatch:
    def __init__(self, grids, compute=ComputePolicy.Mixed, use_cuda_graph: bool = True, serial_nd: bool = True,
                 prioritize: bool = True):
        import torch

        self.torch = torch
        self.grids = list(grids)
        self.solvers = []
        for g in self.grids:
            o = NewtonOptions()
            o.backend = BackendKind.CUDA
            o.compute = compute
            o.use_cuda_graph = use_cuda_graph
            o.custom.serial_nd = serial_nd
            s = NewtonSolver(o)
            s.initialize(g.indptr, g.indices, g.data, g.n_bus, g.n_bus, g.pv, g.pq)
            self.solvers.append(s)
        if prioritize:
            # (least, greatest) urgency, e.g. (0, -5): a lower number is more
            # urgent; the largest grid gets the most urgent priority
            least, greatest = torch.cuda.Stream.priority_range()
            order = sorted(range(len(self.grids)), key=lambda i: -self.grids[i].n_bus)
            prio = [0] * len(self.grids)
            for rank, i in enumerate(order):
                prio[i] = min(least, greatest + rank)
            self.priorities = prio
            self.streams = [torch.cuda.Stream(priority=p) for p in prio]
        else:
            self.priorities = [0] * len(self.grids)
            self.streams = [torch.cuda.Stream() for _ in self.grids]

    def solve(self, sbus_list, v0_list, config: NRConfig | None = None, concurrent: bool = True):
        """sbus_list[i], v0_list[i]: complex128 CUDA tensors [B_i, n_i] for grid i.
        Returns [(V_i, final_mismatch_i, iterations_i)] in grid order."""
        t = self.torch
        cfg = config or NRConfig()
        out = [None] * len(self.grids)
        errors = []
        producer = t.cuda.current_stream()

        def run(i):
            try:
                st = self.streams[i]
                st.wait_stream(producer)  # inputs were written on the caller's stream
                with t.cuda.stream(st):
                    out[i] = self.solvers[i].solve_batch_device(sbus_list[i], v0_list[i], config=cfg)
            except Exception as e:  # re-raised in the caller's thread
                errors.append(e)

        if concurrent:
            threads = [threading.Thread(target=run, args=(i,)) for i in range(len(self.grids))]
            for th in threads:
                th.start()
            for th in threads:
                th.join()
        else:
            for i in range(len(self.grids)):
                run(i)
        if errors:
            raise errors[0]
        for st in self.streams:
            producer.wait_stream(st)
        return out
