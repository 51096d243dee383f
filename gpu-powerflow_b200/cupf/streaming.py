"""Host-batch pipeline: a stream of batches whose inputs and results live in
pinned host memory, with the copies overlapped with the solves.

The reference's host entry point (NewtonSolver::solve_batch,
newton_solver.cpp:245-342 with CudaBatchedStorage::upload / download_batch,
cuda_batched_storage.cpp:234-407) uploads a batch, solves it and downloads
it, one after the other.  HostPipeline keeps that per-batch contract (each
batch's inputs go host -> device and its results device -> host) but runs
three batches at once on three streams:

    upload stream    H2D of batch k+1 into the free one of two device slots
    caller's stream  the solve of batch k
    download stream  D2H of batch k-1's voltages and final mismatches

so a steady stream of batches costs about max(solve, upload, download) per
batch instead of their sum (PCIe is full duplex; the copies use the copy
engines, not the SMs).  With several solve lanes (one solver handle each),
several batches solve at once on their own streams.  An optional prepare stage (the warm start's network
inference) runs batch k+1 on a fourth stream while batch k solves: the
solve's narrow levels leave SMs idle that the GEMMs can use.  Events order
everything: a prepare and a solve wait for their upload, a solve for its
prepare, a download for its solve, and a slot (input buffer, prepared state)
is overwritten only after the solve that read it.
"""
from __future__ import annotations


class HostPipeline:
    """solve(sbus_device) -> (V_device, final_mismatch_device) runs one batch
    on the current stream (e.g. ``lambda s: warm.solve(solver, s, cfg)[:2]``
    or ``lambda s: solver.solve_batch_device(s, v0, config=cfg)[:2]``).

    With prepare(sbus_device, slot) -> state, the pipeline calls
    solve(sbus_device, state) instead; prepare runs on its own stream, one
    batch ahead, and must keep its state in storage of its slot (e.g.
    ``prepare=lambda s, j: warm.predict_standardized(s, slot=j)`` with
    ``solve=lambda s, p: warm.solve(solver, s, cfg, pred=p)[:2]``).

    solve may also be a list of L such callables, each over its own solver
    handle: batches then go round-robin to L solve lanes, each with its own
    stream and worker thread, so L solves are in flight at once and one
    batch's latency-bound phases (the narrow top of the front tree, the
    small per-iteration kernels) overlap another's wide ones.  Slots number
    2 L; prepare states are per slot."""

    def __init__(self, solve, device=None, prepare=None):
        import torch

        self.torch = torch
        self.solves = list(solve) if isinstance(solve, (list, tuple)) else [solve]
        if not self.solves:
            raise ValueError("HostPipeline: at least one solve lane")
        self.lanes = len(self.solves)
        self.prepare = prepare
        self.dev = torch.device(device or "cuda")
        if self.dev.index is None:  # the worker threads select the device by index
            self.dev = torch.device("cuda", torch.cuda.current_device())
        self.up = torch.cuda.Stream(self.dev)
        self.down = torch.cuda.Stream(self.dev)
        self.prep = torch.cuda.Stream(self.dev) if prepare is not None else None
        # lane 0 solves on the caller's stream (as a single-lane pipeline does),
        # the others on streams of their own
        self.comp = [None] + [torch.cuda.Stream(self.dev) for _ in range(self.lanes - 1)]
        self._slots = None

    def _slot_buffers(self, rows: int, n: int):
        t = self.torch
        ns = 2 * self.lanes
        if self._slots is None or self._slots[0].shape[0] < rows or self._slots[0].shape[1] != n:
            self._slots = [t.empty(rows, n, dtype=t.complex128, device=self.dev) for _ in range(ns)]
        return self._slots

    def run(self, sbus, V_out, fm_out) -> None:
        """sbus: sequence of complex128 [B_k, n] host tensors (pinned, for the
        copies to overlap); V_out[k] (complex128 [B_k, n]) and fm_out[k]
        (float64 [B_k]) receive batch k's voltages and final mismatch norms.
        Output tensors may repeat in the lists: downloads run in batch order
        on one stream.  Returns when every download has landed.

        The solves run in worker threads, one per lane, each lane's batches
        one after another on its stream (the engine's solve blocks its thread
        until the batch is done and releases the GIL meanwhile); this thread
        issues the uploads and the prepare stage ahead of the solves.
        Python's cyclic garbage collector is paused while the batches
        stream (a collection pass holds every thread for up to tens of
        milliseconds) and resumed afterwards."""
        import gc

        resume = gc.isenabled()
        gc.disable()
        try:
            self._run(sbus, V_out, fm_out)
        finally:
            if resume:
                gc.enable()

    def _run(self, sbus, V_out, fm_out) -> None:
        import queue
        import threading

        t = self.torch
        K = len(sbus)
        if len(V_out) != K or len(fm_out) != K:
            raise ValueError("HostPipeline.run: one output pair per input batch")
        if K == 0:
            return
        n = sbus[0].shape[1]
        for k in range(K):
            if sbus[k].dim() != 2 or sbus[k].shape[1] != n or sbus[k].dtype != t.complex128:
                raise ValueError("HostPipeline.run: inputs must be complex128 [B, n] with one n")
            if tuple(V_out[k].shape) != tuple(sbus[k].shape) or fm_out[k].shape[0] != sbus[k].shape[0]:
                raise ValueError("HostPipeline.run: output shapes must match their input batch")
        L = self.lanes
        NS = 2 * L
        slots = self._slot_buffers(max(int(s.shape[0]) for s in sbus), n)
        comp = [c if c is not None else t.cuda.current_stream(self.dev) for c in self.comp]
        solved = [None] * NS                                   # event after the last solve that read each slot
        free = [threading.Semaphore(1) for _ in range(NS)]     # the slot's last solve has been issued
        ready = [queue.Queue() for _ in range(L)]
        down_ready = [threading.Event() for _ in range(K)]     # batch k's solve event is recorded
        done_ev = [None] * K
        failure = []
        lock = threading.Lock()

        def worker(lane: int) -> None:
            cs = comp[lane]
            try:
                t.cuda.set_device(self.dev)
                with t.cuda.stream(cs):
                    while True:
                        item = ready[lane].get()
                        if item is None:
                            return
                        k, j, dst, state, up_ev, prep_ev = item
                        cs.wait_event(up_ev)
                        if prep_ev is not None:
                            cs.wait_event(prep_ev)
                            V, fm = self.solves[lane](dst, state)
                        else:
                            V, fm = self.solves[lane](dst)
                        ev = t.cuda.Event()
                        ev.record(cs)
                        solved[j] = ev
                        # keep the device results alive until their download ran
                        V.record_stream(self.down)
                        fm.record_stream(self.down)
                        done_ev[k] = (ev, V, fm)
                        down_ready[k].set()
                        free[j].release()
            except BaseException as e:  # handed to the caller's thread
                with lock:
                    failure.append(e)
                for f in free:
                    f.release()
                for d in down_ready:
                    d.set()

        def downloader() -> None:
            # downloads in batch order, each after its batch's solve; after a
            # failure, the batches solved before it still land
            try:
                t.cuda.set_device(self.dev)
                for k in range(K):
                    down_ready[k].wait()
                    if done_ev[k] is None:
                        return
                    ev, V, fm = done_ev[k]
                    self.down.wait_event(ev)
                    with t.cuda.stream(self.down):
                        V_out[k].copy_(V, non_blocking=True)
                        fm_out[k].copy_(fm, non_blocking=True)
                    done_ev[k] = None
            except BaseException as e:
                with lock:
                    failure.append(e)

        threads = [threading.Thread(target=worker, args=(l,), daemon=True) for l in range(L)]
        dl = threading.Thread(target=downloader, daemon=True)
        for th in threads:
            th.start()
        dl.start()
        issued = 0
        try:
            for k in range(K):
                j = k % NS
                free[j].acquire()           # the slot's previous batch was issued to its lane
                if failure:
                    break
                up_ev = t.cuda.Event()
                with t.cuda.stream(self.up):
                    if solved[j] is not None:
                        self.up.wait_event(solved[j])  # its reads of the slot come first
                    dst = slots[j][: sbus[k].shape[0]]
                    dst.copy_(sbus[k], non_blocking=True)
                    up_ev.record(self.up)
                state, prep_ev = None, None
                if self.prepare is not None:
                    prep_ev = t.cuda.Event()
                    with t.cuda.stream(self.prep):
                        self.prep.wait_event(up_ev)
                        state = self.prepare(dst, j)
                        prep_ev.record(self.prep)
                ready[k % L].put((k, j, dst, state, up_ev, prep_ev))
                issued += 1
        finally:
            for q in ready:
                q.put(None)  # each worker stops after the batches it was given
            for th in threads:
                th.join()
            if issued < K:
                for d in down_ready:
                    d.set()
            dl.join()
            # after a failure the downloader stops at the first batch without
            # a result; every batch whose solve did finish still lands
            for k in range(K):
                if done_ev[k] is not None:
                    ev, V, fm = done_ev[k]
                    self.down.wait_event(ev)
                    with t.cuda.stream(self.down):
                        V_out[k].copy_(V, non_blocking=True)
                        fm_out[k].copy_(fm, non_blocking=True)
                    done_ev[k] = None
        self.down.synchronize()  # no copy into the caller's buffers is left running
        if failure:
            raise failure[0]
