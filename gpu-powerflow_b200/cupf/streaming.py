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
engines, not the SMs).  An optional prepare stage (the warm start's network
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
    batch ahead, and must keep its state in storage of its slot (0 or 1)
    (e.g. ``prepare=lambda s, j: warm.predict_standardized(s, slot=j)`` with
    ``solve=lambda s, p: warm.solve(solver, s, cfg, pred=p)[:2]``)."""

    def __init__(self, solve, device=None, prepare=None):
        import torch

        self.torch = torch
        self.solve = solve
        self.prepare = prepare
        self.dev = torch.device(device or "cuda")
        if self.dev.index is None:  # the worker thread selects the device by index
            self.dev = torch.device("cuda", torch.cuda.current_device())
        self.up = torch.cuda.Stream(self.dev)
        self.down = torch.cuda.Stream(self.dev)
        self.prep = torch.cuda.Stream(self.dev) if prepare is not None else None
        self._slots = None

    def _slot_buffers(self, rows: int, n: int):
        t = self.torch
        if self._slots is None or self._slots[0].shape[0] < rows or self._slots[0].shape[1] != n:
            self._slots = [t.empty(rows, n, dtype=t.complex128, device=self.dev) for _ in range(2)]
        return self._slots

    def run(self, sbus, V_out, fm_out) -> None:
        """sbus: sequence of complex128 [B_k, n] host tensors (pinned, for the
        copies to overlap); V_out[k] (complex128 [B_k, n]) and fm_out[k]
        (float64 [B_k]) receive batch k's voltages and final mismatch norms.
        Output tensors may repeat in the lists: downloads run in batch order
        on one stream.  Returns when every download has landed.

        The solves run in a worker thread, one after another on the caller's
        stream (the engine's solve blocks its thread until the batch is done
        and releases the GIL meanwhile); this thread issues the uploads and
        the prepare stage of the next batch during the current solve."""
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
        slots = self._slot_buffers(max(int(s.shape[0]) for s in sbus), n)
        comp = t.cuda.current_stream(self.dev)
        solved = [None, None]                                # event after the last solve that read each slot
        free = [threading.Semaphore(1), threading.Semaphore(1)]  # the slot's last solve has been issued
        ready: queue.Queue = queue.Queue()
        failure = []

        def worker() -> None:
            try:
                t.cuda.set_device(self.dev)
                with t.cuda.stream(comp):
                    for k in range(K):
                        item = ready.get()
                        if item is None:
                            return
                        j, dst, state, up_ev, prep_ev = item
                        comp.wait_event(up_ev)
                        if prep_ev is not None:
                            comp.wait_event(prep_ev)
                            V, fm = self.solve(dst, state)
                        else:
                            V, fm = self.solve(dst)
                        done = t.cuda.Event()
                        done.record(comp)
                        solved[j] = done
                        self.down.wait_event(done)
                        with t.cuda.stream(self.down):
                            V_out[k].copy_(V, non_blocking=True)
                            fm_out[k].copy_(fm, non_blocking=True)
                        # keep the device results alive until their download ran
                        V.record_stream(self.down)
                        fm.record_stream(self.down)
                        free[j].release()
            except BaseException as e:  # handed to the caller's thread
                failure.append(e)
                for f in free:
                    f.release()

        th = threading.Thread(target=worker, daemon=True)
        th.start()
        issued = 0
        try:
            for k in range(K):
                j = k % 2
                free[j].acquire()           # batch k-2's solve was issued (and its event recorded)
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
                ready.put((j, dst, state, up_ev, prep_ev))
                issued += 1
        finally:
            if issued < K:
                ready.put(None)  # the worker stops after the batches it was given
            th.join()
        self.down.synchronize()  # no copy into the caller's buffers is left running
        if failure:
            raise failure[0]
