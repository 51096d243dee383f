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
engines, not the SMs).  Events order everything: a solve waits for its
upload, a download waits for its solve, and a slot is overwritten only after
the solve that read it.
"""
from __future__ import annotations


class HostPipeline:
    """solve(sbus_device) -> (V_device, final_mismatch_device) runs one batch
    on the current stream (e.g. ``lambda s: warm.solve(solver, s, cfg)[:2]``
    or ``lambda s: solver.solve_batch_device(s, v0, config=cfg)[:2]``)."""

    def __init__(self, solve, device=None):
        import torch

        self.torch = torch
        self.solve = solve
        self.dev = torch.device(device or "cuda")
        self.up = torch.cuda.Stream(self.dev)
        self.down = torch.cuda.Stream(self.dev)
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
        on one stream.  Returns when every download has landed."""
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
        uploaded = [t.cuda.Event(), t.cuda.Event()]
        solved = [None, None]   # the event after the last solve that read each slot
        inputs = [None, None]

        def upload(k: int) -> None:
            j = k % 2
            with t.cuda.stream(self.up):
                if solved[j] is not None:
                    self.up.wait_event(solved[j])  # the slot's previous reader is done
                dst = slots[j][: sbus[k].shape[0]]
                dst.copy_(sbus[k], non_blocking=True)
                uploaded[j].record(self.up)
            inputs[j] = dst

        upload(0)
        for k in range(K):
            j = k % 2
            if k + 1 < K:
                upload(k + 1)
            comp.wait_event(uploaded[j])
            V, fm = self.solve(inputs[j])
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
        self.down.synchronize()
