"""Benchmark: converged Newton-Raphson solves/s, 2,000-bus grid x 1,024 load scenarios.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference]

One step = one batched Newton solve of every scenario of the batch to
||F||_inf <= 1e-8 pu (max 10 iterations) on the synthetic 2,000-bus grid
(400 PV, 1,599 PQ, Jacobian 3,598 x 3,598), per-bus load factors U(0.8, 1.2).

value      : converged solves/s of the mixed-precision engine (FP32 Jacobian and
             factors, FP64 mismatch / state / convergence test) started from the
             learned warm start (BF16 network trained before the timed region on
             engine solutions at load factors U(0.7, 1.3); flat-start fallback
             for any scenario not converged within the cap).  Inputs resident in
             HBM; device time from CUDA events on the solve stream, network
             inference included.
fp64       : the plain FP64 flat-start engine path on the same batch (the metric's
             denominator); "speedup_vs_fp64" = value / fp64.value.
mixed_flat : the mixed-precision path from the flat start.
e2e        : the headline path through the public API with pinned host buffers:
             H2D of Sbus and D2H of V and the per-scenario mismatch inside the
             timed region.
Multi-GPU (torchrun): every rank solves its own shard (weak scaling, no
collective on the data path); value = all converged solves / max rank time.
--impl reference: the reference's own CPU NewtonSolver (cpu-klu path compiled
from its sources, KLU replaced by the oracle LU) on all host cores, on a
bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import gc
import json
import os
import statistics
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
for _p in (ROOT / "gpu-powerflow_b200", ROOT):
    if str(_p) not in sys.path:
        sys.path.insert(0, str(_p))

import numpy as np  # noqa: E402

METRIC = "NR solves/sec at ||F||inf<=1e-8 pu: plain FP64 vs mixed+warm-start, 1 B200"
UNIT = "converged solves/s"
BATCH = 1024
TOL = 1e-8
C5_TOL = 1e-10  # the gradient case: its 1e-6 relative bar on dL/dP wants V well inside 1e-8
MAX_ITER = 10



# DRAM traffic (read + write) of one Mixed factorization of the 2,000-bus
# grid, per 1,024 scenarios: its 19 level launches captured with ncu at 256
# scenarios (72.2 MB read; the writes stay in L2 at that size), scaled by 4
# (the read traffic grows with the batch; a capture at 1,024 scenarios read
# 278.8 MB and wrote 11.9 MB)
FACTOR_DRAM_BYTES_B1024 = 288_800_000

def _peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": float(d["hbm_gbs"]), "bf16_tflops": float(d["bf16_tflops"]), "source": "measured"}
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "source": "fallback"}


class ClockSampler:
    """SM clocks and throttle reasons during the timed region (reads only, no
    settings).  Sampled every 20 ms by an nvidia-smi child process, so that
    this process's threads and interpreter lock do not thin the samples;
    NVML from a background thread when nvidia-smi is absent."""

    # clocks_event_reasons.active bits (nvml.h nvmlClocksEventReason*)
    BITS = ((0x8, "hw_slowdown"), (0x40, "hw_thermal_slowdown"), (0x20, "sw_thermal_slowdown"),
            (0x4, "sw_power_cap"), (0x80, "hw_power_brake"))
    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"),
               ("hw_power_brake", "nvmlClocksEventReasonHwPowerBrakeSlowdown"))

    def __init__(self, index: int, uuid: str | None = None, period: float = 0.01):
        self.index, self.uuid, self.period = index, uuid, period
        self.sm, self.reasons, self.max_mhz = [], set(), None
        self._stop = None
        self._proc = None
        self._path = None

    def parse(self, text: str) -> None:
        """Lines of 'clocks.sm, clocks.max.sm, clocks_event_reasons.active'."""
        for line in text.splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) != 3:
                continue
            try:
                sm, mx, bits = float(parts[0]), float(parts[1]), int(parts[2], 16)
            except ValueError:
                continue
            self.sm.append(sm)
            self.max_mhz = mx
            for bit, name in self.BITS:
                if bits & bit:
                    self.reasons.add(name)

    def _start_smi(self) -> bool:
        import shutil
        import subprocess
        import tempfile

        exe = shutil.which("nvidia-smi")
        if not exe:
            return False
        fd, self._path = tempfile.mkstemp(suffix=".csv")
        target = f"GPU-{self.uuid}" if self.uuid else str(self.index)
        with os.fdopen(fd, "w") as out:
            self._proc = subprocess.Popen(
                [exe, "-i", target, "--query-gpu=clocks.sm,clocks.max.sm,clocks_event_reasons.active",
                 "--format=csv,noheader,nounits", "-lms", "20"], stdout=out, stderr=subprocess.DEVNULL)
        t0 = time.time()
        while time.time() - t0 < 5.0 and os.path.getsize(self._path) == 0 and self._proc.poll() is None:
            time.sleep(0.02)
        if os.path.getsize(self._path) > 0:
            with open(self._path) as f:  # samples from before the timed region do not count
                self._skip = len(f.read().splitlines())
            return True
        self._end_smi()
        return False

    def _end_smi(self) -> str:
        text = ""
        if self._proc is not None:
            self._proc.terminate()
            try:
                self._proc.wait(timeout=5)
            except Exception:
                self._proc.kill()
            self._proc = None
        if self._path:
            with open(self._path) as f:
                text = f.read()
            os.unlink(self._path)
            self._path = None
        return text

    def __enter__(self):
        # both samplers run; nvidia-smi's samples are used when it produced any
        self._skip = 0
        self.source = None
        self._nvml = ([], set(), None)
        self._start_smi()
        import threading
        try:
            import pynvml as nv
            nv.nvmlInit()
            h = nv.nvmlDeviceGetHandleByIndex(self.index)
            nv_max = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
        except Exception:
            return self
        self._stop = threading.Event()
        sm, reasons = [], set()
        self._nvml = (sm, reasons, nv_max)

        def run():
            while True:
                try:
                    sm.append(float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)))
                    bits = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                    for name, attr in self.REASONS:
                        if bits & getattr(nv, attr, 0):
                            reasons.add(name)
                except Exception:
                    pass
                if self._stop.wait(self.period):
                    break
        self._thread = threading.Thread(target=run, daemon=True)
        self._thread.start()
        return self

    def __exit__(self, *a):
        if self._stop is not None:
            self._stop.set()
            self._thread.join(timeout=5)
        if self._proc is not None:
            lines = self._end_smi().splitlines()
            self.parse("\n".join(lines[self._skip:]))
        if self.sm:
            self.source = "nvidia-smi, every 20 ms"
        elif self._nvml[0]:
            self.sm, self.reasons, self.max_mhz = list(self._nvml[0]), set(self._nvml[1]), self._nvml[2]
            self.source = "NVML from a thread, every 10 ms"

    def summary(self) -> dict:
        return {"sm_mhz": statistics.median(self.sm) if self.sm else None, "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons), "samples": len(self.sm), "source": self.source}


def _launch_ranks(n: int) -> int:
    """``--gpus N`` outside torchrun: run this script as N local ranks (one per
    GPU) through torch.distributed.run on 127.0.0.1 and return its exit code."""
    import socket
    import subprocess

    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
           "--master-addr=127.0.0.1", f"--master-port={port}", str(Path(__file__).resolve()), *sys.argv[1:]]
    return subprocess.run(cmd).returncode


def _dist():
    """World, rank and local rank from torchrun's environment; the process
    group is NCCL on GPUs (communicator set-up logged by NCCL_DEBUG=INFO,
    INIT lines only), gloo where CUDA is absent."""
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1 and not dist.is_initialized():
        import datetime
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            os.environ.setdefault("NCCL_DEBUG", "INFO")
            os.environ.setdefault("NCCL_DEBUG_SUBSYS", "INIT")
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def _barrier(world: int) -> None:
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def _reduce(value: float, op: str, world: int, device) -> float:
    """Max or sum of a per-rank number over the ranks (every rank gets it)."""
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    if dist.get_backend() == "gloo":
        device = "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def factor_bytes_per_scenario(solver, elem: int) -> int:
    """Algorithmic bytes of one factorization for one scenario: read J (elem * nnzJ),
    read F (8 * dimF), write the U rows (elem * sum nc*fsz) and y (elem * dimF)."""
    inf = solver.info()
    fsz = solver.plan_array("fp_fsz").astype(np.int64)
    nc = solver.plan_array("fp_nc").astype(np.int64)
    return int(elem * inf["nnz_jacobian"] + 8 * inf["dim_f"] + elem * int((nc * fsz).sum()) + elem * inf["dim_f"])


def make_solver(grid, compute, graph: bool = True):
    import cupf
    o = cupf.NewtonOptions()
    o.backend = cupf.BackendKind.CUDA
    o.compute = compute
    o.custom.serial_nd = True
    o.use_cuda_graph = graph  # one Newton iteration captured once, replayed per iteration
    s = cupf.NewtonSolver(o)
    s.initialize(grid.indptr, grid.indices, grid.data, grid.n_bus, grid.n_bus, grid.pv, grid.pq)
    return s


def run_engine(args) -> None:
    import torch

    import cupf
    from cupf import grids
    from cupf.sharding import scenario_shard

    if torch.cuda.device_count() < int(os.environ.get("WORLD_SIZE", "1")):
        sys.exit(f"bench.py: the engine needs one CUDA device per rank ({torch.cuda.device_count()} visible)")
    world, rank, local = _dist()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    g = grids.grid_2000()
    B = args.batch
    # weak scaling: every rank solves its own contiguous shard of B scenarios
    s_all = g.scenarios(B * world, seed=9100)
    lo_, hi_ = scenario_shard(B * world, rank, world)
    sbus_h = np.ascontiguousarray(s_all[lo_:hi_])
    v0_h = g.flat_start(B)
    sbus = torch.tensor(sbus_h, device=dev)
    v0 = torch.tensor(v0_h, device=dev)
    cfg = cupf.NRConfig(tolerance=TOL, max_iter=MAX_ITER)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)  # > 126 MB L2
    stream = torch.cuda.current_stream(dev)

    mixed = make_solver(g, cupf.ComputePolicy.Mixed, graph=not args.no_graph)
    fp64 = make_solver(g, cupf.ComputePolicy.FP64, graph=not args.no_graph)

    # learned warm start: trained before the timed region on engine solutions
    ws, warm_info = None, None
    if not args.no_warm:
        from cupf.warm_start import WarmStart

        t0 = time.perf_counter()
        ws = WarmStart(g, hidden=1024, layers=3, seed=0)
        X, Y, keep = ws.generate(mixed, args.train, lo=0.7, hi=1.3, seed=777)
        t1 = time.perf_counter()
        hist = ws.fit(X, Y, epochs=args.epochs, batch=1024, lr=2e-3)
        torch.cuda.synchronize(dev)
        warm_info = {"train_scenarios": int(X.shape[0]), "drawn": args.train, "load_range": [0.7, 1.3],
                     "epochs": args.epochs, "generate_s": round(t1 - t0, 2),
                     "train_s": round(time.perf_counter() - t1, 2), "final_train_loss": hist[-1],
                     "net": "loads+PV setpoints 4400 -> 3 x 1024 GELU -> 3598 (+ input skip into the output layer)",
                     "output_layer": "least-squares refit on the trained hidden features; inference with split "
                                     "bf16 hi+lo weights"}
        del X, Y, keep

    def step_flat(solver):
        v, fm, it = solver.solve_batch_device(sbus, v0, config=cfg)
        return v, fm, it, 0, solver.info()["last_kernel_launches"]

    def step_warm():
        v, fm, it, nfb = ws.solve(mixed, sbus, cfg)
        launches = mixed.info()["last_kernel_launches"] + 1 + (ws.mlp.layers + 1)
        return v, fm, it, nfb, launches

    def timed(step, steps: int, warmup: int):
        for _ in range(warmup):
            step()
        _barrier(world)
        torch.cuda.synchronize(dev)
        times, conv, iters, fb, launches = [], 0, 0, 0, 0
        gc.collect()
        gc.disable()  # (a collection pass inside a step would delay its launches)
        for _ in range(steps):
            flush.fill_(1.0)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            v, fm, it, nfb, nl = step()
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
            conv += int((fm <= TOL).sum().item())
            iters, fb, launches = it, fb + nfb, launches + nl
        gc.enable()
        torch.cuda.synchronize(dev)
        _barrier(world)
        return {"ms": statistics.mean(times), "conv": conv / steps, "iters": iters, "fallback": fb / steps,
                "launches": launches, "v": v}

    def agg(r):
        ms = _reduce(r["ms"], "max", world, dev)
        return _reduce(r["conv"], "sum", world, dev) / (ms / 1e3), ms

    # first solve of each solver at this batch size: tunes the factor
    # launches and captures the solve graph, outside the profiled range
    step_flat(mixed)
    step_flat(fp64)
    if ws:
        step_warm()
    torch.cuda.synchronize(dev)
    # the timed legs sit between cudaProfilerStart/Stop, so a profiler started
    # with profiling off (ncu --profile-from-start off) sees exactly them
    uuid = None
    try:
        uuid = str(torch.cuda.get_device_properties(dev).uuid)
    except Exception:
        pass
    with ClockSampler(local, uuid) as clk:
        torch.cuda.profiler.start()
        r_mix = timed(lambda: step_flat(mixed), args.steps, args.warmup)
        r_64 = timed(lambda: step_flat(fp64), args.steps, args.warmup)
        r_warm = timed(step_warm, args.steps, args.warmup) if ws else None
        torch.cuda.profiler.stop()
    value_mix, ms_mix = agg(r_mix)
    value_64, ms_64 = agg(r_64)
    head = r_warm if ws else r_mix
    value, ms_head = agg(head)

    # accuracy of every timed leg against the FP64 oracle run to 1e-12, every
    # scenario of the batch (after the timed region; the oracle solves the
    # batch on all host cores)
    acc = None
    if rank == 0:
        acc = accuracy_vs_oracle(g, sbus_h, v0_h, {"headline": head["v"], "fp64_flat": r_64["v"],
                                                   "mixed_flat": r_mix["v"]})

    # e2e: public API with pinned host buffers (H2D of Sbus + D2H of V and the
    # per-scenario results inside the timed region)
    sbus_p = torch.from_numpy(sbus_h).pin_memory()
    v0_p = torch.from_numpy(v0_h).pin_memory()
    if ws:
        v_host = torch.empty(B, g.n_bus, dtype=torch.complex128).pin_memory()
        fm_host = torch.empty(B, dtype=torch.float64).pin_memory()

        def e2e_step():
            s_dev = sbus_p.to(dev, non_blocking=True)
            v, fm, _, _ = ws.solve(mixed, s_dev, cfg)
            v_host.copy_(v, non_blocking=True)
            fm_host.copy_(fm, non_blocking=True)
            torch.cuda.synchronize(dev)
            return int((fm_host <= TOL).sum())
        h2d = B * g.n_bus * 16
        d2h = B * g.n_bus * 16 + B * 8
    else:
        sb, vb = sbus_p.numpy(), v0_p.numpy()

        def e2e_step():
            r = mixed.solve_batch(g.indptr, g.indices, g.data, g.n_bus, g.n_bus, sb, vb, g.pv, g.pq, cfg)
            return int(r.converged_numpy.sum())
        h2d = 2 * B * g.n_bus * 16
        d2h = B * g.n_bus * 16 + B * (4 + 8 + 1)
    for _ in range(args.warmup):
        e2e_step()
    _barrier(world)
    torch.cuda.synchronize(dev)
    t_e2e, conv_e2e = [], 0
    for _ in range(args.steps):
        flush.fill_(1.0)
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        conv_e2e += e2e_step()
        t_e2e.append((time.perf_counter() - t0) * 1e3)
    ms_e2e_serial = _reduce(statistics.mean(t_e2e), "max", world, dev)
    e2e_serial_value = _reduce(conv_e2e / args.steps, "sum", world, dev) / (ms_e2e_serial / 1e3)

    # e2e pipelined (cupf.streaming.HostPipeline): the same steps as a stream
    # of batches; step k+1's upload and step k-1's download overlap step k's
    # solve.  Every step still copies its Sbus in and its V and norms out;
    # the L2 flush runs inside each step, before its solve.
    from cupf.streaming import HostPipeline

    # three solve lanes: more engine handles, so batches solve at once on
    # their own streams (one batch's latency-bound phases overlap another's
    # wide ones); primed like the first before any timing.  (A fourth lane
    # measured within 1-2 % of three.)
    extra_lanes = []
    for _ in range(2):
        sv = make_solver(g, cupf.ComputePolicy.Mixed, graph=not args.no_graph)
        step_flat(sv)
        if ws:
            ws.solve(sv, sbus, cfg)
        extra_lanes.append(sv)
    mixed2, mixed3 = extra_lanes
    torch.cuda.synchronize(dev)

    def make_pipe(lanes):
        if ws:
            # the network of a step runs on its own stream ahead of the step's solve
            def pipe_prepare(s_dev, slot):
                return ws.predict_standardized(s_dev, slot=slot)

            def lane(sv):
                def pipe_solve(s_dev, pred):
                    flush.fill_(1.0)
                    v, fm, _, _ = ws.solve(sv, s_dev, cfg, pred=pred)
                    return v, fm
                return pipe_solve
            return HostPipeline([lane(sv) for sv in lanes], dev, prepare=pipe_prepare)
        v0_dev = v0

        def lane(sv):
            def pipe_solve(s_dev):
                flush.fill_(1.0)
                v, fm, _ = sv.solve_batch_device(s_dev, v0_dev, config=cfg)
                return v, fm
            return pipe_solve
        return HostPipeline([lane(sv) for sv in lanes], dev)

    # each lane count: three runs of K_E2E steps (at least 20: a stream of
    # batches, so that filling and draining the pipeline weigh little), the
    # median run reported; every run's ms per step is listed in the line
    # The warm-up steps of a pipeline with L lanes cover its 2 L slots (each
    # slot's network buffers are allocated at its first use).
    K_E2E = max(args.steps, 20)
    W_E2E = max(args.warmup, 2 * 3 + 2)
    v_bufs = [torch.empty(B, g.n_bus, dtype=torch.complex128).pin_memory() for _ in range(4)]
    fm_bufs = [torch.empty(B, dtype=torch.float64).pin_memory() for _ in range(max(K_E2E, W_E2E))]
    e2e_lanes, e2e_runs = {}, {}
    for nl, lanes in ((1, [mixed]), (2, [mixed, mixed2]), (3, [mixed, mixed2, mixed3])):
        pipe = make_pipe(lanes)
        pipe.run([sbus_p] * W_E2E, [v_bufs[k % 4] for k in range(W_E2E)], fm_bufs[:W_E2E])
        runs = []
        for _ in range(3):
            _barrier(world)
            torch.cuda.synchronize(dev)
            t0 = time.perf_counter()
            pipe.run([sbus_p] * K_E2E, [v_bufs[k % 4] for k in range(K_E2E)], fm_bufs[:K_E2E])
            ms_l = _reduce((time.perf_counter() - t0) * 1e3 / K_E2E, "max", world, dev)
            conv_l = sum(int((f <= TOL).sum()) for f in fm_bufs[:K_E2E])
            runs.append((ms_l, _reduce(conv_l / K_E2E, "sum", world, dev) / (ms_l / 1e3)))
        runs.sort()
        e2e_lanes[nl] = runs[1]
        e2e_runs[nl] = [round(r[0], 4) for r in runs]
    ms_e2e, e2e_value = e2e_lanes[3]

    # the warm start on 4,096 held-out scenarios from its training distribution
    # (per-bus U(0.7, 1.3), a seed the training draws do not use): warm against
    # flat start, in batches of the timed size, outside the timed region
    heldout = None
    if ws:
        rng = np.random.default_rng(31337)
        hw = {"scenarios": 0, "load_range": [0.7, 1.3], "warm_norm_evaluations": [], "flat_norm_evaluations": [],
              "converged_warm": 0, "converged_flat": 0, "fallback_to_flat": 0}
        dv_warm, dv_flat, within = 0.0, 0.0, 0
        for _ in range(max(1, 4096 // B)):
            f = rng.uniform(0.7, 1.3, size=(B, g.n_bus))
            s_np = g.sgen[None, :] - f * g.sload[None, :]
            s_h = torch.tensor(s_np, device=dev)
            v_w, fm_w, it_w, nfb_w = ws.solve(mixed, s_h, cfg)
            v_f, fm_f, it_f = mixed.solve_batch_device(s_h, v0, config=cfg)
            if rank == 0:
                a = accuracy_vs_oracle(g, s_np, v0_h, {"warm": v_w, "flat": v_f})
                dv_warm = max(dv_warm, a["warm"]["max_abs_dV_vs_fp64_oracle"])
                dv_flat = max(dv_flat, a["flat"]["max_abs_dV_vs_fp64_oracle"])
                within += a["warm"]["within_1e-8"]
            hw["scenarios"] += B
            hw["warm_norm_evaluations"].append(int(it_w))
            hw["flat_norm_evaluations"].append(int(it_f))
            hw["converged_warm"] += int((fm_w <= TOL).sum())
            hw["converged_flat"] += int((fm_f <= TOL).sum())
            hw["fallback_to_flat"] += int(nfb_w)
        if rank == 0:
            hw["accuracy"] = {"max_abs_dV_vs_fp64_oracle_warm": dv_warm, "max_abs_dV_vs_fp64_oracle_flat": dv_flat,
                              "scenarios_checked": hw["scenarios"], "warm_within_1e-8": within}
        heldout = hw

    # roofline of the dominant kernel (the front factorization): stage timers
    # (CUDA events around each stage's launches) over one extra Mixed solve
    # launched stage by stage, outside the timed region
    prof = make_solver(g, cupf.ComputePolicy.Mixed, graph=False)
    prof.solve_batch_device(sbus, v0, config=cfg)
    prof.set_profiling(True)
    flush.fill_(1.0)
    prof.solve_batch_device(sbus, v0, config=cfg)
    st = prof.stage_times()
    prof.set_profiling(False)
    fact_ms, _ = st["factorize"]
    n_fact = max(1, r_mix["iters"] - 1)
    per_fact_ms = fact_ms / n_fact
    fbytes = factor_bytes_per_scenario(prof, 4) * B
    peaks = _peaks()
    achieved = fbytes / (per_fact_ms / 1e3) / 1e9
    # DRAM bytes (read + write) of the level launches of one Mixed
    # factorization at 1,024 scenarios, from one ncu capture of this
    # workload; scaled by the batch
    traffic = int(FACTOR_DRAM_BYTES_B1024 * B / 1024) if g.n_bus == 2000 else None

    extras = run_extras(args, dev) if (rank == 0 and world == 1 and not args.no_extra) else None

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(g, args.cpu_sample)

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_head, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f64 state/mismatch, f32 Jacobian+factors" + (", bf16 warm-start network" if ws else ""),
            "data": "synthetic: seeded 2,000-bus grid, per-bus load factors U(0.8,1.2)",
            "config": {"workload": "2000-bus x 1024-scenario batched NR, mixed precision, "
                                   + ("learned warm start" if ws else "flat start"),
                       "grid_buses": g.n_bus, "jacobian_dim": g.dim_f, "batch_per_gpu": B, "tolerance": TOL,
                       "max_iter": MAX_ITER, "warm_start": warm_info or "none",
                       "l2": "256 MB buffer written between steps",
                       "iterations": int(head["iters"]), "converged_per_step": head["conv"],
                       "cuda_graph": not args.no_graph,
                       "fallback_per_step": head["fallback"]},
            "fp64": {"value": round(value_64, 1), "ms_per_step": round(ms_64, 4), "iterations": int(r_64["iters"]),
                     "converged_per_step": r_64["conv"], "start": "flat"},
            "mixed_flat": {"value": round(value_mix, 1), "ms_per_step": round(ms_mix, 4),
                           "iterations": int(r_mix["iters"]), "converged_per_step": r_mix["conv"]},
            "speedup_vs_fp64": round(value / value_64, 3) if value_64 else None,
            "accuracy": acc,
            "warm_start_heldout": heldout,
            "e2e": {"value": round(e2e_value, 1), "unit": UNIT, "h2d_bytes_per_step": B * g.n_bus * 16,
                    "d2h_bytes_per_step": B * g.n_bus * 16 + B * 8, "ms_per_step": round(ms_e2e, 4),
                    "method": "cupf.streaming.HostPipeline over pinned host batches with three solve lanes "
                              "(three engine handles, streams and worker threads; batches round-robin): each "
                              "step uploads its Sbus and downloads its V and final norms; uploads, network "
                              "inference and downloads overlap the solves, and up to three solves run at once; "
                              "median of three runs of %d steps" % K_E2E,
                    "runs_ms_per_step": e2e_runs[3],
                    "two_lanes": {"value": round(e2e_lanes[2][1], 1), "ms_per_step": round(e2e_lanes[2][0], 4),
                                  "runs_ms_per_step": e2e_runs[2], "method": "the same pipeline with two solve lanes"},
                    "one_lane": {"value": round(e2e_lanes[1][1], 1), "ms_per_step": round(e2e_lanes[1][0], 4),
                                 "runs_ms_per_step": e2e_runs[1], "method": "the same pipeline with one solve lane"},
                    "serial": {"value": round(e2e_serial_value, 1), "ms_per_step": round(ms_e2e_serial, 4),
                               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                               "method": "upload, solve, download one after the other"}},
            "roofline": {"kernel": "k_front_factor (all level launches of one factorization)", "bound": "hbm",
                         "achieved": round(achieved, 1), "peak": peaks["hbm_gbs"], "unit": "GB/s",
                         "frac": round(achieved / peaks["hbm_gbs"], 4), "traffic": traffic,
                         "algorithmic_bytes": fbytes, "ms_per_factorization": round(per_fact_ms, 4),
                         "peak_source": peaks["source"]},
            "stage_ms_per_solve": {k: round(v[0], 4) for k, v in st.items()},
            "other_configs": extras,
            "cpu_baseline": cpu,
            "gpu_launches": int(head["launches"]),
            "clocks": clk.summary(),
        }
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def run_extras(args, dev) -> dict:
    """The other configurations of the workload, measured after the headline:
    the uneven multi-grid batch, the differentiable 10,000-bus case and the
    118-bus grid at batch 1."""
    import torch

    import cupf
    from cupf import grids
    from cupf.batching import UnevenBatch

    out = {}
    cfg = cupf.NRConfig(tolerance=TOL, max_iter=MAX_ITER)
    # uneven batch: 118/500/2,000/10,000 buses x 256/128/96/32 instances, one
    # engine and CUDA stream per grid, solved concurrently (mixed, flat start)
    inst = grids.uneven_grids()
    ub = UnevenBatch([g for g, _ in inst])
    ub_flat = UnevenBatch([g for g, _ in inst], prioritize=False)
    S = [torch.tensor(g.scenarios(c, seed=600 + i), device=dev) for i, (g, c) in enumerate(inst)]
    V0 = [torch.tensor(g.flat_start(c), device=dev) for g, c in inst]
    for _ in range(2):
        ub.solve(S, V0, cfg)
        ub_flat.solve(S, V0, cfg)
    res = {}
    for mode, u, conc in (("concurrent", ub, True), ("concurrent_equal_priority", ub_flat, True),
                          ("sequential", ub, False)):
        ts, conv = [], 0
        for _ in range(3):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            r = u.solve(S, V0, cfg, concurrent=conc)
            e1.record()
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
            conv = sum(int((fm <= TOL).sum()) for _, fm, _ in r)
        res[mode] = {"ms": round(statistics.mean(ts), 3), "converged": conv,
                     "value": round(conv / (statistics.mean(ts) / 1e3), 1)}
    # every instance of the last concurrent solve against the FP64 oracle
    r = ub.solve(S, V0, cfg, concurrent=True)
    per_grid = {}
    for i, ((g, c), (v, _, _)) in enumerate(zip(inst, r)):
        a = accuracy_vs_oracle(g, S[i].cpu().numpy(), V0[i].cpu().numpy(), {"v": v})
        per_grid[str(g.n_bus)] = {"max_abs_dV_vs_fp64_oracle": a["v"]["max_abs_dV_vs_fp64_oracle"],
                                  "within_1e-8": a["v"]["within_1e-8"], "scenarios_checked": c}
    res["accuracy"] = per_grid
    out["uneven_batch"] = {"instances": sum(c for _, c in inst),
                           "grids": [[g.n_bus, c] for g, c in inst], "unit": UNIT,
                           "method": "one engine + CUDA stream per grid, host thread per grid; streams prioritized "
                                     "by grid size (largest first) unless stated", **res}
    # differentiable large case: 10,000 buses x 64, mixed forward through the
    # torch autograd wrapper, loss = sum (Vm - 1)^2, backward = adjoint J^T solve.
    # Warm start: every scenario starts from the converged nominal-load state
    # (solved once per grid, outside the timed region); the flat start is
    # timed beside it.
    from cupf.warm_start import nominal_state

    g = grids.grid_10000()
    o = cupf.NewtonOptions()
    o.backend = cupf.BackendKind.CUDA
    o.compute = cupf.ComputePolicy.Mixed
    o.custom.serial_nd = True
    o.use_cuda_graph = True  # the forward solve as one graph launch
    s = cupf.NewtonSolver(o)
    s.initialize(g.indptr, g.indices, g.data, g.n_bus, g.n_bus, g.pv, g.pq)
    B = 64
    lp, lq = g.load_scenarios(B, seed=808)
    base_re = torch.tensor(g.sgen.real, device=dev, dtype=torch.float32)
    base_im = torch.tensor(g.sgen.imag, device=dev, dtype=torch.float32)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    vnom = nominal_state(s, g, device=dev)
    torch.cuda.synchronize()
    setup_ms = (time.perf_counter() - t0) * 1e3
    v0 = torch.tensor(g.v0, device=dev)
    starts = {"flat": (torch.angle(v0).float(), torch.abs(v0).float()),
              "warm": (torch.angle(vnom).float(), torch.abs(vnom).float())}
    c5cfg = cupf.NRConfig(tolerance=C5_TOL, max_iter=20)
    # the problem the forward solves: Sbus from FP32 base and loads (the Mixed
    # torch dtype) differenced in FP64, and the PV and slack magnitudes of the
    # FP32 start (both starts round them alike)
    f32 = lambda x: x.astype(np.float32).astype(np.float64)
    sb_h = (f32(g.sgen.real)[None, :] - f32(lp)) + 1j * (f32(g.sgen.imag)[None, :] - f32(lq))
    S = torch.tensor(sb_h, device=dev)
    va0, vm0 = starts["flat"]
    v0_h = np.repeat((vm0.double() * torch.exp(1j * va0.double())).cpu().numpy()[None, :], B, axis=0)
    c5 = {}
    for name, (va0, vm0) in starts.items():
        tf, tb = [], []
        for rep in range(4):
            load_p = torch.tensor(lp, device=dev, dtype=torch.float32, requires_grad=True)
            load_q = torch.tensor(lq, device=dev, dtype=torch.float32, requires_grad=True)
            e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
            e0.record()
            va, vm = cupf.solve(load_p, load_q, s, sbus_base_re=base_re, sbus_base_im=base_im, v0_va=va0,
                                v0_vm=vm0, config=c5cfg)
            loss = ((vm - 1.0) ** 2).sum()
            e1.record()
            loss.backward()
            e2.record()
            e2.synchronize()
            if rep:
                tf.append(e0.elapsed_time(e1))
                tb.append(e1.elapsed_time(e2))
        # the same start through the device entry point (FP64 V out): Newton
        # norms and the oracle check
        V0 = (vm0.double() * torch.exp(1j * va0.double()))[None, :].expand(B, -1).contiguous()
        V, fm, it = s.solve_batch_device(S, V0, config=c5cfg)
        c5[name] = {"forward_ms": round(statistics.mean(tf), 3), "backward_ms": round(statistics.mean(tb), 3),
                    "newton_norms": int(it), "converged": int((fm <= C5_TOL).sum()), "V": V,
                    "grad_p": load_p.grad.double().cpu().numpy(), "grad_q": load_q.grad.double().cpu().numpy(),
                    "loss": float(loss.item())}
    from oracle.oracle import Oracle

    acc = accuracy_vs_oracle(g, sb_h, v0_h, {k: c5[k].pop("V") for k in c5})
    orc = Oracle()
    checked = (0, 21, 42, 63)
    adj = []
    for b in checked:
        V = orc.solve(g, sb_h[b], v0_h[b], tol=1e-12, max_iter=30)["V"]
        adj.append(orc.adjoint(g, V, np.zeros(g.n_bus), 2.0 * (np.abs(V) - 1.0)))
    for k in c5:
        gp, gq = c5[k].pop("grad_p"), c5[k].pop("grad_q")
        c5[k]["grad_rel_err_vs_fp64_oracle_adjoint"] = max(
            float(np.abs(gx[b] - a[key]).max() / np.abs(a[key]).max())
            for b, a in zip(checked, adj) for gx, key in ((gp, "grad_p"), (gq, "grad_q")))
        c5[k]["max_abs_dV_vs_fp64_oracle"] = acc[k]["max_abs_dV_vs_fp64_oracle"]
        c5[k]["within_1e-8"] = acc[k]["within_1e-8"]
    out["c5_10000x64"] = {"forward_ms": c5["warm"]["forward_ms"], "backward_ms": c5["warm"]["backward_ms"],
                          "warm": c5["warm"], "flat": c5["flat"], "warm_setup_ms": round(setup_ms, 1),
                          "tolerance": C5_TOL, "scenarios_checked": B, "gradient_scenarios_checked": list(checked),
                          "path": "cupf.solve (CuPFFunction), mixed, CUDA graph; warm start = the converged nominal-load "
                                  "state (nominal_state, once per grid, untimed); backward = J^T solve on the "
                                  "final-state factors; dV vs the FP64 oracle (1e-12, from the flat start) on the "
                                  "same problem (FP32 inputs: Sbus, PV and slack magnitudes); gradients vs the oracle's FP64 adjoint at its solution"}
    # single systems: the 118-bus grid at batch 1 (the reference's CPU-runnable
    # case), FP64 flat start, one graph per solve, device time per solve and
    # through the host API (Sbus and V0 in, V out); the 118-bus grid (C1) and,
    # for the reference's published batch-1 figure, the 2,000-bus grid
    for key, make in (("c1_118_batch1", grids.grid_118), ("c2_2000_batch1", grids.grid_2000)):
        g1 = make()
        s1 = {}
        for name, comp in (("fp64", cupf.ComputePolicy.FP64), ("mixed", cupf.ComputePolicy.Mixed)):
            o = cupf.NewtonOptions()
            o.backend = cupf.BackendKind.CUDA
            o.compute = comp
            o.custom.serial_nd = True
            o.use_cuda_graph = True
            sv = cupf.NewtonSolver(o)
            sv.initialize(g1.indptr, g1.indices, g1.data, g1.n_bus, g1.n_bus, g1.pv, g1.pq)
            S1 = torch.tensor(g1.scenarios(1, seed=5), device=dev)
            V1 = torch.tensor(g1.flat_start(1), device=dev)
            sh, vh = g1.scenarios(1, seed=5), g1.flat_start(1)
            for _ in range(5):
                sv.solve_batch_device(S1, V1, config=cfg)
                sv.solve_batch(g1.indptr, g1.indices, g1.data, g1.n_bus, g1.n_bus, sh, vh, g1.pv, g1.pq, cfg)
            ts, th = [], []
            for _ in range(50):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                _, fm1, it1 = sv.solve_batch_device(S1, V1, config=cfg)
                e1.record()
                e1.synchronize()
                ts.append(e0.elapsed_time(e1))
                t0 = time.perf_counter()
                r1 = sv.solve_batch(g1.indptr, g1.indices, g1.data, g1.n_bus, g1.n_bus, sh, vh, g1.pv, g1.pq, cfg)
                th.append((time.perf_counter() - t0) * 1e3)
            s1[name] = {"device_ms": round(statistics.median(ts), 4), "host_api_ms": round(statistics.median(th), 4),
                        "iterations": int(it1), "converged": bool(r1.converged_numpy.all())}
        out[key] = {**s1, "method": "batch of 1 (single-system schedule: the factorization as one launch over "
                                  "the front tree); median of 50 solves"}
    return out


def accuracy_vs_oracle(g, sbus_h, v0_h, results: dict) -> dict:
    """max |V - V_oracle| over every scenario of each result (complex [B][n]
    tensors or arrays), the oracle being the FP64 CPU restatement run to
    ||F||inf <= 1e-12 from the same start on all host cores."""
    from oracle.oracle import Oracle

    ref = Oracle().solve_many(g, sbus_h, v0_h, tol=1e-12, max_iter=30, threads=os.cpu_count() or 1)
    out = {"oracle": "FP64 CPU restatement (oracle/pf_oracle.c) to 1e-12",
           "oracle_max_final_mismatch": float(ref["final_mismatch"].max())}
    for name, v in results.items():
        v = v.cpu().numpy() if hasattr(v, "cpu") else np.asarray(v)
        dv = np.abs(v - ref["V"]).max(axis=1)
        out[name] = {"max_abs_dV_vs_fp64_oracle": float(dv.max()), "scenarios_checked": int(dv.size),
                     "within_1e-8": int((dv <= 1e-8).sum())}
    return out


def cpu_baseline(g, sample: int) -> dict:
    """The reference's own CPU path (or the oracle port) on all host cores."""
    from oracle import oracle as orc
    threads = os.cpu_count() or 1
    S = g.scenarios(sample, seed=4242)
    V0 = g.flat_start(sample)
    kind = "reference" if orc.reference_available() else "port"
    solver = orc.Reference() if kind == "reference" else orc.Oracle()
    t0 = time.perf_counter()
    r = solver.solve_many(g, S, V0, TOL, MAX_ITER, threads)
    dt = time.perf_counter() - t0
    conv = int((r["final_mismatch"] <= TOL).sum())
    # the same path on one core, on a smaller slice of the same scenarios
    n1 = max(8, sample // 16)
    t1 = time.perf_counter()
    r1 = solver.solve_many(g, S[:n1], V0[:n1], TOL, MAX_ITER, 1)
    dt1 = time.perf_counter() - t1
    conv1 = int((r1["final_mismatch"] <= TOL).sum())
    return {"value": round(conv / dt, 2), "unit": UNIT, "cores": threads, "kind": kind,
            "sample": f"{sample} scenarios of the 2,000-bus workload, one solver per thread, "
                      f"{'reference cpu-klu NewtonSolver (KLU replaced by the oracle LU)' if kind == 'reference' else 'oracle C port'}",
            "single_core": {"value": round(conv1 / dt1, 2), "unit": UNIT, "cores": 1,
                            "sample": f"the first {n1} of those scenarios on one thread"}}


def run_reference(args) -> None:
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from cupf import grids
    g = grids.grid_2000()
    cb = None
    vals = []
    for _ in range(args.warmup):
        cpu_baseline(g, max(8, args.cpu_sample // 8))
    for _ in range(args.steps):
        cb = cpu_baseline(g, args.cpu_sample)
        vals.append(cb["value"])
    v = statistics.mean(vals)
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": round(v, 2), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * args.cpu_sample / v, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic: seeded 2,000-bus grid, per-bus load factors U(0.8,1.2)",
        "config": {"workload": "2000-bus batched NR on the reference CPU path, bounded sample",
                   "sample_scenarios_per_step": args.cpu_sample, "tolerance": TOL, "max_iter": MAX_ITER},
        "cpu_baseline": cb, "e2e": {"value": round(v, 2), "unit": UNIT, "h2d_bytes_per_step": 0,
                                     "d2h_bytes_per_step": 0}}))


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--batch", type=int, default=BATCH)
    ap.add_argument("--cpu-sample", type=int, default=512)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-warm", action="store_true", help="skip the learned warm start (flat start only)")
    ap.add_argument("--no-graph", action="store_true", help="launch every kernel from the host (no CUDA graph)")
    ap.add_argument("--no-extra", action="store_true", help="skip the uneven-batch and 10,000-bus measurements")
    ap.add_argument("--train", type=int, default=200000, help="warm-start training scenarios (engine-solved)")
    ap.add_argument("--epochs", type=int, default=40)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    world = int(os.environ.get("WORLD_SIZE", "0"))
    if world == 0 and args.gpus > 1:
        sys.exit(_launch_ranks(args.gpus))
    if max(world, 1) != args.gpus:
        sys.exit(f"bench.py: --gpus {args.gpus} but the launcher started {max(world, 1)} ranks")
    if args.impl == "reference":
        run_reference(args)
    else:
        run_engine(args)


if __name__ == "__main__":
    main()
