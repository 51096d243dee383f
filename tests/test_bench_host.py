"""Host-side parts of bench.py, checked without a GPU: the clock sampler's
parsing of nvidia-smi samples (which decides whether a bench line is
accepted), its behaviour where neither nvidia-smi nor NVML answers, and the
multi-rank plumbing (``--gpus N`` launching N ranks, max-over-ranks timing,
per-rank shards) on gloo ranks."""
import shutil
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

import bench  # noqa: E402


def test_clock_samples_and_throttle_reasons_are_parsed():
    c = bench.ClockSampler(0)
    c.parse("1965, 1965, 0x0000000000000000\n"
            "1800, 1965, 0x0000000000000004\n"     # sw_power_cap
            "[N/A], 1965, 0x0\n"                    # skipped
            "1372, 1965, 0x0000000000000048\n")     # hw_slowdown + hw_thermal_slowdown
    c.source = "test"
    s = c.summary()
    assert s["samples"] == 3 and s["sm_mhz"] == 1800.0 and s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == ["hw_slowdown", "hw_thermal_slowdown", "sw_power_cap"]


@pytest.mark.skipif(shutil.which("nvidia-smi") is not None, reason="a GPU machine: the sampler has a source")
def test_sampler_without_a_gpu_reports_no_samples():
    with bench.ClockSampler(0) as k:
        pass
    s = k.summary()
    assert s["samples"] == 0 and s["sm_mhz"] is None and s["reasons"] == []


def _rank_main(rank, world, port, out):
    import os

    os.environ.update({"WORLD_SIZE": str(world), "RANK": str(rank), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, str(ROOT))
    import torch.distributed as dist

    import bench as b
    from cupf.sharding import scenario_shard

    w, r, local = b._dist()
    assert dist.get_backend() == "gloo" and (w, r, local) == (world, rank, rank)
    b._barrier(w)
    t_max = b._reduce(10.0 + rank, "max", w, "cpu")
    n_sum = b._reduce(float(rank + 1), "sum", w, "cpu")
    lo, hi = scenario_shard(1024 * w, r, w)
    out.put((rank, t_max, n_sum, lo, hi))
    dist.destroy_process_group()


def test_bench_rank_logic_on_two_gloo_ranks():
    """bench.py's rank plumbing on two CPU ranks (gloo): the group comes up from
    torchrun's variables, the step time is the maximum over ranks, converged
    counts add up, and each rank takes its own contiguous 1,024-scenario shard."""
    import socket

    import torch.multiprocessing as mp

    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [11.0, 11.0] and [r[2] for r in res] == [3.0, 3.0]
    assert [(r[3], r[4]) for r in res] == [(0, 1024), (1024, 2048)]


@pytest.mark.skipif(not (ROOT / "oracle" / "_ref" / "libcupf_ref.so").exists() and
                    not (ROOT / "oracle" / "liboracle.so").exists(), reason="the CPU oracle is not built")
def test_bench_gpus_2_launches_two_ranks_and_prints_one_line():
    """`python bench.py --impl reference --gpus 2` outside torchrun starts two
    local ranks through torch.distributed.run; rank 0 prints the one JSON line
    with n_gpus 2 (the reference arm runs on the host cores, so this works
    without a GPU)."""
    import json
    import os
    import subprocess

    env = dict(os.environ)
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK", "MASTER_ADDR", "MASTER_PORT"):
        env.pop(k, None)
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--gpus", "2", "--steps", "1",
                        "--warmup", "3", "--cpu-sample", "16"], capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0


def test_bench_rejects_a_rank_count_other_than_gpus():
    import os
    import subprocess

    env = dict(os.environ, WORLD_SIZE="1", RANK="0", LOCAL_RANK="0")
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--gpus", "2"], capture_output=True, text=True,
                       timeout=300, env=env)
    assert r.returncode != 0 and "--gpus 2 but the launcher started 1 ranks" in r.stderr
