"""Build the engine's shared library in-tree (sm_100a only).

    python gpu-powerflow_b200/build.py

Compiles every csrc/*.cu and csrc/*.cpp with nvcc for sm_100a into
_build/*.o (parallel) and links cupf/libcupf_b200.so with the CUDA runtime
and the METIS static library shipped with the CUDA toolkit.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
OUT_DIR = HERE / "_build"
LIB = HERE / "cupf" / "libcupf_b200.so"
CUDA = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
NVCC = str(CUDA / "bin" / "nvcc")
METIS = CUDA / "targets" / "x86_64-linux" / "lib" / "libmetis_static.a"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O3", "--expt-relaxed-constexpr",
          "-I", str(CSRC), "-I", str(HERE.parent / "include")]


def _needs(obj: Path, deps: list[Path]) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(verbose: bool = False, force: bool = False) -> Path:
    OUT_DIR.mkdir(exist_ok=True)
    srcs = sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))
    headers = list(CSRC.glob("*.hpp")) + list(CSRC.glob("*.cuh")) + [HERE.parent / "include" / "cupf_b200.h"]
    jobs = []
    for s in srcs:
        o = OUT_DIR / (s.name + ".o")
        if force or _needs(o, [s] + headers):
            cmd = [NVCC, *ARCH, *COMMON, "-x", "cu" if s.suffix == ".cu" else "c++", "-c", str(s), "-o", str(o)]
            jobs.append((s, cmd))
    def run(job):
        s, cmd = job
        r = subprocess.run(cmd, capture_output=True, text=True)
        return s, r
    failed = []
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        for s, r in ex.map(run, jobs):
            if verbose or r.returncode:
                sys.stderr.write(r.stdout + r.stderr)
            if r.returncode:
                failed.append(s.name)
    if failed:
        raise RuntimeError("nvcc failed for: " + ", ".join(failed))
    objs = [str(OUT_DIR / (s.name + ".o")) for s in srcs]
    if force or jobs or not LIB.exists():
        cmd = [NVCC, *ARCH, "-shared", "-o", str(LIB), *objs, str(METIS), "-lcudart_static", "-ldl", "-lrt",
               "-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode:
            raise RuntimeError("link failed:\n" + r.stdout + r.stderr)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
