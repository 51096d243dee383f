"""The C ABI (include/cupf_b200.h, libcupf_b200.so) and the Python mirror of
the reference's cupf API, exercised without a GPU: symbols, option defaults,
argument checks and error behaviour."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

import cupf
from cupf import _capi
from cupf import grids as G

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "cupf_b200.h"
MLP_HEADER = ROOT / "include" / "cupf_mlp.h"


def declared_functions(header: Path = HEADER, prefixes: str = "pf|cls") -> list[str]:
    text = header.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = re.sub(r"//[^\n]*", "", text)
    names = re.findall(r"\b((?:" + prefixes + r")_[a-z0-9_]+)\s*\(", text)
    seen = []
    for n in names:
        if n not in seen:
            seen.append(n)
    return seen


def test_library_exports_every_declared_symbol():
    lib = _capi.load()
    decl = declared_functions()
    assert len(decl) >= 30
    missing = [n for n in decl if not hasattr(lib, n)]
    assert not missing, f"declared in cupf_b200.h but not exported: {missing}"


def test_binding_table_matches_header():
    assert set(_capi.EXPORTS) == set(declared_functions())


def test_mlp_header_symbols_exported():
    lib = _capi.load()
    decl = declared_functions(MLP_HEADER, "mlp")
    assert set(decl) == set(_capi.MLP_EXPORTS)
    missing = [n for n in decl if not hasattr(lib, n)]
    assert not missing, f"declared in cupf_mlp.h but not exported: {missing}"


def test_mlp_gemm_rejects_bad_shapes():
    """Shape checks run on the host, before any device work."""
    lib = _capi.load()
    assert lib.mlp_gemm_bf16(None, 64, None, 64, 100, 128, 64, 0, None, 128, None, None, 0, None) == 1
    assert b"multiples" in lib.mlp_last_error()
    assert lib.mlp_gemm_bf16(None, 64, None, 64, 128, 128, 64, 9, None, 128, None, None, 0, None) == 1
    assert lib.mlp_gemm_bf16(None, 32, None, 64, 128, 128, 64, 0, None, 128, None, None, 0, None) == 1


def test_library_is_the_in_tree_build():
    lib = _capi.load()
    assert Path(lib._name).resolve().parent == (ROOT / "gpu-powerflow_b200" / "cupf").resolve()


def test_status_strings():
    lib = _capi.load()
    texts = [lib.cls_status_string(i).decode() for i in range(7)]
    assert texts[0] == "success"
    assert len(set(texts)) == 7 and all(texts)


def test_option_defaults_mirror_reference():
    """cuPF/tests/smoke/test_bindings.py:34-46 and newton_solver_types.hpp defaults."""
    o = cupf.NewtonOptions()
    assert o.backend == cupf.BackendKind.CPU
    assert o.compute in (cupf.ComputePolicy.FP64, cupf.ComputePolicy.Mixed)
    assert o.cpu_linear_solver == cupf.CpuLinearSolverKind.KLU
    assert o.cuda_jacobian == cupf.CudaJacobianKind.Edge
    assert o.cuda_linear_solver == cupf.CudaLinearSolverKind.Custom
    assert o.use_cuda_graph is False
    c = cupf.NRConfig()
    assert c.tolerance == 1e-8 and c.max_iter == 50
    cs = cupf.CustomSolverConfig()
    assert cs.max_panel_width == 8 and cs.shift_retry_epsilon == 1e-8
    assert cs.autotune is True  # the engine's own option: per-level factor launch shapes
    assert cs.pivot_strategy == cupf.CustomPivotStrategy.StaticDiagonalShift
    so = cupf.SolveOptions()
    assert so.prepare_adjoint_cache is False
    ao = cupf.AdjointOptions()
    assert ao.compute_load_gradients and ao.use_transpose_solve
    o.compute = cupf.ComputePolicy.FP32
    assert o.compute == cupf.ComputePolicy.FP32
    with pytest.raises(AttributeError):
        cupf.NRConfig(tolerence=1.0)


def test_unsupported_backends_raise():
    with pytest.raises(ValueError):
        cupf.NewtonSolver(cupf.NewtonOptions())  # CPU backend
    o = cupf.NewtonOptions()
    o.backend = cupf.BackendKind.CUDA
    o.cuda_linear_solver = cupf.CudaLinearSolverKind.CuDSS
    with pytest.raises(ValueError):
        cupf.NewtonSolver(o)
    o = cupf.NewtonOptions()
    o.backend = cupf.BackendKind.CUDA
    o.custom.max_panel_width = 9
    with pytest.raises(ValueError):
        cupf.NewtonSolver(o)


def test_fp32_compute_policy_constructs():
    """ComputePolicy.FP32 (FP32 state, mismatch and voltage update; the
    reference's CudaFp32CustomPipeline) is a solver of its own, with the
    reference's float32 tensor dtype (torch_bridge.cpp:133-141), whatever
    factor precision is asked for (FP64 factors fall back to FP32)."""
    for prec in (cupf.CustomPrecision.FP64, cupf.CustomPrecision.FP32, cupf.CustomPrecision.TF32):
        o = cupf.NewtonOptions()
        o.backend = cupf.BackendKind.CUDA
        o.compute = cupf.ComputePolicy.FP32
        o.custom.precision = prec
        s = cupf.NewtonSolver(o)
        assert s.dtype_name == "float32"


def _solver():
    o = cupf.NewtonOptions()
    o.backend = cupf.BackendKind.CUDA
    return cupf.NewtonSolver(o)


def test_solve_before_initialize_raises():
    """cuPF/tests/unit/test_minimal_solver.cpp:37-59."""
    c = G.two_bus_case()
    s = _solver()
    with pytest.raises(RuntimeError):
        s.solve(c["indptr"], c["indices"], c["data"], 2, 2, c["sbus"], c["v0"], c["pv"], c["pq"])


def test_argument_checks():
    c = G.two_bus_case()
    s = _solver()
    with pytest.raises(ValueError):
        s.initialize(c["indptr"][:-1], c["indices"], c["data"], 2, 2, c["pv"], c["pq"])
    with pytest.raises(ValueError):
        s.initialize(c["indptr"], c["indices"], c["data"][:-1], 2, 2, c["pv"], c["pq"])
    with pytest.raises(ValueError):
        s.solve_batch(c["indptr"], c["indices"], c["data"], 2, 2, c["sbus"], c["v0"], c["pv"], c["pq"])
    with pytest.raises(ValueError):
        s.solve(c["indptr"], c["indices"], c["data"], 2, 2, c["sbus"][:1], c["v0"], c["pv"], c["pq"])
    with pytest.raises(ValueError):
        s.solve_adjoint(np.zeros((2, 3)), np.zeros((2, 2)), c["pv"], c["pq"])


def test_bad_pv_pq_rejected_by_analysis():
    """make_jacobian_indexing (jacobian_analysis.cpp:174-222) rejects out-of-range
    buses and an empty pv+pq set."""
    g = G.grid_118()
    s = _solver()
    with pytest.raises(ValueError):
        s.analyze_host(g.indptr, g.indices, g.n_bus, np.zeros(0, np.int32), np.zeros(0, np.int32))
    with pytest.raises(ValueError):
        s.analyze_host(g.indptr, g.indices, g.n_bus, np.array([-1], np.int32), g.pq)
    with pytest.raises(ValueError):
        s.analyze_host(g.indptr, g.indices, g.n_bus, g.pv, np.array([g.n_bus + 5], np.int32))


def test_plan_array_errors():
    g = G.grid_118()
    s = _solver()
    s.analyze_host(g.indptr, g.indices, g.n_bus, g.pv, g.pq)
    with pytest.raises(ValueError):
        s.plan_array("no_such_array")
    with pytest.raises(ValueError):
        s.plan_array64("no_such_array")
    inf = s.info()
    assert inf["n_bus"] == 118 and inf["dim_f"] == g.dim_f
    assert inf["max_panel"] <= 8 and inf["num_levels"] >= 1


def test_linear_solver_state_machine():
    ls = cupf.LinearSolver()
    with pytest.raises(cupf.linear_solver.CustomSolverError) as e:
        ls.analyze()
    assert e.value.status == 2  # INVALID_STATE: analyze before set_data
    with pytest.raises(cupf.linear_solver.CustomSolverError):
        ls.set_data(np.array([0, 1, 3], np.int32), np.array([0], np.int32))  # nnz mismatch
    with pytest.raises(cupf.linear_solver.CustomSolverError):
        cupf.LinearSolver(cupf.SolverConfig(max_panel_width=0))


def test_null_handle_calls_are_rejected():
    lib = _capi.load()
    assert lib.pf_info(None, None) != 0
    assert lib.cls_setup(None, 4) != 0
    assert lib.pf_set_profiling(None, 1) != 0
    assert isinstance(lib.cls_last_error(None), bytes)
    assert isinstance(lib.pf_last_error(None), bytes)


def test_new_options_and_exports_are_checked(tmp_path):
    """autotune must be 0 or 1 and the parallel-ND parameters non-negative;
    the front CSV needs an analysed plan and a writable path."""
    lib = _capi.load()
    for bad in ({"autotune": 2}, {"parallel_nd_depth": -1}, {"parallel_nd_base_small": -5},
                {"parallel_nd_base_large": -1}, {"batch1_schedule": 2}, {"batch1_schedule": -1}):
        c = _capi.ClsConfig(0, 0, 1, 1, 8, 1e-8, 0, 0, 0, 0)
        for k, v in bad.items():
            setattr(c, k, v)
        h = C.c_void_p()
        assert lib.cls_create(C.byref(c), C.byref(h)) != 0, bad
    # zero parallel-ND fields are the defaults
    c = _capi.ClsConfig(0, 0, 1, 1, 8, 1e-8, 0, 0, 0, 0)
    h = C.c_void_p()
    assert lib.cls_create(C.byref(c), C.byref(h)) == 0
    assert lib.cls_dump_fronts_csv(h, str(tmp_path / "f.csv").encode()) != 0  # nothing analysed yet
    lib.cls_destroy(h)
    assert lib.cls_dump_fronts_csv(None, b"x") != 0
    assert lib.pf_dump_fronts_csv(None, b"x") != 0
    g = G.grid_118()
    s = _solver()
    s.analyze_host(g.indptr, g.indices, g.n_bus, g.pv, g.pq)
    with pytest.raises(ValueError):
        s.dump_fronts_csv(tmp_path / "missing_dir" / "f.csv")
    s.dump_fronts_csv(tmp_path / "f.csv")
    lines = (tmp_path / "f.csv").read_text().splitlines()
    assert len(lines) == 1 + s.info()["num_panels"]
