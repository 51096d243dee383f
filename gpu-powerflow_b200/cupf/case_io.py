"""The reference's dump-case directory format: read (native) and write.

A case directory holds dump_Ybus.mtx (MatrixMarket coordinate complex),
dump_Sbus.txt and dump_V.txt ("re im" per bus), dump_pv.txt and dump_pq.txt
(one bus index per line) and, optionally, dump_Vref.txt (a reference
solution).

- load_dump_case mirrors cupf::tests::load_dump_case
  (cuPF/tests/dump_case_loader.cpp:210-232) through the engine library's
  pf_case_* entry points;
- save_dump_case mirrors benchmark/common/matpower_data.py:341-359 (same
  file names, MatrixMarket writer, "%.18e" complex pairs, "%d" indices,
  metadata.json);
- replicate_scenarios builds the batch cuPF/tests/cupf_bench.cpp:188-198
  solves: case b scales every Sbus entry by 1 + step * b.
"""
from __future__ import annotations

import ctypes as C
import json
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

from . import _capi


@dataclass
class DumpCaseData:
    """Fields of DumpCaseData (cuPF/tests/dump_case_loader.hpp:14-40)."""

    case_name: str
    rows: int
    cols: int
    indptr: np.ndarray
    indices: np.ndarray
    ybus_data: np.ndarray
    sbus: np.ndarray
    v0: np.ndarray
    pv: np.ndarray
    pq: np.ndarray
    vref: np.ndarray | None = None
    metadata: dict = field(default_factory=dict)

    @property
    def n_bus(self) -> int:
        return self.rows


def load_dump_case(case_dir) -> DumpCaseData:
    """Read a case directory; raises RuntimeError with the reference's message
    for a missing directory or file, a malformed line, an unsupported header,
    an out-of-range entry or mismatched sizes."""
    lib = _capi.load()
    h = C.c_void_p()
    st = lib.pf_case_load(str(case_dir).encode(), C.byref(h))
    if st != 0:
        msg = lib.pf_case_last_error().decode()
        raise (ValueError if st == 1 else RuntimeError)(msg)
    try:
        rows, cols, nnz, npv, npq, hv = (C.c_int32() for _ in range(6))
        lib.pf_case_dims(h, C.byref(rows), C.byref(cols), C.byref(nnz), C.byref(npv), C.byref(npq), C.byref(hv))
        n = rows.value
        indptr = np.zeros(n + 1, np.int32)
        indices = np.zeros(nnz.value, np.int32)
        ybus = np.zeros(nnz.value, np.complex128)
        sbus = np.zeros(n, np.complex128)
        v0 = np.zeros(n, np.complex128)
        pv = np.zeros(npv.value, np.int32)
        pq = np.zeros(npq.value, np.int32)
        vref = np.zeros(n, np.complex128) if hv.value else None
        p = lambda a: None if a is None else a.ctypes.data  # noqa: E731
        lib.pf_case_copy(h, p(indptr), p(indices), p(ybus), p(sbus), p(v0), p(pv), p(pq), p(vref))
        name = lib.pf_case_name(h).decode()
    finally:
        lib.pf_case_destroy(h)
    meta_path = Path(case_dir) / "metadata.json"
    meta = json.loads(meta_path.read_text()) if meta_path.exists() else {}
    return DumpCaseData(name, rows.value, cols.value, indptr, indices, ybus, sbus, v0, pv, pq, vref, meta)


def _write_pairs(path: Path, values) -> None:
    v = np.asarray(values, dtype=np.complex128).reshape(-1)
    np.savetxt(path, np.column_stack((v.real, v.imag)), fmt="%.18e")


def _write_ints(path: Path, values) -> None:
    np.savetxt(path, np.asarray(values).astype(np.int32, copy=False), fmt="%d")


def save_dump_case(output_root, case_name: str, indptr, indices, data, sbus, v0, pv, pq, vref=None,
                   metadata: dict | None = None) -> Path:
    """Write output_root/case_name in the dump-case format; returns the directory.
    Ybus (CSR) goes through scipy's MatrixMarket writer, as the reference's
    writer does, so a symmetric Ybus is stored as its lower triangle."""
    import scipy.io
    import scipy.sparse as sp

    d = Path(output_root) / case_name
    d.mkdir(parents=True, exist_ok=True)
    n = len(indptr) - 1
    y = sp.csr_matrix((np.asarray(data, np.complex128), np.asarray(indices), np.asarray(indptr)), shape=(n, n))
    scipy.io.mmwrite(d / "dump_Ybus.mtx", y)
    _write_pairs(d / "dump_Sbus.txt", sbus)
    _write_pairs(d / "dump_V.txt", v0)
    _write_ints(d / "dump_pv.txt", pv)
    _write_ints(d / "dump_pq.txt", pq)
    if vref is not None:
        _write_pairs(d / "dump_Vref.txt", vref)
    meta = {"case_name": case_name, "n_bus": int(n), "ybus_nnz": int(y.nnz), "n_pv": int(len(pv)),
            "n_pq": int(len(pq)), "n_ref": int(n - len(pv) - len(pq))}
    meta.update(metadata or {})
    (d / "metadata.json").write_text(json.dumps(meta, indent=2, sort_keys=True), encoding="utf-8")
    return d


def save_grid(output_root, grid, case_name: str | None = None, vref=None) -> Path:
    """Write a synthetic grid (cupf.grids.Grid) as a dump case."""
    return save_dump_case(output_root, case_name or f"synthetic_{grid.n_bus}", grid.indptr, grid.indices,
                          grid.data, grid.sbus, grid.v0, grid.pv, grid.pq, vref=vref)


def replicate_scenarios(case: DumpCaseData, batch: int, load_scale_step: float = 0.001):
    """(sbus [batch, n], v0 [batch, n]) with case b's Sbus scaled by
    1 + load_scale_step * b and every V0 the case's start voltage."""
    scale = 1.0 + load_scale_step * np.arange(batch, dtype=np.float64)
    sbus = case.sbus[None, :] * scale[:, None]
    v0 = np.repeat(case.v0[None, :], batch, axis=0)
    return np.ascontiguousarray(sbus), np.ascontiguousarray(v0)
