"""Seeded synthetic transmission grids and load scenarios.

The reference benchmarks on MATPOWER cases (case118, case_ACTIVSg2000, ...)
that are not available here; these generators stand in for them with the
shapes, sizes and value distributions the workloads are quoted on:

* buses uniform in the unit square;
* Euclidean minimum spanning tree plus extra 4-nearest-neighbour edges, drawn
  at random among the 4-NN pairs until the branch target is reached;
* per branch r ~ U(0.005, 0.05) pu, x = r * U(3, 10), line charging
  b ~ U(0, 0.1) pu, pi-model stamped into Ybus;
* one slack bus (Va = 0, Vm = 1) at the best-connected bus, PV buses placed as
  a greedy dominating set with Vm ~ U(0.98, 1.05), the rest PQ;
* loads P ~ 0.3 * LogNormal(ln 0.3, 0.6) pu, Q = P * U(0.1, 0.5);
* PV generation dispatched so that every PV bus angle is 0 in the base case
  (total = load + losses, about 1.00-1.01 x load);
* Sbus = Sgen - Sload, flat start (PV |V| = setpoint).

The three calibrations (random 4-NN extras, dominating PV placement with the
angle-holding dispatch, the 0.3 load factor) exist because with uniformly
random PV buses, shortest-first extra edges, 1.03 x generation and full loads,
no AC solution exists above a few hundred buses and flat-start NR diverges on
every scenario.

Ybus is returned in CSR with column indices sorted inside every row, the layout
``NewtonSolver.initialize`` expects (cuPF/cpp/inc/newton_solver/core/
newton_solver_types.hpp:17-24).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class Grid:
    """One power-flow case: Ybus (CSR), bus types, base injections, flat start."""

    name: str
    n_bus: int
    indptr: np.ndarray          # int32 [n+1]
    indices: np.ndarray         # int32 [nnz]
    data: np.ndarray            # complex128 [nnz]
    pv: np.ndarray              # int32, ascending
    pq: np.ndarray              # int32, ascending
    slack: int
    sgen: np.ndarray            # complex128 [n]: generation injection (P only)
    sload: np.ndarray           # complex128 [n]: base load
    v0: np.ndarray              # complex128 [n]: flat start
    seed: int = 0
    branches: np.ndarray = field(default_factory=lambda: np.zeros((0, 2), np.int64))

    @property
    def sbus(self) -> np.ndarray:
        return self.sgen - self.sload

    @property
    def dim_f(self) -> int:
        return int(self.pv.size + 2 * self.pq.size)

    @property
    def nnz(self) -> int:
        return int(self.indices.size)

    def scenarios(self, batch: int, lo: float = 0.8, hi: float = 1.2,
                  seed: int | None = None) -> np.ndarray:
        """Per-bus independent load scaling U(lo, hi): returns Sbus [batch, n]."""
        rng = np.random.default_rng(self.seed * 7919 + 17 if seed is None else seed)
        f = rng.uniform(lo, hi, size=(batch, self.n_bus))
        return self.sgen[None, :] - f * self.sload[None, :]

    def load_scenarios(self, batch: int, lo: float = 0.8, hi: float = 1.2,
                       seed: int | None = None) -> tuple[np.ndarray, np.ndarray]:
        """Scaled loads (P, Q) [batch, n] for the torch-style entry points."""
        rng = np.random.default_rng(self.seed * 7919 + 17 if seed is None else seed)
        f = rng.uniform(lo, hi, size=(batch, self.n_bus))
        ld = f * self.sload[None, :]
        return ld.real.copy(), ld.imag.copy()

    def flat_start(self, batch: int) -> np.ndarray:
        return np.repeat(self.v0[None, :], batch, axis=0)

    def branch_scaled_ybus(self, batch: int, lo: float = 0.9, hi: float = 1.1,
                           seed: int | None = None) -> np.ndarray:
        """Per-scenario Ybus values [batch, nnz] on this grid's pattern: the
        series admittance between every connected bus pair is scaled by its
        own U(lo, hi) factor (a parameter or contingency sweep; a factor of 0
        takes the pair out of service).  With Y_ij = -y_ij and
        Y_ii = sum_j y_ij + shunt_i, scaling y_ij by f gives
        Y'_ij = f Y_ij and Y'_ii = Y_ii - (f - 1) Y_ij; shunts are kept."""
        rng = np.random.default_rng(self.seed * 104729 + 5 if seed is None else seed)
        rows = np.repeat(np.arange(self.n_bus), np.diff(self.indptr))
        cols = self.indices.astype(np.int64)
        off = rows != cols
        lo_r, hi_c = np.minimum(rows, cols), np.maximum(rows, cols)
        pair = lo_r * self.n_bus + hi_c
        uniq, pid = np.unique(pair[off], return_inverse=True)
        f = rng.uniform(lo, hi, size=(batch, uniq.size))
        y = np.repeat(self.data[None, :], batch, axis=0)
        fo = f[:, pid]                                   # factor of each off-diagonal entry
        y[:, off] = self.data[off][None, :] * fo
        dpos = np.flatnonzero(~off)                      # diagonal positions, one per row
        drow = rows[dpos]
        delta = np.zeros((batch, self.n_bus), np.complex128)
        np.add.at(delta.T, rows[off], (-(fo - 1.0) * self.data[off][None, :]).T)
        y[:, dpos] += delta[:, drow]
        return y


def _mst_edges(xy: np.ndarray) -> np.ndarray:
    """Euclidean MST (Kruskal over the Delaunay edges, which contain it)."""
    from scipy.spatial import Delaunay

    n = xy.shape[0]
    if n == 2:
        return np.array([[0, 1]], dtype=np.int64)
    tri = Delaunay(xy)
    s = tri.simplices
    cand = np.concatenate([s[:, [0, 1]], s[:, [1, 2]], s[:, [0, 2]]])
    cand = np.sort(cand, axis=1)
    cand = np.unique(cand, axis=0)
    length = np.linalg.norm(xy[cand[:, 0]] - xy[cand[:, 1]], axis=1)
    order = np.lexsort((cand[:, 1], cand[:, 0], length))
    parent = np.arange(n)

    def find(a: int) -> int:
        while parent[a] != a:
            parent[a] = parent[parent[a]]
            a = parent[a]
        return a

    out = []
    for e in order:
        a, b = int(cand[e, 0]), int(cand[e, 1])
        ra, rb = find(a), find(b)
        if ra != rb:
            parent[ra] = rb
            out.append((a, b))
            if len(out) == n - 1:
                break
    return np.asarray(out, dtype=np.int64)


def _knn_candidates(xy: np.ndarray, existing: set, k: int = 4) -> np.ndarray:
    """All 4-nearest-neighbour pairs that are not tree edges, as sorted (a, b) rows."""
    from scipy.spatial import cKDTree

    n = xy.shape[0]
    kk = min(k + 1, n)
    _, nb = cKDTree(xy).query(xy, k=kk)
    cand = set()
    for i in range(n):
        for j in np.atleast_1d(nb[i])[1:]:
            a, b = (i, int(j)) if i < int(j) else (int(j), i)
            if (a, b) not in existing:
                cand.add((a, b))
    if not cand:
        return np.zeros((0, 2), dtype=np.int64)
    return np.asarray(sorted(cand), dtype=np.int64)


def _dominating_pv(indptr: np.ndarray, indices: np.ndarray, slack: int, n_pv: int) -> np.ndarray:
    """Greedy dominating-set placement of the PV buses.

    Repeatedly picks the bus that voltage-regulates the most not-yet-covered
    buses (itself and its neighbours), ties to the lowest index.  Spreading the
    regulated buses this way keeps every PQ cluster small, which a uniformly
    random placement does not on large sparse grids.
    """
    n = indptr.size - 1
    nbrs = [indices[indptr[i]:indptr[i + 1]] for i in range(n)]
    covered = np.zeros(n, dtype=bool)
    covered[nbrs[slack]] = True
    covered[slack] = True
    gain = np.array([int((~covered[nb]).sum()) for nb in nbrs], dtype=np.int64)
    taken = np.zeros(n, dtype=bool)
    taken[slack] = True
    out = []
    for _ in range(n_pv):
        g = np.where(taken, -1, gain)
        i = int(np.argmax(g))
        taken[i] = True
        out.append(i)
        for j in nbrs[i]:
            if not covered[j]:
                covered[j] = True
                gain[nbrs[j]] -= 1
    return np.sort(np.asarray(out, dtype=np.int64))


def _polar_nr(Y, sbus: np.ndarray, v0: np.ndarray, pv: np.ndarray, pq: np.ndarray,
              tol: float = 1e-10, max_iter: int = 30) -> np.ndarray:
    """Dense-free scipy Newton-Raphson used only while *building* a grid."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spl

    V = v0.astype(np.complex128).copy()
    va, vm = np.angle(V), np.abs(V)
    pvpq = np.r_[pv, pq]
    npvpq = pvpq.size
    for _ in range(max_iter):
        I = Y @ V
        mis = V * np.conj(I) - sbus
        F = np.r_[mis[pvpq].real, mis[pq].imag]
        if np.abs(F).max() <= tol:
            return V
        dV, dI, dVn = sp.diags(V), sp.diags(I), sp.diags(V / np.abs(V))
        dS_dVm = dV @ (Y @ dVn).conj() + dI.conj() @ dVn
        dS_dVa = 1j * dV @ (dI - Y @ dV).conj()
        J = sp.bmat([[dS_dVa[pvpq][:, pvpq].real, dS_dVm[pvpq][:, pq].real],
                     [dS_dVa[pq][:, pvpq].imag, dS_dVm[pq][:, pq].imag]]).tocsc()
        dx = spl.spsolve(J, F)
        va[pvpq] -= dx[:npvpq]
        vm[pq] -= dx[npvpq:]
        V = vm * np.exp(1j * va)
        if not np.all(np.isfinite(V)):
            break
    raise RuntimeError("grid construction: dispatch power flow did not converge")


def make_grid(n_bus: int, n_branch: int, n_pv: int, seed: int, name: str = "",
              load_scale: float = 0.3, max_draws: int = 16) -> Grid:
    """Build one seeded synthetic grid (see module docstring for the recipe).

    A draw whose base case has no flat-start Newton solution within 8
    iterations (or four +-30 % per-bus load draws more than 9) is rejected and redrawn from seed + 7919 * k (k = 1, 2, ...);
    the seed actually used is stored on the grid.
    """
    last = None
    for k in range(max_draws):
        s = seed + 7919 * k
        try:
            g = _draw_grid(n_bus, n_branch, n_pv, s, name, load_scale)
        except RuntimeError as e:
            last = e
            continue
        if _flat_start_ok(g):
            return g
        last = RuntimeError(f"seed {s}: base case does not converge from flat start")
    raise RuntimeError(f"no solvable draw for {n_bus} buses: {last}")


def _flat_start_ok(g: "Grid", max_iter: int = 8) -> bool:
    import scipy.sparse as sp

    Y = sp.csr_matrix((g.data, g.indices, g.indptr), shape=(g.n_bus, g.n_bus))
    pv, pq = g.pv.astype(np.int64), g.pq.astype(np.int64)
    try:
        # the base case, and four +-30 % per-bus load draws (the stress the
        # load scenarios put on the single slack bus)
        _polar_nr(Y, g.sbus, g.v0, pv, pq, tol=1e-8, max_iter=max_iter)
        rng = np.random.default_rng(g.seed + 3)
        for _ in range(4):
            f = rng.uniform(0.7, 1.3, size=g.n_bus)
            _polar_nr(Y, g.sgen - f * g.sload, g.v0, pv, pq, tol=1e-8, max_iter=max_iter + 1)
    except (RuntimeError, FloatingPointError, ValueError):
        return False
    return True


def _draw_grid(n_bus: int, n_branch: int, n_pv: int, seed: int, name: str,
               load_scale: float) -> Grid:
    if n_bus < 2:
        raise ValueError("a grid needs at least two buses")
    import scipy.sparse as sp

    rng = np.random.default_rng(seed)
    xy = rng.random((n_bus, 2))

    tree = _mst_edges(xy)
    existing = {(int(a), int(b)) for a, b in tree}
    cand = _knn_candidates(xy, existing)
    n_extra = max(0, min(n_branch - tree.shape[0], cand.shape[0]))
    pick = np.sort(np.random.default_rng(seed + 1).choice(cand.shape[0], size=n_extra, replace=False)) \
        if n_extra else np.zeros(0, np.int64)
    br = np.concatenate([tree, cand[pick]], axis=0)
    m = br.shape[0]

    r = rng.uniform(0.005, 0.05, size=m)
    x = r * rng.uniform(3.0, 10.0, size=m)
    bsh = rng.uniform(0.0, 0.1, size=m)
    y = 1.0 / (r + 1j * x)

    # pi-model stamps: Y_ii += y + j b/2, Y_ij -= y
    rows = np.concatenate([br[:, 0], br[:, 1], br[:, 0], br[:, 1]])
    cols = np.concatenate([br[:, 0], br[:, 1], br[:, 1], br[:, 0]])
    vals = np.concatenate([y + 0.5j * bsh, y + 0.5j * bsh, -y, -y])
    Y = sp.coo_matrix((vals, (rows, cols)), shape=(n_bus, n_bus)).tocsr()
    Y.sum_duplicates()
    Y.sort_indices()
    indptr = Y.indptr.astype(np.int32)
    indices = Y.indices.astype(np.int32)

    # bus types: slack = best-connected bus (ties: closest to the centre)
    deg = np.diff(indptr)
    slack = int(np.lexsort((np.linalg.norm(xy - 0.5, axis=1), -deg))[0])
    pv = _dominating_pv(indptr, indices, slack, n_pv) if n_pv > 0 else np.zeros(0, np.int64)
    others = np.setdiff1d(np.arange(n_bus), np.r_[pv, [slack]])
    pq = others

    p_load = load_scale * rng.lognormal(mean=np.log(0.3), sigma=0.6, size=n_bus)
    q_load = p_load * rng.uniform(0.1, 0.5, size=n_bus)
    sload = p_load + 1j * q_load
    vm_set = rng.uniform(0.98, 1.05, size=pv.size)

    v0 = np.ones(n_bus, dtype=np.complex128)
    v0[pv] = vm_set

    # Dispatch: each PV unit produces the real power that holds its bus angle at 0
    # in the base case (all PV buses and the slack held at their set voltage).
    sgen = np.zeros(n_bus, dtype=np.complex128)
    if pv.size:
        Vd = _polar_nr(Y, -sload, v0, np.zeros(0, np.int64), pq)
        inj = Vd * np.conj(Y @ Vd)
        sgen[pv] = inj[pv].real + p_load[pv]

    return Grid(
        name=name or f"synthetic{n_bus}",
        n_bus=n_bus,
        indptr=indptr,
        indices=indices,
        data=Y.data.astype(np.complex128),
        pv=pv.astype(np.int32),
        pq=pq.astype(np.int32),
        slack=slack,
        sgen=sgen,
        sload=sload,
        v0=v0,
        seed=seed,
        branches=br,
    )


# The workloads, named by what they are.  Seeds are fixed per grid: 1000 + n_bus.
def grid_118() -> Grid:
    """118 buses, 186 branches, 53 PV, 64 PQ (Jacobian 181 x 181)."""
    return make_grid(118, 186, 53, seed=1118, name="synthetic118")


def grid_2000() -> Grid:
    """2,000 buses, ~3,000 branches, 400 PV, 1,599 PQ (Jacobian 3,598 x 3,598)."""
    return make_grid(2000, 3000, 400, seed=3000, name="synthetic2000")


def grid_10000() -> Grid:
    """10,000 buses, ~15,000 branches, 2,000 PV, 7,999 PQ (Jacobian 17,998 x 17,998)."""
    return make_grid(10000, 15000, 2000, seed=11000, name="synthetic10000")


def grid_500() -> Grid:
    """500 buses, PV fraction 0.2 (one of the four uneven-batch grids)."""
    return make_grid(500, 750, 100, seed=1500, name="synthetic500")


def uneven_grids() -> list[tuple[Grid, int]]:
    """Four grids of 118/500/2,000/10,000 buses with 256/128/96/32 instances, PV fraction 0.2."""
    return [
        (make_grid(118, 186, 23, seed=1118 + 7, name="uneven118"), 256),
        (make_grid(500, 750, 100, seed=1500 + 7, name="uneven500"), 128),
        (make_grid(2000, 3000, 400, seed=3000 + 7, name="uneven2000"), 96),
        (make_grid(10000, 15000, 2000, seed=11000 + 7, name="uneven10000"), 32),
    ]


def two_bus_case() -> dict:
    """The reference's analytic 2-bus case (cuPF/tests/unit/small_cases.cpp:9-31):
    y = 1 - 5j, slack 1+0j, PQ bus solution 0.97 - 0.05j, Sbus chosen so that it is exact."""
    y = 1.0 - 5.0j
    slack_v = 1.0 + 0.0j
    pq_v = 0.97 - 0.05j
    pq_current = y * (pq_v - slack_v)
    pq_sbus = pq_v * np.conjugate(pq_current)
    return {
        "indptr": np.array([0, 2, 4], dtype=np.int32),
        "indices": np.array([0, 1, 0, 1], dtype=np.int32),
        "data": np.array([y, -y, -y, y], dtype=np.complex128),
        "sbus": np.array([0.0 + 0.0j, pq_sbus], dtype=np.complex128),
        "v0": np.array([slack_v, 1.0 + 0.0j], dtype=np.complex128),
        "expected_v": np.array([slack_v, pq_v], dtype=np.complex128),
        "pv": np.array([], dtype=np.int32),
        "pq": np.array([1], dtype=np.int32),
    }
