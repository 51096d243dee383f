"""Seeded synthetic grids: sizes, determinism and solvability from flat start."""
import numpy as np
import pytest

from cupf import grids as G


@pytest.mark.parametrize("mk,n,n_pv,dim", [(G.grid_118, 118, 53, 181), (G.grid_2000, 2000, 400, 3598),
                                           (G.grid_10000, 10000, 2000, 17998)])
def test_grid_sizes(mk, n, n_pv, dim):
    g = mk()
    assert g.n_bus == n and g.pv.size == n_pv and g.dim_f == dim
    assert g.pq.size == n - 1 - n_pv
    assert np.intersect1d(g.pv, g.pq).size == 0 and g.slack not in set(g.pv) | set(g.pq)
    assert g.indptr.size == n + 1 and g.indices.size == g.data.size
    # Ybus is structurally symmetric with a full diagonal
    rows = np.repeat(np.arange(n), np.diff(g.indptr))
    pairs = set(zip(rows.tolist(), g.indices.tolist()))
    assert all((c, r) in pairs for r, c in pairs)
    assert all((i, i) in pairs for i in range(n))


def test_grid_is_deterministic():
    a, b = G.grid_118(), G.grid_118()
    assert np.array_equal(a.data, b.data) and np.array_equal(a.pv, b.pv)
    assert np.array_equal(a.scenarios(4, seed=3), b.scenarios(4, seed=3))
    assert not np.array_equal(a.scenarios(4, seed=3), a.scenarios(4, seed=4))


def test_scenarios_scale_loads_only():
    g = G.grid_118()
    S = g.scenarios(64, seed=1)
    gen = g.sgen
    load = gen[None, :] - S
    base = g.sload
    m = np.abs(base) > 0
    ratio = (load[:, m] / base[None, m]).real
    assert ratio.min() >= 0.8 - 1e-12 and ratio.max() <= 1.2 + 1e-12


def test_flat_start_converges_on_oracle(oracle):
    g = G.grid_2000()
    S = g.scenarios(3, seed=2)
    for b in range(3):
        r = oracle.solve(g, S[b], g.v0, tol=1e-8, max_iter=10)
        assert r["converged"] and r["iterations"] <= 8


def test_uneven_batch_composition():
    inst = G.uneven_grids()
    assert [(g.n_bus, b) for g, b in inst] == [(118, 256), (500, 128), (2000, 96), (10000, 32)]
    assert sum(b for _, b in inst) == 512
