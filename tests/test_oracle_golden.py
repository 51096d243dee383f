"""The CPU oracle (oracle/pf_oracle.c) pinned against the reference's own outputs.

Fixtures in tests/golden/ were produced by the reference's CPU NewtonSolver and
solve_adjoint (tests/golden/make_golden.py); these tests run on any CPU.
"""
import numpy as np
import pytest

from cupf import grids as G

GOLD = __import__("pathlib").Path(__file__).resolve().parent / "golden"


class _Case:
    def __init__(self, c):
        self.indptr, self.indices, self.data = c["indptr"], c["indices"], c["data"]
        self.pv, self.pq, self.n_bus = c["pv"], c["pq"], 2
        self.dim_f = self.pv.size + 2 * self.pq.size


def test_two_bus_analytic(oracle):
    """cuPF/tests/unit/test_minimal_solver.cpp:61-91: converges, |V - V*| <= 1e-8."""
    c = G.two_bus_case()
    r = oracle.solve(_Case(c), c["sbus"], c["v0"], tol=1e-10, max_iter=20)
    assert r["converged"]
    assert np.abs(r["V"] - c["expected_v"]).max() <= 1e-8
    gold = np.load(GOLD / "two_bus.npz")
    # the reference ran at 1e-8 / 20; compare the oracle on the same stopping rule
    r8 = oracle.solve(_Case(c), c["sbus"], c["v0"], tol=1e-8, max_iter=20)
    assert r8["iterations"] == int(gold["iterations"])
    assert np.array_equal(r8["V"], gold["V"])


@pytest.mark.parametrize("name", ["118", "2000"])
@pytest.mark.parametrize("tag,tol,max_iter", [("t8", 1e-8, 10), ("t12", 1e-12, 30)])
def test_nr_matches_reference(oracle, name, tag, tol, max_iter):
    g = {"118": G.grid_118, "2000": G.grid_2000}[name]()
    gold = np.load(GOLD / f"nr_{name}.npz")
    for b in range(gold["sbus"].shape[0]):
        r = oracle.solve(g, gold["sbus"][b], gold["v0"][b], tol=tol, max_iter=max_iter)
        assert r["iterations"] == int(gold[f"it_{tag}"][b])
        assert r["final_mismatch"] == pytest.approx(float(gold[f"fm_{tag}"][b]), rel=1e-6, abs=1e-15)
        assert np.abs(r["V"] - gold[f"V_{tag}"][b]).max() <= 1e-13


@pytest.mark.parametrize("name", ["118", "2000"])
def test_adjoint_matches_reference(oracle, name):
    g = {"118": G.grid_118, "2000": G.grid_2000}[name]()
    gold = np.load(GOLD / f"adjoint_{name}.npz")
    a = oracle.adjoint(g, gold["V"], gold["grad_va"], gold["grad_vm"])
    for k, gk in (("lambda", "lam"), ("grad_p", "grad_p"), ("grad_q", "grad_q")):
        ref = gold[gk]
        assert np.abs(a[k] - ref).max() <= 1e-9 * max(1.0, np.abs(ref).max()), k
    assert a["residual"] <= 1e-10


def test_adjoint_matches_central_differences(oracle):
    """dL/dP_load and dL/dQ_load by central differences (h = 1e-6) on the 118-bus grid."""
    g = G.grid_118()
    S = g.scenarios(1, seed=5)[0]
    rng = np.random.default_rng(0)
    ga, gm = rng.standard_normal(g.n_bus), rng.standard_normal(g.n_bus)

    def loss(sbus):
        r = oracle.solve(g, sbus, g.v0, tol=1e-13, max_iter=40)
        assert r["converged"]
        return float(ga @ np.angle(r["V"]) + gm @ np.abs(r["V"]))

    V = oracle.solve(g, S, g.v0, tol=1e-13, max_iter=40)["V"]
    a = oracle.adjoint(g, V, ga, gm)
    h = 1e-6
    for bus in list(g.pq[:3]) + list(g.pv[:2]):
        for kind, unit in (("grad_p", 1.0), ("grad_q", 1.0j)):
            if kind == "grad_q" and bus in set(g.pv.tolist()):
                continue
            # load P/Q enter Sbus with a minus sign: Sbus = Sgen - Sload
            fd = (loss(S - h * unit * _e(g.n_bus, bus)) - loss(S + h * unit * _e(g.n_bus, bus))) / (2 * h)
            an = a[kind][bus]
            assert abs(fd - an) <= 1e-6 * max(1.0, abs(an)) + 1e-7, (kind, bus, fd, an)


def _e(n, i):
    v = np.zeros(n, dtype=np.complex128)
    v[i] = 1.0
    return v


def test_jacobian_analysis_matches_reference(oracle):
    g = G.grid_118()
    gold = np.load(GOLD / "jacobian_118.npz")
    ja = oracle.jacobian_analysis(g)
    for k in gold.files:
        assert np.array_equal(ja[k], gold[k]), k


def test_oracle_solve_many_threads_agree(oracle):
    g = G.grid_118()
    S = g.scenarios(6, seed=11)
    V0 = g.flat_start(6)
    one = oracle.solve_many(g, S, V0, 1e-8, 10, 1)
    many = oracle.solve_many(g, S, V0, 1e-8, 10, 3)
    assert np.array_equal(one["V"], many["V"])
    assert np.array_equal(one["iterations"], many["iterations"])


@pytest.mark.skipif(not __import__("oracle.oracle", fromlist=["LIB_REF"]).LIB_REF.exists(),
                    reason="oracle/_ref not built (reference sources absent)")
@pytest.mark.parametrize("name", ["500", "10000"])
def test_nr_matches_the_reference_live(oracle, name):
    """The oracle's C port against the reference's own CPU NewtonSolver (built
    in oracle/_ref) on grids the golden fixtures do not hold: the same
    iteration counts, final mismatches to rounding, V to 1e-10."""
    from oracle.oracle import Reference

    g = {"500": G.grid_500, "10000": G.grid_10000}[name]()
    S, V0 = g.scenarios(2, seed=515), g.flat_start(2)
    ref = Reference()
    for b in range(2):
        r = ref.solve(g, S[b], V0[b], 1e-8, 10)
        o = oracle.solve(g, S[b], V0[b], tol=1e-8, max_iter=10)
        assert int(o["iterations"]) == int(r["iterations"])
        assert o["final_mismatch"] <= 1e-8 and r["final_mismatch"] <= 1e-8
        assert np.abs(o["V"] - r["V"]).max() <= 1e-10


@pytest.mark.skipif(not __import__("oracle.oracle", fromlist=["LIB_REF"]).LIB_REF.exists(),
                    reason="oracle/_ref not built (reference sources absent)")
@pytest.mark.parametrize("name", ["500", "10000"])
def test_adjoint_matches_the_reference_live(oracle, name):
    """The oracle's adjoint against the reference's own CPU adjoint pipeline
    (newton_solver_adjoint.cpp:33-153, built in oracle/_ref) on grids the
    golden fixtures do not hold: lambda and both load gradients to 1e-9
    relative."""
    from oracle.oracle import Reference

    g = {"500": G.grid_500, "10000": G.grid_10000}[name]()
    S, V0 = g.scenarios(1, seed=77)[0], g.flat_start(1)[0]
    rng = np.random.default_rng(5)
    ga, gm = rng.standard_normal(g.n_bus), rng.standard_normal(g.n_bus)
    r = Reference().adjoint(g, S, V0, ga, gm, 1e-12, 30)
    a = oracle.adjoint(g, r["V"], ga, gm)
    for k, rk in (("lambda", "lambda"), ("grad_p", "grad_p"), ("grad_q", "grad_q")):
        assert np.abs(a[k] - r[rk]).max() <= 1e-9 * max(1.0, np.abs(r[rk]).max()), k
