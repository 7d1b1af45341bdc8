"""Jacobi and Gauss-Seidel on the GPU (Src/Solver/Linear/Iterative) against
the compiled reference's own results (the golden fixtures).

Gauss-Seidel's lexicographic sweep runs as one launch per hyperplane
i + j + k, and every cell gets the values the sequential sweep gives it. The
sweeps do not read the global sums, so the iterate after a given number of
sweeps equals the reference's bit for bit in both sum modes; the sum order
only decides where a run stops. With exact sums the iteration counts are the
reference's as well."""
import numpy as np
import pytest

from golden_util import NAMES, bc_of, load, problem_of

pytestmark = pytest.mark.gpu

RUNS = [(n, s) for n in NAMES for s in ("jacobi", "gs") if s + "_x" in load(n)]


def _session(engine, g, P, ci=True):
    s = engine.Session(*P.dims, P.h, bc=bc_of(P))
    s.upload_matrix({k: g["A_" + k] for k in "cwesnbt"})
    if ci:
        s.upload_ci(g["ci"])
    return s


def _solver(engine, name, s, exact):
    cls = engine.Jacobi if name == "jacobi" else engine.GaussSeidel
    return cls(s, exact_sums=exact)


@pytest.mark.parametrize("name,solver", RUNS)
def test_stationary_bit_exact(engine, oracle, name, solver):
    g = load(name)
    P = problem_of(g, oracle)
    rr, mi = float(g[solver + "_resrat"]), int(g[solver + "_maxit"])
    with _session(engine, g, P) as s:
        for exact in (True, False):
            x = np.zeros(P.N)
            kr = _solver(engine, solver, s, exact)
            ok = kr.solve(x, g["b"].copy(), 1, mi, None, rr, 1e-18)
            printed = kr.last.iterations + (1 if kr.last.status == engine.MAXITER else 0)
            if exact or printed == int(g[solver + "_iterations"]):
                assert printed == int(g[solver + "_iterations"])
                assert ok == bool(g[solver + "_converged"])
                assert np.array_equal(x, g[solver + "_x"])
            else:  # tree sums stopped one sweep apart: close, not equal
                assert abs(printed - int(g[solver + "_iterations"])) <= 1


@pytest.mark.parametrize("solver", ["jacobi", "gs"])
def test_stationary_matches_oracle_history(engine, oracle, solver):
    """The residual after every sweep (exact sums) equals the oracle's."""
    g = load("odd15")
    P = problem_of(g, oracle)
    P.ci = g["ci"].copy()
    xo, st = oracle.cg(P, solver=solver, res_rat=1e-2, maxit=2000, res_tol=1e-18, hist=True)
    with _session(engine, g, P) as s:
        x = np.zeros(P.N)
        kr = _solver(engine, solver, s, True)
        kr.solve(x, P.b.copy(), 1, 2000, None, 1e-2, 1e-18)
        h = s.history()
        n = min(len(h), len(st["hist"]))
        assert n > 50
        assert np.array_equal(h[:n], st["hist"][:n])
        assert kr.last.res0 == st["res0"]
        assert np.array_equal(x, xo)


def test_ci_upload_and_default(engine, oracle):
    """Without an uploaded ci the solvers divide by 1/c; a new matrix drops
    the uploaded ci. On the cylinder fixture the body's cells have ci != 1/c
    (ci is formed before c *= 1e-12), but their right-hand side is zero, so
    both give the same iterate there."""
    g = load("cyl24")
    P = problem_of(g, oracle)
    solid = P.solid.astype(bool)
    assert solid.any()
    assert not np.array_equal(g["ci"][solid], 1.0 / g["A_c"][solid])
    res = []
    for ci in (True, False):
        with _session(engine, g, P, ci=ci) as s:
            x = np.zeros(P.N)
            engine.GaussSeidel(s, exact_sums=True).solve(x, g["b"].copy(), 1, 50, None, 1e-2, 1e-18)
            res.append(x)
    assert np.array_equal(res[0], res[1])
    # an uploaded ci is dropped when the matrix changes: a scaled ci, then a re-upload
    with _session(engine, g, P, ci=False) as s:
        s.upload_ci(g["ci"] * 0.5)
        xa = np.zeros(P.N)
        engine.Jacobi(s, exact_sums=True).solve(xa, g["b"].copy(), 1, 5, None, 1e-2, 1e-18)
        s.upload_matrix({k: g["A_" + k] for k in "cwesnbt"})
        xb = np.zeros(P.N)
        engine.Jacobi(s, exact_sums=True).solve(xb, g["b"].copy(), 1, 5, None, 1e-2, 1e-18)
    assert not np.array_equal(xa, xb)


def test_stationary_stale_window(engine, oracle):
    """Gauss-Seidel's stale window (gaussseidel.cpp:85-105) ends a run whose
    residual stops falling: the same sweep count as the oracle's."""
    g = load("flat2d")
    P = problem_of(g, oracle)
    P.ci = g["ci"].copy()
    xo, st = oracle.cg(P, solver="gs", res_rat=1e-12, maxit=3000, res_tol=1e-18, stalecount=3)
    with _session(engine, g, P) as s:
        x = np.zeros(P.N)
        kr = engine.GaussSeidel(s, exact_sums=True)
        kr.solve(x, P.b.copy(), 1, 3000, None, 1e-12, 1e-18, 1.0, 3)
        assert kr.last.iterations == st["iterations"]
        assert kr.last.status == (engine.STALE if st["status"] == 2 else engine.MAXITER)
        assert np.array_equal(x, xo)
