"""Oracle vs the compiled reference run live (only where oracle/_ref was
built, i.e. where the reference sources exist)."""
import numpy as np
import pytest

import oracle_py


pytestmark = pytest.mark.skipif(not oracle_py.harness_available(),
                                reason="reference harness not built here")


@pytest.mark.parametrize("kind,kw", [(0, dict(n=20)), (1, dict(n=28, nb=4, rmin=2.0, rmax=5.0, rc=6.0)),
                                     (2, dict(index=5, n2d=8, s2=(30, 50)))])
def test_live_cg_and_ac(oracle, kind, kw):
    P = oracle.Problem(kind, 11, **kw)
    meta, arr = oracle.run_reference(P, "cg")
    x, st = oracle.cg(P)
    assert st["printed"] == int(meta["iterations"])
    assert np.array_equal(x, arr["x"])
    meta, arr = oracle.run_reference(P, "ac")
    x, st = oracle.AC(P).cycle()
    assert st["cycles"] == int(meta["cycles"])
    assert np.array_equal(x, arr["x"])


@pytest.mark.parametrize("prec", ["ic0", "ic2", "ic3"])
@pytest.mark.parametrize("kind,kw", [(0, dict(n=10)), (1, dict(n=12, nb=2, rmin=2.0, rmax=3.0, rc=3.0)),
                                     (2, dict(index=1, n2d=2, s2=(10, 14), s3=(6, 8))),
                                     (2, dict(index=0, n2d=2, s2=(10, 14), s3=(6, 8)))])
def test_oracle_ic_cg_equals_reference(oracle, prec, kind, kw):
    """CG with Prec::ic0/ic2/ic3: the oracle's factor and sweeps give the
    compiled reference's iterations and solution bit for bit (on 2-D grids
    the reference's IC3 factor breaks down into NaN; the oracle does the
    same)."""
    P = oracle.Problem(kind, 5, **kw)
    meta, arr = oracle.run_reference(P, solver="cg", resrat=1e-8, prec=prec)
    x, st = oracle.cg(P, prec=prec, res_rat=1e-8, res_tol=1e-15)
    assert st["printed"] == int(meta["iterations"])
    assert np.array_equal(x, arr["x"], equal_nan=True)


@pytest.mark.parametrize("solver", ["jacobi", "gs"])
@pytest.mark.parametrize("resrat,maxit", [(0.5, 300), (1e-3, 7), (1e-2, 1), (0.9, 50)])
@pytest.mark.parametrize("kind,kw", [(1, dict(n=12, nb=2, rmin=2.0, rmax=3.0, rc=3.0)),
                                     (2, dict(index=3, n2d=2, s2=(10, 14), s3=(6, 8)))])
def test_oracle_stationary_equals_reference(oracle, solver, resrat, maxit, kind, kw):
    """Jacobi::solve and GaussSeidel::solve: early stops, caps of one and a few
    sweeps, 2-D and bodies; the oracle (with the reference's stored ci) gives
    the compiled reference's sweep count, convergence flag and iterate."""
    P = oracle.Problem(kind, 9, **kw)
    meta, arr = oracle.run_reference(P, solver=solver, resrat=resrat, maxit=maxit)
    P.ci = arr["ci"].copy()
    x, st = oracle.cg(P, solver=solver, res_rat=resrat, maxit=maxit, res_tol=1e-18)  # ResTol(atto)
    assert st["printed"] == int(meta["iterations"])
    assert bool(st["converged"]) == bool(meta["converged"])
    assert np.array_equal(x, arr["x"])
