"""Batched solves (pbg_batch_*): uneven 2-D / 3-D problems solved together.

Checked with the oracle: every problem reaches the FP64 true residual
|b - A x| / |b| <= 1e-8 (recomputed on the CPU from the oracle's own
assembly), the solution agrees with the single-problem engine, a problem's
result is bit-for-bit the same alone and in any mix (slot, neighbours, entry
time), and finished problems free their slots for waiting ones."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-8


def relres(oracle, P, x):
    r = oracle.resid(P, x, P.b)
    return float(np.linalg.norm(r) / np.linalg.norm(P.b))


def uneven(oracle, n, seed=11, s2=(20, 90), s3=(9, 30)):
    return [oracle.Problem(oracle.KIND_BATCH, seed, index=i, n2d=n // 2, s2=s2, s3=s3) for i in range(n)]


def add_all(B, probs):
    return [B.add(P.dims, P.h, rho=P.rho, solid=P.solid, b=P.b) for P in probs]


@pytest.mark.parametrize("precision", [0, 1])
def test_batch_reaches_tolerance_and_matches_engine(engine, oracle, precision):
    probs = uneven(oracle, 10)
    assert any(P.dims[2] == 1 for P in probs) and any(P.dims[2] > 1 for P in probs)
    with engine.Batch(precision=precision, slots=16) as B:
        ids = add_all(B, probs)
        res = B.solve(ids, tol=TOL)
        xs = [B.get_x(i) for i in ids]
    for P, r, x in zip(probs, res, xs):
        assert r.converged and r.status == 0, (P.dims, r.as_dict())
        rel = relres(oracle, P, x)
        assert rel <= TOL * 1.0001, (P.dims, rel)
        assert abs(rel - r.relres) <= 1e-3 * rel + 1e-15
        with engine.Session(*P.dims, P.h) as s:
            s.assemble_pressure(P.rho, P.solid)
            xe = np.zeros(P.N)
            assert engine.Engine(s).solve(xe, P.b.copy(), tol=TOL, precision=precision)
        assert np.linalg.norm(x - xe) / np.linalg.norm(xe) < 1e-4


@pytest.mark.parametrize("precision", [0, 1])
def test_alone_equals_in_mix(engine, oracle, precision):
    """The same problem solved alone, and among others in a different slot
    that it enters while others are already running, gives the same bits."""
    probs = uneven(oracle, 9, seed=5)
    target = probs[4]
    with engine.Batch(precision=precision, slots=1) as B:
        i = B.add(target.dims, target.h, rho=target.rho, solid=target.solid, b=target.b)
        (r_alone,) = B.solve([i], tol=TOL)
        x_alone = B.get_x(i)
    # three slots for nine problems: the target waits for a free slot, then
    # runs next to problems that are mid-solve
    with engine.Batch(precision=precision, slots=3) as B:
        ids = add_all(B, probs)
        res = B.solve(ids, tol=TOL)
        x_mix = B.get_x(ids[4])
    r_mix = res[4]
    assert r_alone.converged and r_mix.converged
    assert (r_alone.iterations, r_alone.sweeps) == (r_mix.iterations, r_mix.sweeps)
    assert r_alone.relres == r_mix.relres
    assert np.array_equal(x_alone, x_mix)
    for P, r, i in zip(probs, res, ids):
        assert r.converged, (P.dims, r.as_dict())


def test_warm_start_and_rhs_update(engine, oracle):
    probs = uneven(oracle, 4, seed=3)
    with engine.Batch(precision=1, slots=4) as B:
        ids = add_all(B, probs)
        cold = B.solve(ids, tol=TOL)
        again = B.solve(ids, tol=TOL)  # from the stored solutions
        for c, a in zip(cold, again):
            assert a.converged and a.iterations <= 1 < c.iterations
        # a new right-hand side on one problem, warm start from the old solution
        P = probs[1]
        b2 = P.b + 0.01 * np.random.default_rng(0).standard_normal(P.N) * np.abs(P.b).max()
        b2[P.solid.astype(bool)] = 0.0
        B.set_rhs(ids[1], b2)
        (r,) = B.solve([ids[1]], tol=TOL)
        x = B.get_x(ids[1])
    assert r.converged and r.iterations < cold[1].iterations
    rr = oracle.resid(P, x, b2)
    assert np.linalg.norm(rr) / np.linalg.norm(b2) <= TOL * 1.0001


def test_matrix_update_refreshes_hierarchy(engine, oracle):
    """New fields on a problem (a moved bubble) rebuild its hierarchy: the
    result equals a fresh problem's, bit for bit."""
    P1 = oracle.Problem(oracle.KIND_CYL, 3, n=24, nb=3, rmin=2.0, rmax=4.0, rc=5.0)
    P2 = oracle.Problem(oracle.KIND_CYL, 9, n=24, nb=4, rmin=2.0, rmax=5.0, rc=6.0)
    with engine.Batch(precision=1, slots=2) as B:
        i = B.add(P1.dims, P1.h, rho=P1.rho, solid=P1.solid, b=P1.b)
        B.solve([i], tol=TOL)
        B.set_fields(i, P2.rho, P2.solid)
        B.set_rhs(i, P2.b)
        B.set_x(i, None)
        (ra,) = B.solve([i], tol=TOL)
        xa = B.get_x(i)
        j = B.add(P2.dims, P2.h, rho=P2.rho, solid=P2.solid, b=P2.b)
        (rb,) = B.solve([j], tol=TOL)
        xb = B.get_x(j)
    assert ra.iterations == rb.iterations and np.array_equal(xa, xb)
    assert relres(oracle, P2, xa) <= TOL * 1.0001


def test_slots_are_reused(engine, oracle):
    probs = uneven(oracle, 7, seed=21)
    with engine.Batch(precision=1, slots=2) as B:
        ids = add_all(B, probs)
        res = B.solve(ids, tol=TOL)
        for P, i, r in zip(probs, ids, res):
            assert r.converged
            assert relres(oracle, P, B.get_x(i)) <= TOL * 1.0001


def test_autotune_and_cache(engine, oracle, tmp_path):
    probs = uneven(oracle, 6, seed=8)
    cache = str(tmp_path / "tune.json")
    with engine.Batch(precision=1, slots=8) as B:
        ids = add_all(B, probs)
        best = B.autotune(ids, cache=cache)
        again = B.autotune(ids, cache=cache)  # read back from the cache
        assert best.as_dict() == again.as_dict()
        res = B.solve(ids, tol=TOL)
        assert all(r.converged for r in res)
    import json
    d = json.load(open(cache))
    assert len(d) == 1 and set(next(iter(d.values()))) >= {"threads", "tile_cells", "grid", "kc_max", "tail_cells"}


def test_bad_inputs_fail_loudly(engine, oracle):
    with engine.Batch(precision=1, slots=2) as B:
        with pytest.raises(engine.PbgError):
            B.add((4, 4, 4), 0.25)  # 64 cells: no coarse level
        with pytest.raises(engine.PbgError):
            B.solve([7])  # unknown id
        P = uneven(oracle, 2)[0]
        i = B.add(P.dims, P.h)  # no matrix yet
        with pytest.raises(engine.PbgError):
            B.solve([i])
