"""The engine's fast solver (flexible CG + AC K-cycle) in FP64 and mixed
precision. Checked with the oracle: the FP64 true residual |b - A x| / |b|
<= 1e-8 (recomputed on the CPU), and the error against the tight oracle
solution (CG to 1e-13) within 10x the error the reference's own CG leaves
when it stops at the same 1e-8 (the oracle's CG to ResRat 1e-8)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = [(0, dict(n=16)), (0, dict(n=64)), (1, dict(n=40, nb=6, rmin=2.0, rmax=5.0, rc=8.0)),
         (2, dict(index=2, n2d=4, s2=(40, 90))), (2, dict(index=9, n2d=4, s3=(21, 33)))]


def true_relres(oracle, P, x):
    r = oracle.resid(P, x, P.b)
    return float(np.linalg.norm(r) / np.linalg.norm(P.b))


@pytest.mark.parametrize("kind,kw", CASES)
@pytest.mark.parametrize("precision", [0, 1])
def test_engine_reaches_1e8(engine, oracle, kind, kw, precision):
    P = oracle.Problem(kind, 3, **kw)
    x = np.zeros(P.N)
    with engine.Session(*P.dims, P.h) as s:
        s.assemble_pressure(P.rho, P.solid)
        E = engine.Engine(s)
        ok = E.solve(x, P.b.copy(), tol=1e-8, precision=precision)
        r = E.last
    assert ok and r.status == 0
    rel = true_relres(oracle, P, x)
    assert rel <= 1e-8 * 1.0001, rel
    assert abs(rel - r.relres) <= 1e-3 * rel + 1e-13  # roundoff floor of a direct solve
    # the error against the tight solution is bounded by what the reference's
    # own CG leaves at the same tolerance (its answer at ResRat 1e-8): both
    # stop at a residual of 1e-8 |b|, so their errors are A^-1 of residuals of
    # that size; the engine's may differ in direction, not in scale
    xt, _ = oracle.cg(P, res_rat=1e-13, maxit=100000)
    xr, _ = oracle.cg(P, res_rat=1e-8, maxit=100000)
    nt = np.linalg.norm(xt)
    err = np.linalg.norm(x - xt) / nt
    err_ref = np.linalg.norm(xr - xt) / nt
    assert err <= 10.0 * err_ref, (err, err_ref)
    if precision == 1:
        assert r.sweeps >= 2


def test_engine_warm_start(engine, oracle):
    P = oracle.Problem(0, 5, n=24)
    with engine.Session(*P.dims, P.h) as s:
        s.assemble_pressure(P.rho, P.solid)
        E = engine.Engine(s)
        x = np.zeros(P.N)
        E.solve(x, P.b.copy(), precision=1)
        cold = E.last.iterations
        x2 = x.copy()
        E.solve(x2, P.b.copy(), precision=1)
        assert E.last.status in (0, 4) and E.last.iterations <= 1
        x3 = x + 1e-3 * np.random.default_rng(0).standard_normal(P.N) * np.abs(x).max()
        E.solve(x3, P.b.copy(), precision=1)
        assert E.last.converged and E.last.iterations < cold
    assert true_relres(oracle, P, x3) <= 1e-8 * 1.0001


@pytest.mark.parametrize("precision", [0, 1])
def test_engine_nonsymmetric(engine, oracle, precision):
    """A mildly non-symmetric matrix (seven-array form, weak upwind
    convection) converges by the refinement around its symmetric part to the
    FP64 target; a strongly non-symmetric one (stronger convection, where that
    refinement stalls) ends unconverged (DIVERGED, BREAKDOWN or MAXITER) with
    an iterate better than the start."""
    P = oracle.Problem(0, 5, n=16, convect=2e-7)
    with engine.Session(*P.dims, P.h) as s:
        s.upload_matrix(P.A)
        assert not s.symmetric()
        x = np.zeros(P.N)
        E = engine.Engine(s)
        assert E.solve(x, P.b.copy(), tol=1e-8, precision=precision)
    assert true_relres(oracle, P, x) <= 1e-8 * 1.0001
    P = oracle.Problem(0, 5, n=16, convect=2e-5)
    with engine.Session(*P.dims, P.h) as s:
        s.upload_matrix(P.A)
        x = np.zeros(P.N)
        E = engine.Engine(s)
        ok = E.solve(x, P.b.copy(), tol=1e-8, precision=precision)
        r = E.last
    assert not ok and r.status in (engine.DIVERGED, engine.BREAKDOWN, engine.MAXITER)
    assert true_relres(oracle, P, x) == pytest.approx(r.relres, rel=1e-6)
    assert r.relres < 1.0


def test_device_arrays(engine, oracle):
    torch = pytest.importorskip("torch")
    P = oracle.Problem(0, 2, n=20)
    with engine.Session(*P.dims, P.h) as s:
        s.assemble_pressure(torch.from_numpy(P.rho).cuda(), torch.from_numpy(P.solid).cuda())
        xd = torch.zeros(P.N, dtype=torch.float64, device="cuda")
        bd = torch.from_numpy(P.b).cuda()
        engine.Engine(s).solve(xd, bd, precision=1)
        x = xd.cpu().numpy()
    assert true_relres(oracle, P, x) <= 1e-8 * 1.0001


@pytest.mark.parametrize("precision", [0, 1])
def test_refresh_equals_fresh_build(engine, oracle, precision):
    """A re-assembled matrix of the same shape reuses the hierarchy's buffers
    (numeric refresh on the device, the dense coarsest inverse included) and
    gives bit-for-bit the solution of a session built for that matrix."""
    P1 = oracle.Problem(1, 3, n=32, nb=4, rmin=2.0, rmax=4.0, rc=6.0)
    P2 = oracle.Problem(1, 8, n=32, nb=5, rmin=2.0, rmax=5.0, rc=7.0)
    assert P1.dims == P2.dims
    with engine.Session(*P1.dims, P1.h) as s:
        E = engine.Engine(s)
        s.assemble_pressure(P1.rho, P1.solid)
        x1 = np.zeros(P1.N)
        assert E.solve(x1, P1.b.copy(), precision=precision)
        s.assemble_pressure(P2.rho, P2.solid)
        xa = np.zeros(P2.N)
        assert E.solve(xa, P2.b.copy(), precision=precision)
        ita = E.last.iterations
    with engine.Session(*P2.dims, P2.h) as s:
        s.assemble_pressure(P2.rho, P2.solid)
        E = engine.Engine(s)
        xb = np.zeros(P2.N)
        assert E.solve(xb, P2.b.copy(), precision=precision)
        itb = E.last.iterations
    assert ita == itb
    assert np.array_equal(xa, xb)
    assert true_relres(oracle, P2, xa) <= 1e-8 * 1.0001


def test_host_polled_loop_matches_device_loop(oracle):
    """PBG_GRAPH_LOOP=0 replays the one-iteration graph in host-polled
    chunks instead of the device-side WHILE loop: the same iterations and
    the same solution bits."""
    import json
    import os
    import subprocess
    import sys
    code = (
        "import sys, json, hashlib, numpy as np; sys.path[:0] = %r\n"
        "import psiboil_b200 as pb, oracle_py as O\n"
        "P = O.Problem(1, 3, n=48, nb=4, rmin=3.0, rmax=6.0, rc=8.0)\n"
        "s = pb.Session(*P.dims, P.h); s.assemble_pressure(P.rho, P.solid)\n"
        "out = {}\n"
        "for prec in (pb.FP64, pb.MIXED):\n"
        "    x = np.zeros(P.N); E = pb.Engine(s); E.solve(x, P.b.copy(), tol=1e-9, precision=prec)\n"
        "    out[str(prec)] = [E.last.iterations, hashlib.sha256(x.tobytes()).hexdigest()]\n"
        "print(json.dumps(out))\n"
    ) % ([os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
          os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle")],)
    res = {}
    for mode in ("0", "1"):
        env = dict(os.environ, PBG_GRAPH_LOOP=mode)
        r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr[-2000:]
        res[mode] = json.loads(r.stdout.strip().splitlines()[-1])
    assert res["0"] == res["1"]


def test_x0_zero_option(engine, oracle):
    """x0_zero ignores what x holds (it is not uploaded) and gives the bits of
    a solve from an explicit zero guess, for host and device buffers."""
    import torch
    P = oracle.Problem(1, 3, n=32, nb=3, rmin=2.0, rmax=4.0, rc=5.0)
    with engine.Session(*P.dims, P.h) as s:
        s.assemble_pressure(P.rho, P.solid)
        E = engine.Engine(s)
        ref = np.zeros(P.N)
        E.solve(ref, P.b.copy(), tol=1e-9, precision=engine.MIXED)
        x = np.full(P.N, 7.0)
        E.solve(x, P.b.copy(), tol=1e-9, precision=engine.MIXED, x0_zero=True)
        assert np.array_equal(x, ref)
        xd = torch.full((P.N,), -3.0, dtype=torch.float64, device="cuda")
        E.solve(xd, torch.from_numpy(P.b).cuda(), tol=1e-9, precision=engine.MIXED, x0_zero=True)
        torch.cuda.synchronize()
        assert np.array_equal(xd.cpu().numpy(), ref)


def test_large_coarse_level_fp16_inverse(engine, oracle):
    """A 4096-cell coarsest level in the mixed path is applied from the
    row-scaled FP16 copy of its inverse: the solve still reaches the FP64
    target, in no more iterations than with the default 512-cell level."""
    P = oracle.Problem(1, 6, n=128, nb=6, rmin=3.0, rmax=8.0, rc=12.0)
    its = {}
    with engine.Session(*P.dims, P.h) as s:
        s.assemble_pressure(P.rho, P.solid)
        E = engine.Engine(s)
        for cm in (512, 4096):
            x = np.zeros(P.N)
            assert E.solve(x, P.b.copy(), tol=1e-8, precision=engine.MIXED, coarse_max=cm)
            its[cm] = E.last.iterations
            r = np.zeros(P.N)
            s.residual(x, P.b, r)
            assert np.linalg.norm(r) <= 1.0001e-8 * np.linalg.norm(P.b)
    assert its[4096] <= its[512] + 2
