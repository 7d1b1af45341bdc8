"""Reference-parity path on the GPU, checked against the oracle and the
reference's golden outputs.

Tolerances: bit-exact for the assembled matrix, SpMV, residual and AC
coarse operators (same per-element operation order). Solvers run in two
reduction modes:
  exact_sums=True  every global sum in the reference's sequential order:
                   CG, BiCGS and AC solutions, iteration / cycle counts and
                   residual histories bit-for-bit equal to the reference;
  exact_sums=False deterministic tree sums (the fast default): CG
                   solutions within 1e-10 relative and counts within 2; AC
                   within 1e-8 (its 20 cycles run thousands of CG steps);
                   BiCGStab's iterates depend on the rounding of its dot
                   products far more (an emulation of the tree order on the
                   CPU moves them by 6e-8..2e-7), so BiCGS is held to 1e-6
                   relative and counts within 6 in that mode.
"""
import numpy as np
import pytest

from golden_util import ACX_RUNS, NAMES, bc_of, load, problem_of

pytestmark = pytest.mark.gpu
RTOL_X = 1e-10


def relerr(x, ref):
    return float(np.abs(x - ref).max() / max(np.abs(ref).max(), 1e-300))


def session_for(engine, P, assemble=True):
    """A session holding P's matrix: assembled on the device, or uploaded
    (always uploaded for the convected fixtures, which the on-device
    pressure assembly does not make)."""
    s = engine.Session(*P.dims, P.h, bc=bc_of(P))
    if assemble and not P.convect and not P.periodic:
        s.assemble_pressure(P.rho, P.solid)
    else:
        s.upload_matrix(P.A)
        s.upload_active((1 - P.solid).astype(np.int32))
    return s


@pytest.mark.parametrize("name", NAMES)
def test_assembly_bit_exact(engine, oracle, name):
    P = problem_of(load(name), oracle)
    if P.convect:
        pytest.skip("the convected fixture is uploaded, not assembled")
    if P.periodic:
        with engine.Session(*P.dims, P.h, bc=bc_of(P)) as s:
            with pytest.raises(engine.PbgError) as e:
                s.assemble_pressure(P.rho, P.solid)
            assert e.value.code == engine.ERR_UNSUPPORTED
        return
    with session_for(engine, P) as s:
        assert s.symmetric()
        M = s.download_matrix()
    for k in "cwesnbt":
        assert np.array_equal(M[k], P.A[k]), k


def test_upload_reference_layout(engine, oracle):
    """The reference's BW=3 Scalar blocks go in unchanged (strided upload)."""
    P = problem_of(load("cyl24"), oracle)
    nx, ny, nz = P.dims
    B = 3
    si, sj = (ny + 2 * B) * (nz + 2 * B), nz + 2 * B
    off = B * (si + sj + 1)
    pad = {}
    for k in "cwesnbt":
        a = np.full((nx + 2 * B) * si, np.nan)
        v = a.reshape(nx + 2 * B, ny + 2 * B, nz + 2 * B)
        v[B:B + nx, B:B + ny, B:B + nz] = P.A[k].reshape(nx, ny, nz)
        pad[k] = a
    with engine.Session(*P.dims, P.h) as s:
        s.upload_matrix(pad, strides=(si, sj, 1), offset=off)
        assert s.symmetric()
        M = s.download_matrix()
        for k in "cwesnbt":
            assert np.array_equal(M[k], P.A[k])
        # strided solve on reference-layout x and b
        bpad = np.zeros_like(pad["c"])
        bpad.reshape(nx + 2 * B, ny + 2 * B, nz + 2 * B)[B:B + nx, B:B + ny, B:B + nz] = P.b.reshape(nx, ny, nz)
        xpad = np.zeros_like(bpad)
        s.upload_active((1 - P.solid).astype(np.int32))
        p = engine.default_params(engine.SOLVER_CG)
        p.max_iter, p.res_rat, p.res_tol = 20000, 1e-8, 1e-18
        r = s.solve(xpad, bpad, p, strides=(si, sj, 1), offset=off)
    x = xpad.reshape(nx + 2 * B, ny + 2 * B, nz + 2 * B)[B:B + nx, B:B + ny, B:B + nz].ravel()
    g = load("cyl24")
    assert relerr(x, g["cg_x"]) <= RTOL_X
    assert abs(r.iterations - int(g["cg_iterations"])) <= 2


@pytest.mark.parametrize("name", NAMES)
def test_spmv_and_residual_bit_exact(engine, oracle, name):
    P = problem_of(load(name), oracle)
    rng = np.random.default_rng(3)
    x = rng.standard_normal(P.N)
    for assemble in (True, False):
        with session_for(engine, P, assemble) as s:
            y = s.spmv(x, np.zeros(P.N))
            r = s.residual(x, P.b, np.zeros(P.N))
        assert np.array_equal(y, oracle.spmv(P, x))
        assert np.array_equal(r, oracle.resid(P, x, P.b))


def test_dots(engine, oracle):
    P = problem_of(load("single16"), oracle)
    rng = np.random.default_rng(4)
    x, y = rng.standard_normal(P.N), rng.standard_normal(P.N)
    with session_for(engine, P) as s:
        d, dv = s.dot(x, y)
    assert abs(d - oracle.dot(x, y)) <= 1e-12 * np.abs(x * y).sum()
    ref = oracle.dot_voldiv_avg(x, y, P.dV)
    assert abs(dv - ref) <= 1e-12 * abs(ref) + 1e-300


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("solver", ["cg", "bicgs"])
@pytest.mark.parametrize("exact", [True, False])
def test_krylov_parity(engine, oracle, name, solver, exact):
    g = load(name)
    if solver + "_x" not in g:
        pytest.skip("no golden run")
    P = problem_of(g, oracle)
    x = np.zeros(P.N)
    with session_for(engine, P) as s:
        K = (engine.CG if solver == "cg" else engine.BiCGS)(s, exact_sums=exact)
        ok = K.solve(x, P.b.copy(), min_iter=1, max_iter=20000, res_rat=1e-8, res_tol=1e-18)
        it = K.last.iterations
    assert ok == bool(g[solver + "_converged"])
    if exact:
        assert it == int(g[solver + "_iterations"])
        assert np.array_equal(x, g[solver + "_x"])
    elif solver == "cg":
        assert abs(it - int(g[solver + "_iterations"])) <= 2
        assert relerr(x, g[solver + "_x"]) <= RTOL_X
    else:
        assert abs(it - int(g[solver + "_iterations"])) <= 6
        assert relerr(x, g[solver + "_x"]) <= 1e-6


AC_RUNS = {"ac": dict(loop=1), "ac_w": dict(loop=4), "ac_f": dict(loop=2),
           "ac_noguard": dict(loop=1, guard=False, max_cyc=6)}


@pytest.mark.parametrize("name,run", [(n, r) for n in NAMES for r in AC_RUNS if r + "_x" in load(n)])
@pytest.mark.parametrize("exact", [True, False])
def test_ac_parity(engine, oracle, name, run, exact):
    g = load(name)
    P = problem_of(g, oracle)
    cfg = AC_RUNS[run]
    x = np.zeros(P.N)
    with session_for(engine, P) as s:
        ac = engine.AC(s, exact_sums=exact)
        ac.stop_if_diverging(cfg.get("guard", True))
        ac.max_cycles(cfg.get("max_cyc", 20))
        ok, ncyc = ac.cycle(x, P.b.copy(), loop=cfg["loop"], factor=1e-8)
        hist = s.history()
    assert ok == bool(g[run + "_converged"])
    if exact:
        assert ncyc == int(g[run + "_cycles"])
        assert np.array_equal(x, g[run + "_x"])
        # the reference prints residuals computed with per-cell volumes
        # (exact on binary-fraction spacings)
        np.testing.assert_allclose(hist, g[run + "_hist"], rtol=1e-13)
    else:
        # tree-ordered sums: the difference grows with the number of CG
        # smoothing steps (20 cycles x ~240 steps here reach ~1e-9)
        assert abs(ncyc - int(g[run + "_cycles"])) <= 2
        n = min(len(hist), len(g[run + "_hist"]))
        h0 = float(g[run + "_hist"][0])
        np.testing.assert_allclose(hist[:n], g[run + "_hist"][:n], rtol=1e-8, atol=1e-12 * h0)
        assert relerr(x, g[run + "_x"]) <= 1e-8, relerr(x, g[run + "_x"])


ACSM_RUNS = [(n, k) for n in NAMES for k in load(n) if k.startswith("acsm_") and k.endswith("_x")]


@pytest.mark.parametrize("name,key", ACSM_RUNS)
def test_ac_with_other_smoothers(engine, oracle, name, key):
    """AC whose levels are smoothed by the Centered object's own solver:
    Gauss-Seidel, Jacobi, BiCGS, CGS or IC0-preconditioned CG instead of CG
    (ref_harness --acsm, --prec). With exact sums the cycles, the residual
    history and the iterate are the compiled reference's."""
    run = key[:-2]
    g = load(name)
    P = problem_of(g, oracle)
    x = np.zeros(P.N)
    sm, _, pr = run.split("_")[1].partition("-")
    with session_for(engine, P) as s:
        s.upload_ci(g["ci"])
        ac = engine.AC(s, exact_sums=True, smoother=sm, prec=pr or "di")
        ok, ncyc = ac.cycle(x, P.b.copy(), loop=engine.CYCLE_V, factor=1e-8)
        hist = s.history()
    assert ok == bool(g[run + "_converged"])
    assert ncyc == int(g[run + "_cycles"])
    np.testing.assert_allclose(hist, g[run + "_hist"], rtol=1e-13)
    assert np.array_equal(x, g[run + "_x"])


@pytest.mark.parametrize("run", ["acsm_gs", "acsm_cg-ic0"])
def test_ac_smoother_without_uploaded_ci(engine, oracle, run):
    """Without an uploaded ci the level-0 smoother takes 1/c for the
    reference's ci; on a fixture whose ci is exactly 1/c (no solid cells)
    the run is the reference's bit for bit."""
    g = load("single12")
    assert np.array_equal(g["ci"], 1.0 / g["A_c"])
    P = problem_of(g, oracle)
    x = np.zeros(P.N)
    sm, _, pr = run.split("_")[1].partition("-")
    with session_for(engine, P) as s:
        ac = engine.AC(s, exact_sums=True, smoother=sm, prec=pr or "di")
        ok, ncyc = ac.cycle(x, P.b.copy(), loop=engine.CYCLE_V, factor=1e-8)
    assert ok == bool(g[run + "_converged"])
    assert ncyc == int(g[run + "_cycles"])
    assert np.array_equal(x, g[run + "_x"])


@pytest.mark.parametrize("name", ["single16", "cyl24", "odd15", "flat2d"])
def test_ac_hierarchy_and_coarse_operators(engine, oracle, name):
    P = problem_of(load(name), oracle)
    ac = oracle.AC(P)
    with session_for(engine, P) as s:
        lv = s.levels(0)
        assert lv == [ac.level_dims(l) for l in range(ac.nlevels)]
        for l in range(1, len(lv)):
            M = s.ac_level_matrix(l)
            R = ac.level_matrix(l)
            for k in "cwesnbt":
                assert np.array_equal(M[k], R[k]), (l, k)


@pytest.mark.slow
def test_config0_64_cg_and_ac(engine, oracle):
    """The 64^3 one-bubble case: CG (566 its in the reference) and AC V-cycles."""
    P = oracle.Problem(oracle.KIND_SINGLE, 1, n=64)
    xo, st = oracle.cg(P)
    xr, sr = oracle.AC(P).cycle(factor=1e-8)
    with session_for(engine, P) as s:
        for exact in (False, True):
            x = np.zeros(P.N)
            K = engine.CG(s, exact_sums=exact)
            K.solve(x, P.b.copy(), max_iter=20000, res_rat=1e-8, res_tol=1e-18)
            assert abs(K.last.iterations - st["iterations"]) <= (0 if exact else 2)
            assert relerr(x, xo) <= (0.0 if exact else RTOL_X)
            xa = np.zeros(P.N)
            ok, ncyc = engine.AC(s, exact_sums=exact).vcycle(xa, P.b.copy(), factor=1e-8)
            assert ncyc == sr["cycles"] and ok == bool(sr["converged"])
            assert relerr(xa, xr) <= (0.0 if exact else RTOL_X)


def test_periodic_couplings_need_a_periodic_session(engine, oracle):
    """A matrix that couples cells across an outer face is refused, with
    PBG_ERR_UNSUPPORTED, by a session whose boundaries there are walls: the
    solvers would otherwise solve a different operator. With periodic
    boundaries on those axes the same matrix is taken, and the engine solver
    (walls only) refuses it."""
    g = load("per12")
    P = problem_of(g, oracle)
    A = {k: g["A_" + k] for k in "cwesnbt"}
    with engine.Session(*P.dims, P.h) as s:
        with pytest.raises(engine.PbgError) as e:
            s.upload_matrix(A)
        assert e.value.code == engine.ERR_UNSUPPORTED
    with engine.Session(*P.dims, P.h, bc=bc_of(P)) as s:
        s.upload_matrix(A)
        assert s.symmetric()
        M = s.download_matrix()
        for k in "cwesnbt":
            assert np.array_equal(M[k], A[k]), k
        with pytest.raises(engine.PbgError) as e:
            engine.Engine(s).solve(np.zeros(P.N), P.b.copy(), tol=1e-8)
        assert e.value.code == engine.ERR_UNSUPPORTED


@pytest.mark.parametrize("run", sorted(ACX_RUNS))
def test_ac_extended_parity(engine, oracle, run):
    """The rest of AC's surface against the reference run that way (fixture
    acx12): flex cycle (AC::resrat 0.1), the "just solve" branch,
    use_linf_error, a full-cycle start (whose divergence check restores the
    initial guess, as the reference's does), AC's own solver, min_cycles.
    Exact sums: cycles, history and iterate bit for bit."""
    g = load("acx12")
    P = problem_of(g, oracle)
    _, ac_kw, cyc_kw = ACX_RUNS[run]
    x = np.zeros(P.N)
    with session_for(engine, P) as s:
        s.upload_ci(g["ci"])
        ac = engine.AC(s, exact_sums=True, solver=ac_kw.get("solver"))
        if "resrat" in ac_kw:
            ac.resrat(ac_kw["resrat"])
        ac.use_linf_error(ac_kw.get("use_linf", False))
        ac.min_cycles(cyc_kw.get("min_cyc", 0))
        ok, ncyc = ac.cycle(x, P.b.copy(), init=cyc_kw.get("init", engine.CYCLE_NONE),
                            loop=cyc_kw["loop"], factor=1e-8)
        hist = s.history()
    assert ok == bool(g[run + "_converged"])
    assert ncyc == int(g[run + "_cycles"])
    np.testing.assert_allclose(hist, g[run + "_hist"], rtol=1e-13)
    assert np.array_equal(x, g[run + "_x"])


def test_ac_rejects_unknown_cycles(engine, oracle):
    P = problem_of(load("acx12"), oracle)
    with session_for(engine, P) as s:
        for loop in (0, 3, 6):
            with pytest.raises(engine.PbgError) as e:
                engine.AC(s).cycle(np.zeros(P.N), P.b.copy(), loop=loop, factor=1e-8)
            assert e.value.code == engine.ERR_ARG
