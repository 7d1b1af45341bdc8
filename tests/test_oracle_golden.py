"""The CPU oracle against the reference's own outputs (golden fixtures made
by tests/golden/make_golden.py from the compiled reference)."""
import numpy as np
import pytest

from golden_util import ACX_RUNS, NAMES, load, problem_of


@pytest.mark.parametrize("name", NAMES)
def test_fixture_matrix_and_rhs_bit_exact(oracle, name):
    g = load(name)
    P = problem_of(g, oracle)
    assert P.dims == tuple(g["dims"])
    for k in "cwesnbt":
        assert np.array_equal(P.A[k], g["A_" + k]), k
    assert np.array_equal(P.ci, g["ci"])
    assert np.array_equal(P.b, g["b"])


def _krylov_runs():
    out = []
    for n in NAMES:
        for key in load(n):
            if key.endswith("_x") and key.split("_")[0] in ("cg", "bicgs", "cgs", "jacobi", "gs"):
                out.append((n, key[:-2]))
    return out


@pytest.mark.parametrize("name,run", _krylov_runs())
def test_krylov_bit_exact(oracle, name, run):
    """CG, BiCGS and CGS, with the diagonal or an IC preconditioner, and
    Jacobi and Gauss-Seidel (with the reference's stored ci), on symmetric
    and convected (non-symmetric) fixtures."""
    g = load(name)
    P = problem_of(g, oracle)
    parts = run.split("_")
    solver, prec = parts[0], (parts[1] if len(parts) > 1 else "di")
    rr, mi = 1e-8, 20000
    if run + "_maxit" in g:
        rr, mi = float(g[run + "_resrat"]), int(g[run + "_maxit"])
        assert np.array_equal(P.ci, g["ci"])
    x, st = oracle.cg(P, res_rat=rr, maxit=mi, solver=solver, prec=prec)
    assert st["printed"] == int(g[run + "_iterations"])
    assert st["converged"] == int(g[run + "_converged"])
    assert np.array_equal(x, g[run + "_x"], equal_nan=True)


AC_RUNS = {"ac": dict(loop=1), "ac_w": dict(loop=4), "ac_f": dict(loop=2),
           "ac_noguard": dict(loop=1, stop_if_div=0, max_cyc=6)}


@pytest.mark.parametrize("name,run", [(n, r) for n in NAMES for r in AC_RUNS if r + "_x" in load(n)])
def test_ac_bit_exact(oracle, name, run):
    g = load(name)
    P = problem_of(g, oracle)
    ac = oracle.AC(P)
    x, st = ac.cycle(factor=1e-8, **AC_RUNS[run])
    assert st["cycles"] == int(g[run + "_cycles"])
    assert st["converged"] == int(g[run + "_converged"])
    # residual values: the reference's cell volume is a product of node-coordinate
    # differences (Domain::dV, domain_surfaces_volumes.cpp:60-61), uniform only to
    # rounding when 1/n is not a binary fraction; solutions stay bit-exact.
    np.testing.assert_allclose(st["hist"], g[run + "_hist"], rtol=1e-13, atol=0)
    assert np.array_equal(x, g[run + "_x"])


@pytest.mark.parametrize("name,run", [(n, k[:-2]) for n in NAMES for k in load(n)
                                      if k.startswith("acsm_") and k.endswith("_x")])
def test_ac_other_smoothers_bit_exact(oracle, name, run):
    """AC whose levels are smoothed by Gauss-Seidel, Jacobi, BiCGS, CGS or
    IC0-preconditioned CG (the reference's Pressure solver of that kind):
    cycles, history and iterate."""
    g = load(name)
    P = problem_of(g, oracle)
    assert np.array_equal(P.ci, g["ci"])
    sm, _, pr = run.split("_")[1].partition("-")
    ac = oracle.AC(P, smoother=sm, prec=pr or "di")
    x, st = ac.cycle(factor=1e-8, loop=1)
    assert st["cycles"] == int(g[run + "_cycles"])
    assert st["converged"] == int(g[run + "_converged"])
    np.testing.assert_allclose(st["hist"], g[run + "_hist"], rtol=1e-13, atol=0)
    assert np.array_equal(x, g[run + "_x"])


def test_mt64_matches_standard_engine(oracle):
    # the 10000th draw of a default-seeded mt19937_64 is fixed by the C++ standard
    import ctypes
    import subprocess, tempfile, os
    src = r'''
    #include <stdio.h>
    #include "problem_gen.h"
    int main(){ pbg_mt64 g; pbg_mt64_seed(&g, 5489ULL); unsigned long long v=0;
      for(int i=0;i<10000;++i) v=pbg_mt64_next(&g); printf("%llu\n", v); return 0; }
    '''
    d = tempfile.mkdtemp()
    c = os.path.join(d, "t.c")
    open(c, "w").write(src)
    exe = os.path.join(d, "t")
    subprocess.check_call(["gcc", "-std=c99", "-I", oracle.PROBLEM_GEN_DIR, c, "-o", exe, "-lm"])
    assert subprocess.check_output([exe]).strip() == b"9981545732273789042"


@pytest.mark.parametrize("run", sorted(ACX_RUNS))
def test_ac_extended_bit_exact(oracle, run):
    """Flex cycle, "just solve", use_linf_error, a full-cycle start, AC's own
    solver and min_cycles, each against the reference run that way."""
    g = load("acx12")
    P = problem_of(g, oracle)
    _, ac_kw, cyc_kw = ACX_RUNS[run]
    ac = oracle.AC(P, **ac_kw)
    x, st = ac.cycle(factor=1e-8, **cyc_kw)
    assert not ac.flex_capped
    assert st["cycles"] == int(g[run + "_cycles"])
    assert st["converged"] == int(g[run + "_converged"])
    np.testing.assert_allclose(st["hist"], g[run + "_hist"], rtol=1e-13)
    assert np.array_equal(x, g[run + "_x"])
