"""The pressure-correction step oracle (oracle/flow.py) against the
reference: the committed fixtures made by the compiled reference's own
Pressure::discretize / update_rhs / CG / Momentum::project
(tests/golden/make_golden.py --steps), and live runs where the reference
harness is built. CPU only."""
import numpy as np
import pytest

import flow
import oracle_py
from golden_util import GOLDEN, problem_of

import os

STEP_NAMES = ["step8", "step2d", "step12"]


def _load(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def _exact_grid(P):
    """True where the reference's grid coordinates are exact multiples of h
    (n a power of two in every real direction)."""
    return all(n & (n - 1) == 0 for n in P.dims if n > 1)


@pytest.mark.parametrize("name", STEP_NAMES)
def test_step_oracle_matches_golden(oracle, name):
    g = _load(name)
    P = problem_of(g, oracle)
    r = flow.step(P, float(g["dt"]), res_rat=float(g["res_rat"]))
    assert r["stats"]["printed"] == int(g["iterations"])
    pairs = [(r["A"][k], g["A_" + k]) for k in "cwsb"] + [(r["b"], g["rhs"])] + \
        [(r[k].reshape(-1), g[k].reshape(-1)) for k in "xuvw"]
    for got, ref in pairs:
        if _exact_grid(P):
            assert np.array_equal(got, ref)
        else:
            # the reference's grid spacings of a non-power-of-two n carry
            # rounding from its node fit; the restatement uses h exactly
            assert np.abs(got - ref).max() <= 1e-11 * max(np.abs(ref).max(), 1e-300)


@pytest.mark.skipif(not oracle_py.harness_available(), reason="reference harness not built here")
@pytest.mark.parametrize("kind,kw,dt", [(0, dict(n=16), 1.0), (0, dict(n=32), 0.002),
                                        (2, dict(index=3, n2d=1, s2=(64, 64)), 0.05),
                                        (2, dict(index=0, n2d=1, s2=(32, 32)), 1.0)])
def test_step_oracle_matches_reference_live(oracle, kind, kw, dt):
    P = oracle.Problem(kind, 13, **kw)
    if not _exact_grid(P):
        pytest.skip("grid %s is not a power of two" % (P.dims,))
    ref = flow.run_reference_step(P, dt)
    r = flow.step(P, dt)
    assert r["stats"]["printed"] == int(ref["meta"]["iterations"])
    for k in "cwesnbt":
        assert np.array_equal(r["A"][k], ref["A"][k]), k
    assert np.array_equal(r["A"]["ci"], ref["ci"])
    for k in "bxuvw":
        assert np.array_equal(np.reshape(r[k], -1), np.reshape(ref[k], -1)), k


@pytest.mark.parametrize("kind,kw,bc", [(0, dict(n=16), [0] * 6), (0, dict(n=16), None),
                                        (1, dict(n=24, nb=3, rmin=2.0, rmax=3.0, rc=5.0), None)])
def test_projection_removes_divergence(oracle, kind, kw, bc):
    """The projected field's divergence is the solver's residual, far below
    the predicted field's: with Neumann sides everywhere; with a Dirichlet
    top, whose wall face the projection keeps (the matrix couples to the
    wall pressure there, so only the cells below it keep a residue); with
    a voxel solid (faces to it closed on both sides)."""
    P = oracle.Problem(kind, 5, **kw)
    dt = 0.01
    r = flow.step(P, dt, res_rat=1e-12, bc=bc)
    sol = P.solid if np.any(P.solid) else None
    d0 = flow.divergence(P.dims, P.h, dt, r["u0"], r["v0"], r["w0"], solid=sol).reshape(P.dims)
    d1 = flow.divergence(P.dims, P.h, dt, r["u"], r["v"], r["w"], solid=sol).reshape(P.dims)
    if bc is None:
        d0, d1 = d0[:, :, :-1], d1[:, :, :-1]
    assert np.abs(d1).max() < 1e-9 * np.abs(d0).max()
    # the projection only touches interior faces
    assert np.all(r["u"][0] == 0.0) and np.all(r["u"][-1] == 0.0)
    assert np.all(r["v"][:, 0] == 0.0) and np.all(r["w"][:, :, -1] == 0.0)


def test_planted_density_error_is_caught(oracle):
    """A harmonic face density in place of PropertyMix's arithmetic mean
    (planted in the oracle) changes the matrix: the golden comparison
    would fail."""
    g = _load("step8")
    P = problem_of(g, oracle)
    col, u, v, w, ra, rb, bc = flow.flow_state(P)
    good = flow.assemble_mix(P.dims, P.h, bc, col, ra, rb)
    saved = flow.face_density
    try:
        def harmonic(cell, axis):
            inv = saved(1.0 / cell, axis)
            return 1.0 / inv
        flow.face_density = harmonic
        bad = flow.assemble_mix(P.dims, P.h, bc, col, ra, rb)
    finally:
        flow.face_density = saved
    assert np.array_equal(good["c"], g["A_c"])
    assert not np.array_equal(bad["c"], g["A_c"])


def _body(g):
    return dict(fV=g["fV"], fS=g["fS"])


@pytest.mark.parametrize("name", ["stepbody16", "stepbody32"])
def test_body_step_oracle_matches_golden(oracle, name):
    """A sphere cut by the reference's own Body (STL): the body branches of
    discretize (cut-cell fractions, off-cell decoupling; a non-symmetric
    matrix), update_rhs (face fractions) and project, bit for bit."""
    g = _load(name)
    P = problem_of(g, oracle)
    r = flow.step(P, float(g["dt"]), res_rat=float(g["res_rat"]), body=_body(g))
    assert r["stats"]["printed"] == int(g["iterations"])
    for k in "cwesnbt":
        assert np.array_equal(r["A"][k], g["A_" + k]), k
    assert not np.array_equal(r["A"]["e"].reshape(P.dims)[:-1], r["A"]["w"].reshape(P.dims)[1:])
    assert np.array_equal(r["A"]["ci"], g["ci"])
    assert np.array_equal(r["b"], g["rhs"])
    for k in "xuvw":
        assert np.array_equal(r[k].reshape(-1), g[k].reshape(-1)), k


@pytest.mark.skipif(not oracle_py.harness_available(), reason="reference harness not built here")
@pytest.mark.parametrize("n,radius,dt", [(32, 9.7, 0.003), (16, 5.55, 1.0)])
def test_body_step_oracle_matches_reference_live(oracle, n, radius, dt):
    P = oracle.Problem(0, 13, n=n)
    ref = flow.run_reference_step(P, dt, body=radius)
    bd = ref["body"]
    cut = (bd["fV"] > 0) & (bd["fV"] < 1)
    assert np.array_equal(bd["listed"] > 0, cut)  # the cut-cell list is the cut cells
    r = flow.step(P, dt, body=bd)
    assert r["stats"]["printed"] == int(ref["meta"]["iterations"])
    for k in "cwesnbt":
        assert np.array_equal(r["A"][k], ref["A"][k]), k
    for k in "bxuvw":
        assert np.array_equal(np.reshape(r[k], -1), np.reshape(ref[k], -1)), k


def test_sampled_sphere_body_is_consistent():
    """The bench's sampled sphere (bench.sphere_body) has the structure of a
    cut body: every cell the surface crosses is cut and keeps an open face,
    no fluid cell meets a cell inside the body, and the oracle's assembly
    with it has a positive diagonal everywhere."""
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(GOLDEN)))  # the repository root
    import bench
    n = 32
    fV, fS = bench.sphere_body(n, n / 6.0)
    V = fV.reshape(n, n, n)
    F = fS.reshape(6, n, n, n)
    off, full, cut = V == 0.0, V == 1.0, (V > 0.0) & (V < 1.0)
    assert cut.sum() > 0 and off.sum() > 0
    assert (F.max(axis=0)[cut] > 0.0).all()
    for ax in range(3):
        a, b = np.swapaxes(off, 0, ax), np.swapaxes(full, 0, ax)
        assert not ((a[1:] & b[:-1]) | (a[:-1] & b[1:])).any()
    A = flow.assemble_mix((n, n, n), 1.0 / n, [0, 0, 0, 0, 0, 1], None, 1.0, 1.0,
                          solid=off.reshape(-1).astype(np.uint8), body=dict(fV=fV, fS=fS))
    assert (A["c"] > 0.0).all()


def _sparse(dims, A):
    """The seven-array matrix (c x - sum a_nb x_nb) as scipy CSR."""
    import scipy.sparse as sp
    nx, ny, nz = dims
    N = nx * ny * nz
    idx = np.arange(N).reshape(dims)
    I, J, K = np.meshgrid(range(nx), range(ny), range(nz), indexing="ij")
    rows, cols, vals = [idx.ravel()], [idx.ravel()], [A["c"]]
    for key, ax, sh, mask in (("w", 0, -1, I > 0), ("e", 0, 1, I < nx - 1), ("s", 1, -1, J > 0),
                              ("n", 1, 1, J < ny - 1), ("b", 2, -1, K > 0), ("t", 2, 1, K < nz - 1)):
        nb = np.roll(idx, -sh, ax)
        rows.append(idx[mask])
        cols.append(nb[mask])
        vals.append(-A[key].reshape(dims)[mask])
    return sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(N, N))


def test_symmetric_part_refinement_on_reference_body():
    """The engine's symmetric approximation of a cut body's matrix (mean of
    the two sides, one-sided couplings dropped, c kept; k_symmetrize),
    restated with scipy on the reference's own sphere matrix: the refinement
    around it with exact inner solves reduces the residual by at most 5e-2
    per sweep past the first."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as sla
    g = _load("stepbody16")
    dims = tuple(int(v) for v in g["dims"])
    M = _sparse(dims, {k: g["A_" + k] for k in "cwesnbt"})
    off = M - sp.diags(M.diagonal())
    offT = off.T.tocsr()
    both = off.multiply(offT) != 0          # couplings both sides keep
    S = (off + offT).multiply(both) * 0.5 + sp.diags(M.diagonal())
    lu = sla.splu(S.tocsc())
    b = g["rhs"]
    x = np.zeros_like(b)
    rel = []
    for _ in range(5):
        r = b - M @ x
        rel.append(np.linalg.norm(r) / np.linalg.norm(b))
        x = x + lu.solve(r)
    for k in range(2, len(rel)):
        assert rel[k] <= 5e-2 * rel[k - 1], rel
