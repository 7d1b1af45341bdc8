"""The pressure-correction step on the GPU (pbg_assemble_mix,
pbg_divergence, pbg_project, pbg_pressure_step) against the oracle
(oracle/flow.py) and the compiled reference's fixtures
(tests/golden/step*.npz).

Tolerances: assembly, divergence and projection are bit-exact against the
oracle on every grid (the reference's operation order, whether a thread
owns one cell or four cells of a k-row). The whole step with the reference-parity CG (exact_sums) is
bit-exact against the reference on grids whose n is a power of two; for
other n the reference's own grid spacings carry rounding, and the step
agrees to 1e-11 relative. The engine's step is held to the divergence it
leaves behind.
"""
import os

import numpy as np
import pytest

import flow
from golden_util import GOLDEN, problem_of

pytestmark = pytest.mark.gpu

CASES = [(0, dict(n=16)), (0, dict(n=12)), (1, dict(n=20, nb=3, rmin=2.0, rmax=3.0, rc=4.0)),
         (2, dict(index=0, n2d=1, s2=(32, 32))), (2, dict(index=3, n2d=1, s2=(20, 40))),
         # nz % 4 == 0 grids run the 4-cells-a-thread kernels, others the one-cell ones
         (1, dict(n=28, nb=4, rmin=2.0, rmax=4.0, rc=6.0)), (0, dict(n=13))]


def _state(oracle, kind, kw, seed=5):
    P = oracle.Problem(kind, seed, **kw)
    col, u, v, w, ra, rb, bc = flow.flow_state(P)
    return P, col, u, v, w, ra, rb, bc


def _solid(P):
    return P.solid if np.any(P.solid) else None


@pytest.mark.parametrize("kind,kw", CASES)
def test_assemble_mix_bit_exact(engine, oracle, kind, kw):
    P, col, u, v, w, ra, rb, bc = _state(oracle, kind, kw)
    sol = _solid(P)
    ref = flow.assemble_mix(P.dims, P.h, bc, col, ra, rb, solid=sol)
    with engine.Session(*P.dims, P.h, bc=bc) as s:
        s.assemble_mix(col, ra, rb, solid=sol)
        assert s.symmetric()
        M = s.download_matrix()
        for k in "cwesnbt":
            assert np.array_equal(M[k], ref[k]), k
        # one fluid: the constant density
        s.assemble_mix(None, ra)
        M = s.download_matrix()
    one = flow.assemble_mix(P.dims, P.h, bc, None, ra, rb)
    for k in "cwesnbt":
        assert np.array_equal(M[k], one[k]), k


@pytest.mark.parametrize("kind,kw", CASES)
@pytest.mark.parametrize("dt", [1.0, 0.0037])
def test_divergence_and_project_bit_exact(engine, oracle, kind, kw, dt):
    P, col, u, v, w, ra, rb, bc = _state(oracle, kind, kw)
    rng = np.random.default_rng(3)
    p = rng.standard_normal(P.N)
    sols = [None] + ([P.solid] if np.any(P.solid) else [])
    with engine.Session(*P.dims, P.h, bc=bc) as s:
        for sol in sols:
            rhs = s.divergence(u, v, w, dt, np.zeros(P.N), solid=sol)
            assert np.array_equal(rhs, flow.divergence(P.dims, P.h, dt, u, v, w, solid=sol))
            if P.nz == 1:
                rhs2 = s.divergence(u, v, None, dt, np.zeros(P.N), solid=sol)
                assert np.array_equal(rhs2, rhs)
            for c in (col, None):
                uu, vv, ww = u.copy(), v.copy(), w.copy()
                s.project(p, c, ra, rb, dt, uu, vv, ww, solid=sol)
                ru, rv, rw = flow.project(P.dims, P.h, dt, p, c, ra, rb, u, v, w, solid=sol)
                assert np.array_equal(uu, ru) and np.array_equal(vv, rv) and np.array_equal(ww, rw)


# Grids whose marching tiles are partial or several: k rows longer than one
# 256-cell tile (264), j beyond one tile of rows, i over several walks, and
# odd extents; a colour field with two ramped bubbles, a solid box, spacings
# that are not powers of two and densities 1000 and 0.8.
TILE_DIMS = [(37, 41, 264), (19, 9, 12), (33, 70, 20)]


def _tile_state(dims, seed=11):
    rng = np.random.default_rng(seed)
    nx, ny, nz = dims
    i, j, k = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    col = np.ones(dims)
    for ci, cj, ck, r in ((0.3, 0.4, 0.5, 0.25), (0.7, 0.7, 0.2, 0.2)):
        d = np.sqrt((i - ci * nx) ** 2 + (j - cj * ny) ** 2 + (k - ck * nz) ** 2)
        col = np.minimum(col, np.clip((d - r * min(dims)) / 3.0 + 0.5, 0.0, 1.0))
    solid = np.zeros(dims, dtype=np.uint8)
    solid[nx // 2:nx // 2 + 3, ny // 3:ny // 3 + 4, :max(1, nz // 4)] = 1
    u = rng.uniform(-0.5, 0.5, (nx + 1, ny, nz))
    v = rng.uniform(-0.5, 0.5, (nx, ny + 1, nz))
    w = rng.uniform(-0.5, 0.5, (nx, ny, nz + 1))
    u[0] = u[-1] = 0.0
    v[:, 0] = v[:, -1] = 0.0
    w[:, :, 0] = w[:, :, -1] = 0.0
    return col, solid.reshape(-1), u, v, w, 1.0 / (nx + 0.5)


@pytest.mark.parametrize("dims", TILE_DIMS)
def test_flow_tiles_bit_exact(engine, dims):
    col, solid, u, v, w, h = _tile_state(dims)
    ra, rb = 1000.0, 0.8
    bc = [0, 0, 0, 0, 0, 1]
    N = int(np.prod(dims))
    # a random pressure, and a flat one with signed zeros (zero differences
    # across most faces, -0 across some: the quotients are signed zeros)
    p = np.random.default_rng(4).standard_normal(N)
    pz = np.zeros(N)
    pz[::7] = -0.0
    pz[::11] = 0.25
    with engine.Session(*dims, h, bc=bc) as s:
        for sol in (None, solid):
            s.assemble_mix(col, ra, rb, solid=sol)
            M = s.download_matrix()
            ref = flow.assemble_mix(dims, h, bc, col, ra, rb, solid=sol)
            for key in "cwesnbt":
                assert np.array_equal(M[key], ref[key]), key
            rhs = s.divergence(u, v, w, 0.0037, np.zeros(N), solid=sol)
            assert np.array_equal(rhs, flow.divergence(dims, h, 0.0037, u, v, w, solid=sol))
            for c in (col, None):
                for pp in (p, pz):
                    uu, vv, ww = u.copy(), v.copy(), w.copy()
                    s.project(pp, c, ra, rb, 0.0037, uu, vv, ww, solid=sol)
                    ru, rv, rw = flow.project(dims, h, 0.0037, pp, c, ra, rb, u, v, w, solid=sol)
                    for a_, b_ in ((uu, ru), (vv, rv), (ww, rw)):
                        assert np.array_equal(a_.view(np.int64), b_.view(np.int64))


def _cg_params(engine, res_rat):
    prm = engine.default_params(engine.SOLVER_CG)
    prm.exact_sums = 1
    prm.res_rat = res_rat
    prm.res_tol = 1e-18
    prm.max_iter = 20000
    return prm


@pytest.mark.parametrize("name", ["step8", "step2d", "step12"])
def test_pressure_step_matches_reference(engine, oracle, name):
    """One call: assemble, divergence, CG (exact sums), project, against the
    reference's own step."""
    g = dict(np.load(os.path.join(GOLDEN, name + ".npz")))
    P = problem_of(g, oracle)
    col, u, v, w, ra, rb, bc = flow.flow_state(P)
    dt = float(g["dt"])
    p = np.zeros(P.N)
    with engine.Session(*P.dims, P.h, bc=bc) as s:
        res = s.pressure_step(col, ra, rb, dt, u, v, w, p, _cg_params(engine, float(g["res_rat"])))
        assert res.iterations == int(g["iterations"])
        M = s.download_matrix()
    exact = all(n & (n - 1) == 0 for n in P.dims if n > 1)
    pairs = [(M[k], g["A_" + k]) for k in "cwsb"] + [(p, g["x"])] + \
        [(a.reshape(-1), g[k].reshape(-1)) for a, k in ((u, "u"), (v, "v"), (w, "w"))]
    for got, ref in pairs:
        if exact:
            assert np.array_equal(got, ref)
        else:
            assert np.abs(got - ref).max() <= 1e-11 * np.abs(ref).max()


def test_pressure_step_device_tensors(engine, oracle):
    """CUDA tensors in, nothing crossing to the host: the same bits as the
    host-buffer call."""
    import torch
    P, col, u, v, w, ra, rb, bc = _state(oracle, 0, dict(n=32))
    prm = _cg_params(engine, 1e-10)
    dt = 0.01
    hu, hv, hw, hp = u.copy(), v.copy(), w.copy(), np.zeros(P.N)
    tu, tv, tw = (torch.from_numpy(a.copy()).cuda() for a in (u, v, w))
    tp = torch.zeros(P.N, dtype=torch.float64, device="cuda")
    tc = torch.from_numpy(col.reshape(-1).copy()).cuda()
    with engine.Session(*P.dims, P.h, bc=bc) as s:
        r1 = s.pressure_step(col, ra, rb, dt, hu, hv, hw, hp, prm)
        r2 = s.pressure_step(tc, ra, rb, dt, tu, tv, tw, tp, prm)
    torch.cuda.synchronize()
    assert r1.iterations == r2.iterations
    assert np.array_equal(tp.cpu().numpy(), hp)
    for t, a in ((tu, hu), (tv, hv), (tw, hw)):
        assert np.array_equal(t.cpu().numpy(), a)


@pytest.mark.parametrize("kind,kw,mixed", [(0, dict(n=64), 0), (0, dict(n=128), 1),
                                           (1, dict(n=128, nb=8, rmin=4.0, rmax=10.0, rc=15.0), 1)])
def test_engine_step_leaves_divergence_free_field(engine, oracle, kind, kw, mixed):
    """Size-independent property at sizes the oracle cannot run quickly:
    with Neumann sides everywhere the projected field's divergence is the
    engine's residual, |div u| / |div u*| <= 10 * tol (a voxel solid
    included: its faces are closed on both sides)."""
    P, col, u, v, w, ra, rb, _ = _state(oracle, kind, kw)
    sol = _solid(P)
    bc = [0] * 6
    dt = 0.01
    prm = engine.default_params(engine.SOLVER_ENGINE)
    prm.precision = mixed
    prm.tol = 1e-9
    p = np.zeros(P.N)
    with engine.Session(*P.dims, P.h, bc=bc) as s:
        d0 = s.divergence(u, v, w, dt, np.zeros(P.N), solid=sol)
        res = s.pressure_step(col, ra, rb, dt, u, v, w, p, prm, solid=sol)
        d1 = s.divergence(u, v, w, dt, np.zeros(P.N), solid=sol)
    assert res.converged
    assert np.linalg.norm(d1) <= 10 * prm.tol * np.linalg.norm(d0)
    assert np.all(u[0] == 0.0) and np.all(u[-1] == 0.0) and np.all(w[:, :, 0] == 0.0)


def _body(g):
    return np.ascontiguousarray(g["fV"]), np.ascontiguousarray(g["fS"])


@pytest.mark.parametrize("name", ["stepbody16", "stepbody32"])
def test_body_step_matches_reference(engine, oracle, name):
    """A sphere cut by the reference's Body: assemble (seven arrays), divergence,
    CG with exact sums and projection equal the reference's step bit for bit."""
    g = dict(np.load(os.path.join(GOLDEN, name + ".npz")))
    P = problem_of(g, oracle)
    col, u, v, w, ra, rb, bc = flow.flow_state(P)
    dt = float(g["dt"])
    p = np.zeros(P.N)
    with engine.Session(*P.dims, P.h, bc=bc) as s:
        s.upload_body(*_body(g))
        res = s.pressure_step(col, ra, rb, dt, u, v, w, p, _cg_params(engine, float(g["res_rat"])))
        assert res.iterations == int(g["iterations"])
        assert not s.symmetric()
        M = s.download_matrix()
    for k in "cwesnbt":
        assert np.array_equal(M[k], g["A_" + k]), k
    assert np.array_equal(p, g["x"])
    for a, k in ((u, "u"), (v, "v"), (w, "w")):
        assert np.array_equal(a.reshape(-1), g[k].reshape(-1)), k


def test_body_stages_match_oracle(engine, oracle):
    """Each stage with the body against the oracle, and the rules around it."""
    g = dict(np.load(os.path.join(GOLDEN, "stepbody16.npz")))
    P = problem_of(g, oracle)
    col, u, v, w, ra, rb, bc = flow.flow_state(P)
    body = dict(fV=g["fV"], fS=g["fS"])
    off = (g["fV"] == 0).astype(np.uint8)
    dt = float(g["dt"])
    ref_A = flow.assemble_mix(P.dims, P.h, bc, col, ra, rb, solid=off, body=body)
    ref_b = flow.divergence(P.dims, P.h, dt, u, v, w, solid=off, body=body)
    x = np.asarray(g["x"], dtype=np.float64)
    ref_uvw = flow.project(P.dims, P.h, dt, x, col, ra, rb, u, v, w, solid=off)
    with engine.Session(*P.dims, P.h, bc=bc) as s:
        s.upload_body(*_body(g))
        s.assemble_mix(col, ra, rb)
        M = s.download_matrix()
        for k in "cwesnbt":
            assert np.array_equal(M[k], ref_A[k]), k
        rhs = np.zeros(P.N)
        s.divergence(u, v, w, dt, rhs)
        assert np.array_equal(rhs, ref_b)
        uu, vv, ww = u.copy(), v.copy(), w.copy()
        s.project(x, col, ra, rb, dt, uu, vv, ww)
        for a, b in zip((uu, vv, ww), ref_uvw):
            assert np.array_equal(a.reshape(-1), np.reshape(b, -1))
        # a body and a voxel mask together are refused
        with pytest.raises(engine.PbgError):
            s.assemble_mix(col, ra, rb, solid=off)
        # the engine's solver takes the seven-array form (refinement around
        # its symmetric part)
        prm = engine.default_params(engine.SOLVER_ENGINE)
        prm.precision = engine.MIXED
        res = s.solve(np.zeros(P.N), rhs, prm)
        assert res.converged and res.relres <= 1e-8
        # without the body the symmetric form comes back
        s.upload_body(None, None)
        s.assemble_mix(col, ra, rb)
        assert s.symmetric()
        # a cut cell on the domain boundary is refused
        fV = np.ones(P.N)
        fV[0] = 0.5
        with pytest.raises(engine.PbgError):
            s.upload_body(fV, np.ones((6, P.N)))


@pytest.mark.parametrize("precision", [0, 1])
def test_engine_step_with_body(engine, oracle, precision):
    """The engine's solver on a cut body's non-symmetric matrix: its hierarchy
    is built from the symmetric part and the FP64 refinement runs against the
    matrix itself, to the same 1e-8 true residual. The pressure is held to a
    tight oracle solve of the same matrix (CG to 1e-13) as in the engine's
    own tests."""
    g = dict(np.load(os.path.join(GOLDEN, "stepbody16.npz")))
    P = problem_of(g, oracle)
    col, u, v, w, ra, rb, bc = flow.flow_state(P)
    dt = float(g["dt"])
    p = np.zeros(P.N)
    prm = engine.default_params(engine.SOLVER_ENGINE)
    prm.precision = precision
    prm.tol = 1e-8
    with engine.Session(*P.dims, P.h, bc=bc) as s:
        s.upload_body(*_body(g))
        res = s.pressure_step(col, ra, rb, dt, u, v, w, p, prm)
        assert res.converged and res.relres <= 1e-8
        M = s.download_matrix()
        b = np.zeros(P.N)
        s.divergence(*[np.asarray(a, dtype=np.float64) for a in flow.flow_state(P)[1:4]], dt, b)
    sp = flow.StepProblem(P.dims, P.h, M, b)
    r = b - oracle.spmv(sp, p)
    assert np.linalg.norm(r) <= 1.0001e-8 * np.linalg.norm(b)
    xt, _ = oracle.cg(sp, b=b, res_rat=1e-13, res_tol=1e-30, maxit=100000, scale=1.0 / dt)
    assert np.linalg.norm(p - xt) <= 1e-4 * np.linalg.norm(xt)
    for a, k in ((u, "u"), (v, "v"), (w, "w")):
        assert np.abs(a.reshape(-1) - g[k].reshape(-1)).max() <= 1e-4 * np.abs(g[k]).max(), k
