"""Pressure-correction step restated in numpy: the oracle of the on-device
assembly from a colour function, the divergence right-hand side and the
velocity projection.

TEST INFRASTRUCTURE ONLY: imported by tests/ and bench.py's CPU legs as the
checker; the engine never imports it.

What it restates (reference file:line):
  * mix_density      PropertyMix::value(i,j,k), Src/Matter/property_value.cpp:52-70
                     (a * col + b * (1 - col), col clamped to [0, 1]).
  * face_density     PropertyMix::value(Comp,i,j,k), :73-85 without a
                     staggered colour: 0.5 * (value(i) + value(i-1)); the
                     ghost cell beyond the domain holds the boundary cell's
                     value (Scalar::bnd_update for Neumann and pseudo sides,
                     Src/Field/Scalar/scalar_bnd_update.cpp:102-104).
  * assemble_mix     Pressure::discretize, Src/Equation/Centered/Pressure/
                     pressure_discretize.cpp:24-67 (a_w = dS / dxw / rho_w,
                     c = w + e + s + n + b + t; dxw is h / 2 on the
                     domain boundary) and :125-148, then
                     Centered::create_system_bnd, Src/Equation/Centered/
                     centered_system_bnd.cpp:17-62 (Neumann, and the pseudo
                     k sides of a 2-D grid: c -= a_bnd, a_bnd = 0, in the
                     order imin, imax, jmin, jmax, kmin, kmax) and :142-184
                     (Dirichlet: a_bnd = 0).
  * divergence       Pressure::update_rhs, pressure_update_rhs.cpp:25-53,
                     134-136 (fnew = 0, += a_w u_w, -= a_e u_e, += a_s v_s,
                     -= a_n v_n, += a_b w_b, -= a_t w_t with a = dS * dti;
                     then += fext + fbnd, both zero here); a solid mask
                     takes the immersed-body branch (:65-101) of a voxel
                     body.
  * project          Momentum::project, Src/Equation/Staggered/Momentum/
                     momentum_project.cpp:26-45: u += (p[i-1] - p[i]) /
                     rho_face * dt / dxc on every interior face (with a
                     solid mask :47-73: faces between fluid cells only,
                     (dp * dt) / rho / dxc); the normal faces on the domain
                     boundary keep their boundary value (the walls of
                     bnd_update_nooutlet, vector_bnd_update.cpp:54-85),
                     and w is not touched in 2-D (kfull false,
                     momentum.cpp:18-30).
The grid is uniform with spacing h: dS = h * h and dxc = h, which are the
reference's own values when the grid coordinates are exact multiples of h
(n a power of two). The operation order follows the reference line by line
(numpy evaluates left to right, without fused multiply-adds).
"""
import ctypes

import numpy as np

import oracle_py as op

PICO = 1.0e-12


def flow_state(P, stream=0):
    """Colour and predicted velocity of pbg_gen_flow for the problem P:
    (col (nx,ny,nz), u (nx+1,ny,nz), v (nx,ny+1,nz), w (nx,ny,nz+1),
    rho_liquid, rho_vapour, bc)."""
    nx, ny, nz = P.dims
    a = P.args
    params = np.array([a["n"], a["nb"], a["rmin"], a["rmax"], a["rc"], a["ratio"], a["index"],
                       a["n2d"], a["s2"][0], a["s2"][1], a["s3"][0], a["s3"][1], stream,
                       a.get("periodic", 0)], dtype=np.float64)
    col = np.zeros((nx, ny, nz))
    u = np.zeros((nx + 1, ny, nz))
    v = np.zeros((nx, ny + 1, nz))
    w = np.zeros((nx, ny, nz + 1))
    rho2 = np.zeros(2)
    bc = np.zeros(6, dtype=np.int32)
    L = op.lib()
    L.orc_gen_flow.restype = ctypes.c_int
    L.orc_gen_flow.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_uint64] + [op._dp] * 5 + [
        ctypes.c_void_p]
    L.orc_gen_flow(P.kind, params.ctypes.data, P.seed, op._p(col), op._p(u), op._p(v), op._p(w),
                   op._p(rho2), bc.ctypes.data)
    return col, u, v, w, float(rho2[0]), float(rho2[1]), [int(t) for t in bc]


def mix_density(col, rho_a, rho_b):
    """Cell density of the two-phase mixture (property_value.cpp:52-70)."""
    c = np.where(col > 1.0, 1.0, col)
    c = np.where(c < 0.0, 0.0, c)
    return rho_a * c + rho_b * (1.0 - c)


def face_density(cell, axis):
    """Density at every face along `axis` (n+1 faces, boundary faces
    included): 0.5 * (value(i) + value(i-1)) with zero-gradient ghosts."""
    first = np.take(cell, [0], axis=axis)
    last = np.take(cell, [cell.shape[axis] - 1], axis=axis)
    g = np.concatenate([first, cell, last], axis=axis)
    n = g.shape[axis]
    hi = np.take(g, np.arange(1, n), axis=axis)
    lo = np.take(g, np.arange(0, n - 1), axis=axis)
    return 0.5 * (hi + lo)


def _cell_density(col, rho_a, rho_b, dims):
    if col is None:
        return None
    return mix_density(np.asarray(col, dtype=np.float64).reshape(dims), rho_a, rho_b)


# the six neighbour directions: matrix key, axis, shift, plane of fS
_DIRS = [("w", 0, -1, 0), ("e", 0, 1, 1), ("s", 1, -1, 2), ("n", 1, 1, 3), ("b", 2, -1, 4),
         ("t", 2, 1, 5)]


def _pair(axis, shift):
    """Index of the cells that have the neighbour (axis, shift) inside the
    domain, and of those neighbours."""
    me = [slice(None)] * 3
    nb = [slice(None)] * 3
    me[axis] = slice(1, None) if shift < 0 else slice(None, -1)
    nb[axis] = slice(None, -1) if shift < 0 else slice(1, None)
    return tuple(me), tuple(nb)


def body_masks(body, dims):
    """off (fV == 0, Body::off_p) and cut (0 < fV < 1, Body::cut_p) cells and
    the face fractions (6, nx, ny, nz) of a body given as fV and fS."""
    fV = np.asarray(body["fV"], dtype=np.float64).reshape(dims)
    fS = np.asarray(body["fS"], dtype=np.float64).reshape((6,) + tuple(dims))
    return fV == 0.0, (fV > 0.0) & (fV < 1.0), fS


def assemble_mix(dims, h, bc, col, rho_a, rho_b, solid=None, body=None):
    """Pressure matrix of a two-phase mixture: dict c, w, e, s, n, b, t, ci
    (flat, compact layout). col None: a single fluid of density rho_a
    (Property::value(Comp) of a constant property is the constant,
    property_value.cpp:18-21). bc: imin..kmax, 0 Neumann / 1 Dirichlet.
    body: dict fV, fS of a cut body (the reference's Body after cutting):
    pressure_discretize.cpp:72-119 over the body's cut-cell list (its cut
    cells): a cut cell's coupling to a cut neighbour times its own face
    fraction, couplings between a listed cell and an off cell zeroed both
    ways, c of every cell not off recomputed."""
    nx, ny, nz = dims
    hx = (h * h) / h
    rc = _cell_density(col, rho_a, rho_b, dims)
    if rc is None:
        fx = np.full((nx + 1, ny, nz), float(rho_a))
        fy = np.full((nx, ny + 1, nz), float(rho_a))
        fz = np.full((nx, ny, nz + 1), float(rho_a))
    else:
        fx, fy, fz = face_density(rc, 0), face_density(rc, 1), face_density(rc, 2)
    # dS / dx of every face: dx is h between two cell centres and h / 2
    # between a boundary cell's centre and the wall, where the reference's
    # ghost cells have zero width (grid1d_correct_boundaries.cpp:11-14,
    # 46-59); the 1-cell dummy direction of a 2-D grid keeps h on both
    # sides (its ghost cells are mirrored, grid1d_dummy_setup.cpp:3-12)
    hxb = (h * h) / (0.5 * h)

    def dsdx(n, axis, shape):
        g = np.full(shape, hx)
        if axis == 2 and n == 1:
            return g
        idx = [slice(None)] * 3
        idx[axis] = 0
        g[tuple(idx)] = hxb
        idx[axis] = n
        g[tuple(idx)] = hxb
        return g

    gx = dsdx(nx, 0, fx.shape)
    gy = dsdx(ny, 1, fy.shape)
    gz = dsdx(nz, 2, fz.shape)
    A = dict(w=gx[:-1] / fx[:-1], e=gx[1:] / fx[1:], s=gy[:, :-1] / fy[:, :-1],
             n=gy[:, 1:] / fy[:, 1:], b=gz[:, :, :-1] / fz[:, :, :-1], t=gz[:, :, 1:] / fz[:, :, 1:])
    c = A["w"] + A["e"] + A["s"] + A["n"] + A["b"] + A["t"]
    sol = None
    if body is not None and np.any(body_masks(body, dims)[1]):
        off, cut, fS = body_masks(body, dims)
        for key, axis, shift, d in _DIRS:
            me, nb = _pair(axis, shift)
            a = A[key][me]
            a = np.where(cut[me] & cut[nb], a * fS[d][me], a)
            a = np.where((cut[me] | cut[nb]) & (off[me] | off[nb]), 0.0, a)
            A[key][me] = a
        c2 = A["w"] + A["e"] + A["s"] + A["n"] + A["b"] + A["t"]
        c = np.where(off, c, c2)
        sol = off
    elif solid is not None and np.any(solid):
        # faces between fluid and solid cells zeroed on both sides; c of
        # fluid cells recomputed (pressure_discretize.cpp:91-117)
        sol = np.asarray(solid).reshape(dims).astype(bool)
        A["w"][1:][sol[1:] != sol[:-1]] = 0.0
        A["e"][:-1][sol[:-1] != sol[1:]] = 0.0
        A["s"][:, 1:][sol[:, 1:] != sol[:, :-1]] = 0.0
        A["n"][:, :-1][sol[:, :-1] != sol[:, 1:]] = 0.0
        A["b"][:, :, 1:][sol[:, :, 1:] != sol[:, :, :-1]] = 0.0
        A["t"][:, :, :-1][sol[:, :, :-1] != sol[:, :, 1:]] = 0.0
        c2 = A["w"] + A["e"] + A["s"] + A["n"] + A["b"] + A["t"]
        c = np.where(sol, c, c2)
    sides = [("w", (0, slice(None), slice(None))), ("e", (nx - 1, slice(None), slice(None))),
             ("s", (slice(None), 0, slice(None))), ("n", (slice(None), ny - 1, slice(None))),
             ("b", (slice(None), slice(None), 0)), ("t", (slice(None), slice(None), nz - 1))]
    for f, (key, sl) in enumerate(sides):
        pseudo = nz == 1 and f >= 4
        if pseudo or bc[f] == 0:
            c[sl] = c[sl] - A[key][sl]
            A[key][sl] = 0.0
    for f, (key, sl) in enumerate(sides):
        if not (nz == 1 and f >= 4) and bc[f] == 1:
            A[key][sl] = 0.0
    ci = 1.0 / c
    if sol is not None:
        c = np.where(sol, c * PICO, c)
        for key in "wesnbt":
            A[key][sol] = 0.0
    out = {k: A[k].reshape(-1).copy() for k in "wesnbt"}
    out["c"] = c.reshape(-1).copy()
    out["ci"] = ci.reshape(-1).copy()
    return out


def divergence(dims, h, dt, u, v, w, solid=None, body=None):
    """Right-hand side of the pressure equation from face velocities
    (flat, compact layout). solid: a voxel body, the immersed-body branch
    of update_rhs (pressure_update_rhs.cpp:65-101; every fluid cell uncut,
    so the face fractions are 1): a face counts only if the cell across it
    is fluid (cells beyond the domain count as fluid), solid cells get 0."""
    nx, ny, nz = dims
    dti = 1.0 / dt
    a = (h * h) * dti
    u = np.asarray(u).reshape(nx + 1, ny, nz)
    v = np.asarray(v).reshape(nx, ny + 1, nz)
    w = np.asarray(w).reshape(nx, ny, nz + 1)
    ad = [a] * 6
    if body is not None and np.any(body_masks(body, dims)[1]):
        # face areas times the cell's face fractions (pressure_update_rhs.cpp:
        # 34-43; an uncut fluid cell's are 1), then the branch below
        off, cut, fS = body_masks(body, dims)
        ad = [np.where(cut, a * fS[d], a) for d in range(6)]
        solid = off
    terms = [(1, ad[0] * u[:-1]), (-1, ad[1] * u[1:]), (1, ad[2] * v[:, :-1]), (-1, ad[3] * v[:, 1:]),
             (1, ad[4] * w[:, :, :-1]), (-1, ad[5] * w[:, :, 1:])]
    if solid is None or not np.any(solid):
        f = 0.0 + terms[0][1]
        for sign, t in terms[1:]:
            f = f + t if sign > 0 else f - t
        f = f + (0.0 + 0.0)
        return f.reshape(-1)
    sol = np.asarray(solid).reshape(dims).astype(bool)
    fluid = ~sol
    pad = np.pad(fluid, 1, constant_values=True)
    nb_open = [pad[:-2, 1:-1, 1:-1], pad[2:, 1:-1, 1:-1], pad[1:-1, :-2, 1:-1],
               pad[1:-1, 2:, 1:-1], pad[1:-1, 1:-1, :-2], pad[1:-1, 1:-1, 2:]]
    f = np.zeros(dims)
    for (sign, t), op_ in zip(terms, nb_open):
        g = f + t if sign > 0 else f - t
        f = np.where(op_, g, f)
    f = np.where(sol, 0.0, f)
    f = f + (0.0 + 0.0)
    return f.reshape(-1)


def project(dims, h, dt, p, col, rho_a, rho_b, u, v, w, solid=None):
    """Projected face velocities (new arrays, the layouts of pbg_gen_flow).
    solid: the immersed-body branch (momentum_project.cpp:47-73): only
    faces between two fluid cells, in the order (dp * dt) / rho / dxc."""
    nx, ny, nz = dims
    p = np.asarray(p).reshape(dims)
    rc = _cell_density(col, rho_a, rho_b, dims)
    u = np.array(u, dtype=np.float64).reshape(nx + 1, ny, nz)
    v = np.array(v, dtype=np.float64).reshape(nx, ny + 1, nz)
    w = np.array(w, dtype=np.float64).reshape(nx, ny, nz + 1)
    body = solid is not None and np.any(solid)
    fluid = ~np.asarray(solid).reshape(dims).astype(bool) if body else None

    def rface(axis, shape):
        if rc is None:
            return np.full(shape, float(rho_a))
        f = face_density(rc, axis)
        return np.take(f, np.arange(1, f.shape[axis] - 1), axis=axis)

    def incr(dp, rho):
        if body:
            return dp * dt / rho / h
        return dp / rho * dt / h

    ru = rface(0, (nx - 1, ny, nz))
    du = incr(p[:-1] - p[1:], ru)
    v_u = u[1:-1] + du
    u[1:-1] = np.where(fluid[:-1] & fluid[1:], v_u, u[1:-1]) if body else v_u
    rv = rface(1, (nx, ny - 1, nz))
    dv = incr(p[:, :-1] - p[:, 1:], rv)
    v_v = v[:, 1:-1] + dv
    v[:, 1:-1] = np.where(fluid[:, :-1] & fluid[:, 1:], v_v, v[:, 1:-1]) if body else v_v
    if nz > 1:
        rw = rface(2, (nx, ny, nz - 1))
        dw = incr(p[:, :, :-1] - p[:, :, 1:], rw)
        v_w = w[:, :, 1:-1] + dw
        w[:, :, 1:-1] = np.where(fluid[:, :, :-1] & fluid[:, :, 1:], v_w, w[:, :, 1:-1]) if body else v_w
    return u, v, w


class StepProblem:
    """An assembled pressure system in the shape oracle_py's solvers take."""

    def __init__(self, dims, h, A, b):
        self.nx, self.ny, self.nz = dims
        self.h = h
        self.N = self.nx * self.ny * self.nz
        self.A = {k: np.ascontiguousarray(A[k]) for k in "cwesnbt"}
        self.b = np.ascontiguousarray(b)

    @property
    def dims(self):
        return (self.nx, self.ny, self.nz)

    @property
    def dV(self):
        return self.h * self.h * self.h

    def mat(self):
        m = op.OrcMat(self.nx, self.ny, self.nz, *[op._p(self.A[k]) for k in "cwesnbt"])
        m._keep = self
        return m


def step(P, dt, res_rat=1e-10, maxit=20000, solver="cg", stream=0, bc=None, body=None):
    """One pressure-correction step: assemble, divergence, Krylov solve from
    p = 0 with scale dti (centered_solve.cpp:25-31), project. Returns a dict
    of A, b, x, u, v, w and the solver's statistics. body: dict fV, fS of a
    cut body (then P's voxel solid is not used)."""
    col, u, v, w, ra, rb, bc0 = flow_state(P, stream)
    bc = list(bc0 if bc is None else bc)
    sol = P.solid if np.any(P.solid) else None
    if body is not None:
        off, cut, _ = body_masks(body, P.dims)
        sol = off.reshape(-1) if np.any(cut) else None
    A = assemble_mix(P.dims, P.h, bc, col, ra, rb, solid=sol, body=body)
    b = divergence(P.dims, P.h, dt, u, v, w, solid=sol, body=body)
    sp = StepProblem(P.dims, P.h, A, b)
    x, st = op.cg(sp, b=b, res_rat=res_rat, res_tol=1e-18, maxit=maxit, scale=1.0 / dt,
                  solver=solver)
    un, vn, wn = project(P.dims, P.h, dt, x, col, ra, rb, u, v, w, solid=sol)
    return dict(A=A, b=b, x=x, u=un, v=vn, w=wn, stats=st, col=col, u0=u, v0=v, w0=w,
                rho=(ra, rb), bc=bc)


def run_reference_step(P, dt, res_rat=1e-10, maxit=20000, solver="cg", timeout=600, body=0.0):
    """The compiled reference's own step (ref_harness --step 1) on P's
    workload: dict of A, b, x, u, v, w and the harness summary. body > 0: a
    sphere of that radius in cells, cut by the reference's Body; its fV and
    fS come back as well."""
    import os
    import shutil
    import subprocess
    import tempfile
    a = P.args
    kind = {op.KIND_SINGLE: "single", op.KIND_CYL: "cyl", op.KIND_BATCH: "batch"}[P.kind]
    tmp = tempfile.mkdtemp(prefix="pbg_step_")
    try:
        out = os.path.join(tmp, "ref")
        cmd = [op.HARNESS, "--kind", kind, "--n", str(a["n"]), "--nb", str(a["nb"]),
               "--rmin", repr(a["rmin"]), "--rmax", repr(a["rmax"]), "--rc", repr(a["rc"]),
               "--ratio", repr(a["ratio"]), "--index", str(a["index"]), "--n2d", str(a["n2d"]),
               "--s2", str(a["s2"][0]), str(a["s2"][1]), "--s3", str(a["s3"][0]),
               str(a["s3"][1]), "--seed", str(P.seed), "--solver", solver,
               "--resrat", repr(res_rat), "--maxit", str(maxit), "--step", "1",
               "--dt", repr(dt), "--out", out, "--body", repr(float(body))]
        subprocess.run(cmd, check=True, capture_output=True, timeout=timeout)
        meta = {}
        for line in open(out + ".txt"):
            parts = line.split()
            if len(parts) >= 2:
                meta[parts[0]] = parts[1] if parts[0] == "solver" else float(parts[1])
        nx, ny, nz = P.dims
        N = P.N
        A = np.fromfile(out + ".A", dtype=np.float64).reshape(8, N)
        res = dict(meta=meta, A={k: A[q] for q, k in enumerate("cwesnbt")}, ci=A[7],
                   b=np.fromfile(out + ".b", dtype=np.float64),
                   x=np.fromfile(out + ".x", dtype=np.float64),
                   u=np.fromfile(out + ".u", dtype=np.float64).reshape(nx + 1, ny, nz),
                   v=np.fromfile(out + ".v", dtype=np.float64).reshape(nx, ny + 1, nz),
                   w=np.fromfile(out + ".w", dtype=np.float64).reshape(nx, ny, nz + 1))
        if body > 0.0:
            bd = np.fromfile(out + ".body", dtype=np.float64).reshape(8, N)
            res["body"] = dict(fV=bd[0].copy(), fS=bd[1:7].copy(), listed=bd[7].copy())
        return res
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
