"""ctypes binding of the C oracle (oracle.c) and of the reference harness.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
the CPU-baseline leg of bench.py, as the checker. The engine never imports
it.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(BUILD, "liboracle.so")
HARNESS = os.path.join(HERE, "_ref", "ref_harness")
PROBLEM_GEN_DIR = os.path.join(os.path.dirname(HERE), "psiboil_b200", "csrc")

_dp = ctypes.POINTER(ctypes.c_double)


def build():
    """Compile oracle.c into oracle/_build/liboracle.so (gcc, IEEE, no FMA)."""
    os.makedirs(BUILD, exist_ok=True)
    src = [os.path.join(HERE, "oracle.c"), os.path.join(HERE, "oracle_gen.c")]
    hdr = [os.path.join(HERE, "oracle.h"), os.path.join(PROBLEM_GEN_DIR, "problem_gen.h")]
    if os.path.exists(LIB) and os.path.getmtime(LIB) >= max(os.path.getmtime(p) for p in src + hdr):
        return LIB
    subprocess.check_call(["gcc", "-O2", "-std=c99", "-fPIC", "-shared", "-ffp-contract=off",
                           "-I", PROBLEM_GEN_DIR, "-o", LIB] + src + ["-lm"])
    return LIB


class OrcMat(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int)] + \
               [(k, _dp) for k in "cwesnbt"] + [("per", ctypes.c_int)]


class OrcStats(ctypes.Structure):
    _fields_ = [("converged", ctypes.c_int), ("iterations", ctypes.c_int),
                ("printed", ctypes.c_int), ("res0", ctypes.c_double),
                ("res", ctypes.c_double), ("status", ctypes.c_int)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB)
        L.orc_spmv.argtypes = [ctypes.POINTER(OrcMat), _dp, _dp]
        L.orc_resid.argtypes = [ctypes.POINTER(OrcMat), _dp, _dp, _dp]
        L.orc_dot.restype = ctypes.c_double
        L.orc_dot.argtypes = [ctypes.c_size_t, _dp, _dp]
        L.orc_dot_voldiv_avg.restype = ctypes.c_double
        L.orc_dot_voldiv_avg.argtypes = [ctypes.c_size_t, _dp, _dp, ctypes.c_double]
        for fn in (L.orc_cg, L.orc_bicgs, L.orc_cg_prec, L.orc_bicgs_prec, L.orc_cgs_prec):
            fn.restype = ctypes.c_int
            fn.argtypes = [ctypes.POINTER(OrcMat), _dp, _dp, ctypes.c_int, ctypes.c_int,
                           ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                           ctypes.c_double, ctypes.POINTER(OrcStats), _dp]
        for fn in (L.orc_cg_prec, L.orc_bicgs_prec, L.orc_cgs_prec):
            fn.argtypes = fn.argtypes + [ctypes.c_int]
        L.orc_jacobi.restype = ctypes.c_int
        L.orc_jacobi.argtypes = [ctypes.POINTER(OrcMat), _dp, _dp, _dp, ctypes.c_int, ctypes.c_int,
                                 ctypes.c_double, ctypes.c_double, ctypes.POINTER(OrcStats), _dp]
        L.orc_gauss_seidel.restype = ctypes.c_int
        L.orc_gauss_seidel.argtypes = [ctypes.POINTER(OrcMat), _dp, _dp, _dp, ctypes.c_int,
                                       ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                       ctypes.c_double, ctypes.c_int, ctypes.c_double,
                                       ctypes.POINTER(OrcStats), _dp]
        L.orc_ac_create.restype = ctypes.c_void_p
        L.orc_ac_create.argtypes = [ctypes.POINTER(OrcMat), ctypes.c_void_p, ctypes.c_double]
        L.orc_ac_destroy.argtypes = [ctypes.c_void_p]
        L.orc_ac_set_smoother.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _dp]
        L.orc_ac_set_params.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                        ctypes.c_int, ctypes.c_int]
        L.orc_ac_flex_capped.restype = ctypes.c_int
        L.orc_ac_flex_capped.argtypes = [ctypes.c_void_p]
        L.orc_ac_set_flex_cap.argtypes = [ctypes.c_void_p, ctypes.c_longlong]
        L.orc_ac_nlevels.restype = ctypes.c_int
        L.orc_ac_nlevels.argtypes = [ctypes.c_void_p]
        L.orc_ac_level_dims.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
        L.orc_ac_coarsen_all.argtypes = [ctypes.c_void_p]
        L.orc_ac_level_matrix.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp]
        L.orc_ac_cycle.restype = ctypes.c_int
        L.orc_ac_cycle.argtypes = [ctypes.c_void_p, _dp, _dp, ctypes.c_int, ctypes.c_int,
                                   ctypes.c_double, ctypes.c_double,
                                   ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                   ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                   ctypes.POINTER(ctypes.c_int), _dp, ctypes.POINTER(ctypes.c_int)]
        L.orc_gen_problem.restype = ctypes.c_int
        L.orc_gen_problem.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_uint64,
                                      ctypes.c_void_p, ctypes.c_void_p, _dp, _dp]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(_dp)


# ---------------------------------------------------------------- problems

KIND_SINGLE, KIND_CYL, KIND_BATCH = 0, 1, 2


class Problem:
    """A seeded fixture problem: dims, density, solid mask, rhs, matrix."""

    def __init__(self, kind, seed, n=16, nb=0, rmin=4.0, rmax=16.0, rc=0.0, ratio=1000.0,
                 index=0, n2d=0, s2=(64, 512), s3=(32, 96), stream=0, convect=0.0, periodic=0):
        """periodic: axes with periodic boundaries (bit 0 i, 1 j, 2 k)."""
        self.kind, self.seed = kind, seed
        self.periodic = int(periodic)
        params = np.array([n, nb, rmin, rmax, rc, ratio, index, n2d, s2[0], s2[1], s3[0], s3[1],
                           stream, self.periodic], dtype=np.float64)
        dims = np.zeros(3, dtype=np.int32)
        hb = np.zeros(2, dtype=np.float64)  # h, rho ratio
        L = lib()
        # first call: dimensions only
        L.orc_gen_problem(kind, params.ctypes.data, seed, dims.ctypes.data, None, _p(hb), None)
        self.nx, self.ny, self.nz = (int(v) for v in dims)
        self.h = float(hb[0])
        N = self.nx * self.ny * self.nz
        self.N = N
        self.args = dict(n=n, nb=nb, rmin=rmin, rmax=rmax, rc=rc, ratio=ratio, index=index,
                         n2d=n2d, s2=s2, s3=s3, periodic=self.periodic)
        out = np.zeros(10 * N, dtype=np.float64)  # rho, rhs, c,w,e,s,n,b,t,ci
        solid = np.zeros(N, dtype=np.uint8)
        L.orc_gen_problem(kind, params.ctypes.data, seed, dims.ctypes.data, solid.ctypes.data,
                          _p(hb), _p(out))
        self.rho = out[0:N].copy()
        self.b = out[N:2 * N].copy()
        self.A = {k: out[(2 + q) * N:(3 + q) * N].copy() for q, k in enumerate("cwesnbt")}
        self.ci = out[9 * N:10 * N].copy()
        self.solid = solid
        self.bc = None
        self.convect = float(convect)
        if self.convect != 0.0:
            # upwind convection along +x: a non-symmetric matrix (pbg_gen_convect)
            L.orc_convect.argtypes = [ctypes.c_int] * 3 + [ctypes.c_double, ctypes.c_void_p, _dp, _dp, _dp]
            L.orc_convect(self.nx, self.ny, self.nz, self.convect, solid.ctypes.data, _p(self.A["c"]),
                          _p(self.A["w"]), _p(self.ci))

    @property
    def dims(self):
        return (self.nx, self.ny, self.nz)

    @property
    def dV(self):
        return self.h * self.h * self.h

    def mat(self):
        m = OrcMat(self.nx, self.ny, self.nz, *[_p(self.A[k]) for k in "cwesnbt"], self.periodic)
        m._keep = self
        return m


# ---------------------------------------------------------------- kernels

def spmv(P, x):
    y = np.zeros_like(x)
    m = P.mat()
    lib().orc_spmv(ctypes.byref(m), _p(x), _p(y))
    return y


def resid(P, x, b):
    r = np.zeros_like(x)
    m = P.mat()
    lib().orc_resid(ctypes.byref(m), _p(x), _p(b), _p(r))
    return r


def dot(x, y):
    return lib().orc_dot(x.size, _p(x), _p(y))


def dot_voldiv_avg(x, y, dV):
    return lib().orc_dot_voldiv_avg(x.size, _p(x), _p(y), dV)


PRECS = {"di": 0, "ic0": 1, "ic2": 2, "ic3": 3}


def cg(P, b=None, x0=None, mini=1, maxit=20000, res_rat=1e-8, res_tol=1e-18, scale=1.0,
       stalecount=-1, hist=False, solver="cg", prec="di"):
    b = P.b if b is None else b
    x = np.zeros(P.N) if x0 is None else x0.copy()
    st = OrcStats()
    h = np.zeros(maxit + 1) if hist else None
    m = P.mat()
    args = (ctypes.byref(m), _p(x), _p(b), mini, maxit, res_rat, res_tol, scale, stalecount, P.dV,
            ctypes.byref(st), _p(h) if hist else None)
    if solver == "jacobi":  # Jacobi::solve: no scale, no stale window, |r| = sqrt(r.r)
        ci = np.ascontiguousarray(P.ci, dtype=np.float64)
        lib().orc_jacobi(ctypes.byref(m), _p(ci), _p(x), _p(b), mini, maxit, res_rat, res_tol,
                         ctypes.byref(st), _p(h) if hist else None)
    elif solver == "gs":
        ci = np.ascontiguousarray(P.ci, dtype=np.float64)
        lib().orc_gauss_seidel(ctypes.byref(m), _p(ci), _p(x), _p(b), mini, maxit, res_rat,
                               res_tol, scale, stalecount, P.dV, ctypes.byref(st),
                               _p(h) if hist else None)
    else:
        fn = {"cg": lib().orc_cg_prec, "bicgs": lib().orc_bicgs_prec,
              "cgs": lib().orc_cgs_prec}[solver]
        fn(*args, PRECS[prec])
    out = dict(converged=st.converged, iterations=st.iterations, printed=st.printed,
               res0=st.res0, res=st.res, status=st.status)
    if hist:
        out["hist"] = h[:st.iterations].copy()
    return x, out


class AC:
    """Oracle AC hierarchy for one problem (reference coarsening rule)."""

    SMOOTHERS = {"cg": 0, "bicgs": 1, "cgs": 2, "jacobi": 3, "gs": 4}

    def __init__(self, P, smoother="cg", prec="di", solver=None, solver_prec="di", resrat=1e-18,
                 restol=1e-18, use_linf=False, flex_cap=1000000):
        """smoother: the levels' solver (the Pressure's Linear); solver: AC's
        own solver for call_solver (AC(cen, sol)), None for the same;
        resrat/restol: AC::resrat/restol; use_linf: AC::use_linf_error."""
        self.P = P
        aflag = (1 - P.solid).astype(np.uint8)
        self._aflag = aflag
        m = P.mat()
        self._m = m
        self.h = lib().orc_ac_create(ctypes.byref(m), aflag.ctypes.data, P.h)
        self._ci = np.ascontiguousarray(P.ci, dtype=np.float64)  # level 0's stored ci
        if smoother != "cg" or prec != "di":
            lib().orc_ac_set_smoother(self.h, self.SMOOTHERS[smoother], PRECS[prec], _p(self._ci))
        elif solver in ("jacobi", "gs"):
            lib().orc_ac_set_smoother(self.h, 0, 0, _p(self._ci))
        lib().orc_ac_set_params(self.h, resrat, restol, int(use_linf),
                                -1 if solver is None else self.SMOOTHERS[solver], PRECS[solver_prec])
        lib().orc_ac_set_flex_cap(self.h, int(flex_cap))

    @property
    def flex_capped(self):
        return bool(lib().orc_ac_flex_capped(self.h))

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_ac_destroy(self.h)
            self.h = None

    @property
    def nlevels(self):
        return lib().orc_ac_nlevels(self.h)

    def level_dims(self, l):
        d = (ctypes.c_int * 3)()
        lib().orc_ac_level_dims(self.h, l, d)
        return tuple(d)

    def level_matrix(self, l):
        lib().orc_ac_coarsen_all(self.h)
        nx, ny, nz = self.level_dims(l)
        n = nx * ny * nz
        out = np.zeros(7 * n)
        lib().orc_ac_level_matrix(self.h, l, _p(out))
        return {k: out[q * n:(q + 1) * n].copy() for q, k in enumerate("cwesnbt")}

    def cycle(self, b=None, x0=None, init=-1, loop=1, toler=-1.0, factor=1e-8, mv=(20, 20, 20),
              ms=(-1, -1, -1), max_cyc=20, min_cyc=0, stop_if_div=1, priority_min_cyc=1):
        P = self.P
        b = P.b if b is None else b
        x = np.zeros(P.N) if x0 is None else x0.copy()
        mv_ = (ctypes.c_int * 3)(*mv)
        ms_ = (ctypes.c_int * 3)(*ms)
        ncyc = ctypes.c_int(0)
        nh = ctypes.c_int(0)
        hist = np.zeros(max_cyc + 4)
        ok = lib().orc_ac_cycle(self.h, _p(x), _p(b), init, loop, toler, factor, mv_, ms_,
                                max_cyc, min_cyc, stop_if_div, priority_min_cyc,
                                ctypes.byref(ncyc), _p(hist), ctypes.byref(nh))
        return x, dict(converged=ok, cycles=ncyc.value, hist=hist[:nh.value].copy())


# ---------------------------------------------------------------- reference harness

def harness_available():
    return os.path.exists(HARNESS)


def run_reference(P, solver="cg", resrat=1e-8, maxit=20000, maxcyc=20, guard=1, cycle="V",
                  out_prefix=None, dump=True, timeout=3600, prec="di", acsm="cg", init="none",
                  acsolver=None, linf=0, acresrat=None, mincyc=0):
    """Run the compiled reference on P's fixture; returns (meta, arrays)."""
    import tempfile
    kind = {KIND_SINGLE: "single", KIND_CYL: "cyl", KIND_BATCH: "batch"}[P.kind]
    a = P.args
    tmp = None
    if out_prefix is None:
        tmp = tempfile.mkdtemp(prefix="pbg_ref_")
        out_prefix = os.path.join(tmp, "ref")
    cmd = [HARNESS, "--kind", kind, "--n", str(a["n"]), "--nb", str(a["nb"]),
           "--rmin", repr(a["rmin"]), "--rmax", repr(a["rmax"]), "--rc", repr(a["rc"]),
           "--ratio", repr(a["ratio"]), "--index", str(a["index"]), "--n2d", str(a["n2d"]),
           "--s2", str(a["s2"][0]), str(a["s2"][1]), "--s3", str(a["s3"][0]), str(a["s3"][1]),
           "--seed", str(P.seed), "--solver", solver, "--resrat", repr(resrat),
           "--maxit", str(maxit), "--maxcyc", str(maxcyc), "--guard", str(guard),
           "--cycle", cycle, "--prec", prec, "--dump", "1" if dump else "0", "--out", out_prefix,
           "--convect", repr(getattr(P, "convect", 0.0)), "--acsm", acsm,
           "--periodic", str(getattr(P, "periodic", 0)), "--init", init, "--linf", str(int(linf)),
           "--mincyc", str(mincyc)]
    if acsolver:
        cmd += ["--acsolver", acsolver]
    if acresrat is not None:
        cmd += ["--acresrat", repr(acresrat)]
    subprocess.run(cmd, check=True, capture_output=True, timeout=timeout)
    meta = {}
    for line in open(out_prefix + ".txt"):
        parts = line.split()
        if not parts:
            continue
        k, v = parts[0], parts[1:]
        if k == "cycle_res":
            meta[k] = [float(t) for t in v]
        elif k in ("solver",):
            meta[k] = v[0]
        else:
            meta[k] = float(v[0]) if v else None
    arrays = None
    if dump:
        N = P.N
        A = np.fromfile(out_prefix + ".A", dtype=np.float64).reshape(8, N)
        arrays = dict(A={k: A[q] for q, k in enumerate("cwesnbt")}, ci=A[7],
                      b=np.fromfile(out_prefix + ".b", dtype=np.float64),
                      x=np.fromfile(out_prefix + ".x", dtype=np.float64))
    if tmp:
        import shutil
        shutil.rmtree(tmp, ignore_errors=True)
    return meta, arrays
