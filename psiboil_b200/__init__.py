"""psiboil_b200 — B200-native pressure-Poisson engine for PSI-BOIL.

Host-side mirror of the reference's solver interface over the engine's C ABI
(include/psiboil_b200.h). The reference's swap points are C++ virtuals; this
module keeps their names, argument meaning and return values:

  CG(sess).solve(A, x, b, MinIter, MaxIter, name, ResRat, ResTol, scale,
                 stalecount) -> bool     Linear::solve, Src/Solver/Linear/linear.h:46-56
  BiCGS(sess).solve(...)                 BiCGS::solve,  Krylov/bicgs.cpp:9-229
  AC(sess).vcycle(ResRat, ...) -> bool   AC::vcycle,    Src/Solver/Additive/additive.h:54-95
  Engine(sess).solve(x, b, tol, precision)   the engine's flexible-CG + AC K-cycle

Arrays are numpy arrays (host) or CUDA tensors (device, e.g. torch) in the
compact layout index (i*ny + j)*nz + k; the strided entry points accept the
reference's BW=3 Scalar blocks. Every compute call runs the CUDA library; if
it cannot be loaded, importing a solver raises — there is no CPU fallback.
"""
import ctypes
import functools
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libpsiboil_b200.so")

PBG_OK = 0
ERR_ARG, ERR_CUDA, ERR_STATE, ERR_NOMEM, ERR_UNSUPPORTED, ERR_ADMISSION = -1, -2, -3, -4, -5, -6
HOST, DEVICE = 0, 1
NEUMANN, DIRICHLET, PERIODIC = 0, 1, 2   # boundary types; PERIODIC goes on both faces of an axis
SOLVER_CG, SOLVER_BICGS, SOLVER_AC, SOLVER_ENGINE, SOLVER_CGS = 0, 1, 2, 3, 4
SOLVER_JACOBI, SOLVER_GAUSS_SEIDEL = 5, 6
# pbg_result.status
CONVERGED, MAXITER, STALE, BREAKDOWN, INITIAL, NAN, DIVERGED = 0, 1, 2, 3, 4, 5, 6
FP64, MIXED = 0, 1
CYCLE_NONE, CYCLE_V, CYCLE_F, CYCLE_W, CYCLE_FLEX = -1, 1, 2, 4, 5
STATUS = {0: "converged", 1: "maxiter", 2: "stale", 3: "breakdown", 4: "initial", 5: "nan",
          6: "diverged"}

_dp = ctypes.POINTER(ctypes.c_double)
_vp = ctypes.c_void_p
_ll = ctypes.c_longlong


class PbgError(RuntimeError):
    """A C-ABI call returned an error status."""

    def __init__(self, code, msg):
        super().__init__("pbg error %d: %s" % (code, msg))
        self.code = code


class Params(ctypes.Structure):
    _fields_ = [("solver", ctypes.c_int), ("precision", ctypes.c_int),
                ("min_iter", ctypes.c_int), ("max_iter", ctypes.c_int),
                ("res_rat", ctypes.c_double), ("res_tol", ctypes.c_double),
                ("scale", ctypes.c_double), ("stalecount", ctypes.c_int),
                ("init_cycle", ctypes.c_int), ("loop_cycle", ctypes.c_int),
                ("toler", ctypes.c_double), ("factor", ctypes.c_double),
                ("max_cycles", ctypes.c_int), ("min_cycles", ctypes.c_int),
                ("stop_if_div", ctypes.c_int), ("priority_min_cyc", ctypes.c_int),
                ("mv", ctypes.c_int * 3), ("ms", ctypes.c_int * 3),
                ("tol", ctypes.c_double), ("inner_tol", ctypes.c_double),
                ("max_sweeps", ctypes.c_int), ("exact_sums", ctypes.c_int),
                ("coarse_max", ctypes.c_int), ("prec", ctypes.c_int), ("x0_zero", ctypes.c_int),
                ("ac_smoother", ctypes.c_int), ("ac_solver", ctypes.c_int), ("ac_solver_prec", ctypes.c_int),
                ("ac_resrat", ctypes.c_double), ("ac_restol", ctypes.c_double), ("use_linf", ctypes.c_int),
                ("flex_visits", ctypes.c_int), ("ac_dt", ctypes.c_double)]


class Result(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("converged", ctypes.c_int),
                ("iterations", ctypes.c_int), ("cycles", ctypes.c_int),
                ("sweeps", ctypes.c_int), ("levels", ctypes.c_int),
                ("res0", ctypes.c_double), ("res", ctypes.c_double),
                ("relres", ctypes.c_double), ("seconds", ctypes.c_double)]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_}
        d["status_name"] = STATUS.get(self.status, str(self.status))
        return d


# exported symbols and their argument types
_SIGS = {
    "pbg_last_error": (ctypes.c_char_p, []),
    "pbg_version": (ctypes.c_int, []),
    "pbg_device_count": (ctypes.c_int, [ctypes.POINTER(ctypes.c_int)]),
    "pbg_params_default": (None, [ctypes.POINTER(Params), ctypes.c_int]),
    "pbg_session_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                          ctypes.POINTER(ctypes.c_int), ctypes.c_int,
                                          ctypes.POINTER(_vp)]),
    "pbg_session_destroy": (ctypes.c_int, [_vp]),
    "pbg_session_info": (ctypes.c_int, [_vp, ctypes.POINTER(_ll), ctypes.POINTER(ctypes.c_int),
                                        ctypes.POINTER(_ll)]),
    "pbg_session_set_cell_volume": (ctypes.c_int, [_vp, ctypes.c_double]),
    "pbg_matrix_upload": (ctypes.c_int, [_vp] + [_vp] * 7 + [_ll, _ll, _ll, _ll, ctypes.c_int]),
    "pbg_matrix_download": (ctypes.c_int, [_vp] + [_vp] * 7 + [ctypes.c_int]),
    "pbg_active_upload": (ctypes.c_int, [_vp, _vp, _ll, _ll, _ll, _ll, ctypes.c_int]),
    "pbg_ci_upload": (ctypes.c_int, [_vp, _vp, _ll, _ll, _ll, _ll, ctypes.c_int]),
    "pbg_body_upload": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int]),
    "pbg_assemble_pressure": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int]),
    "pbg_assemble_mix": (ctypes.c_int, [_vp, _vp, ctypes.c_double, ctypes.c_double, _vp, ctypes.c_int]),
    "pbg_divergence": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, ctypes.c_double, _vp, ctypes.c_int]),
    "pbg_project": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_double, ctypes.c_double, _vp, ctypes.c_double,
                                   _vp, _vp, _vp, ctypes.c_int]),
    "pbg_pressure_step": (ctypes.c_int, [_vp, _vp, ctypes.c_double, ctypes.c_double, _vp, ctypes.c_double,
                                         _vp, _vp, _vp, _vp, ctypes.c_int, ctypes.POINTER(Params),
                                         ctypes.POINTER(Result)]),
    "pbg_generate_flow": (ctypes.c_int, [ctypes.c_int, _dp, ctypes.c_uint64, _vp, _vp, _vp, _vp, _dp]),
    "pbg_solve": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int, ctypes.POINTER(Params),
                                 ctypes.POINTER(Result)]),
    "pbg_solve_strided": (ctypes.c_int, [_vp, _vp, _vp, _ll, _ll, _ll, _ll, ctypes.c_int,
                                         ctypes.POINTER(Params), ctypes.POINTER(Result)]),
    "pbg_history": (ctypes.c_int, [_vp, _dp, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]),
    "pbg_spmv": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int]),
    "pbg_residual": (ctypes.c_int, [_vp, _vp, _vp, _vp, ctypes.c_int]),
    "pbg_dot": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int, _dp]),
    "pbg_seq_sum": (ctypes.c_int, [_vp, _vp, _vp, _ll, ctypes.c_int, _dp]),
    "pbg_levels": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                  ctypes.POINTER(ctypes.c_int), ctypes.c_int]),
    "pbg_ac_level_matrix": (ctypes.c_int, [_vp, ctypes.c_int, _vp, ctypes.c_int]),
    "pbg_launch_count": (ctypes.c_ulonglong, []),
    "pbg_session_stream": (ctypes.c_int, [_vp, ctypes.POINTER(_vp)]),
    "pbg_bench_kernel": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp, _dp]),
    "pbg_dot_noalloc": (ctypes.c_int, [_vp, _vp, _ll, ctypes.c_double, _vp, _vp]),
    "pbg_generate": (ctypes.c_int, [ctypes.c_int, _dp, ctypes.c_uint64, ctypes.POINTER(ctypes.c_int),
                                    _dp, _vp, _vp, _vp]),
}


class BatchConfig(ctypes.Structure):
    _fields_ = [("precision", ctypes.c_int), ("slots", ctypes.c_int), ("threads", ctypes.c_int),
                ("tile_cells", ctypes.c_int), ("grid", ctypes.c_int), ("kc_max", ctypes.c_int),
                ("tail_cells", ctypes.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_BCP = ctypes.POINTER(BatchConfig)
_SIGS.update({
    "pbg_batch_config_default": (None, [_BCP]),
    "pbg_batch_create": (ctypes.c_int, [_BCP, ctypes.c_int, ctypes.POINTER(_vp)]),
    "pbg_batch_destroy": (ctypes.c_int, [_vp]),
    "pbg_batch_problem_bytes": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                               ctypes.POINTER(_ll)]),
    "pbg_batch_add": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                     ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]),
    "pbg_batch_remove": (ctypes.c_int, [_vp, ctypes.c_int]),
    "pbg_batch_set_fields": (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp, ctypes.c_int]),
    "pbg_batch_set_rhs": (ctypes.c_int, [_vp, ctypes.c_int, _vp, ctypes.c_int]),
    "pbg_batch_set_x": (ctypes.c_int, [_vp, ctypes.c_int, _vp, ctypes.c_int]),
    "pbg_batch_get_x": (ctypes.c_int, [_vp, ctypes.c_int, _vp, ctypes.c_int]),
    "pbg_batch_solve": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_int), ctypes.c_int,
                                       ctypes.POINTER(Params), ctypes.POINTER(Result)]),
    "pbg_batch_autotune": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_int), ctypes.c_int,
                                          ctypes.POINTER(Params), ctypes.c_char_p, _BCP]),
})


class ServerConfig(ctypes.Structure):
    _fields_ = [("precision", ctypes.c_int), ("slots", ctypes.c_int), ("hbm_budget", ctypes.c_longlong),
                ("iters_per_poll", ctypes.c_int), ("threads", ctypes.c_int), ("tile_cells", ctypes.c_int),
                ("grid", ctypes.c_int), ("kc_max", ctypes.c_int), ("tail_cells", ctypes.c_int),
                ("tol", ctypes.c_double),
                ("inner_tol", ctypes.c_double), ("max_sweeps", ctypes.c_int), ("max_iter", ctypes.c_int)]


class ServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_longlong), ("completed", ctypes.c_longlong),
                ("queued", ctypes.c_longlong), ("in_flight", ctypes.c_longlong),
                ("sessions", ctypes.c_longlong), ("device_bytes", ctypes.c_longlong),
                ("kernel_launches", ctypes.c_ulonglong)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_SCP = ctypes.POINTER(ServerConfig)
_SIGS.update({
    "pbg_server_config_default": (None, [_SCP]),
    "pbg_server_create": (ctypes.c_int, [_SCP, ctypes.c_int, ctypes.POINTER(_vp)]),
    "pbg_server_destroy": (ctypes.c_int, [_vp]),
    "pbg_server_open_session": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                               ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]),
    "pbg_server_close_session": (ctypes.c_int, [_vp, ctypes.c_int]),
    "pbg_server_submit": (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp, _vp, ctypes.c_int, ctypes.POINTER(_ll)]),
    "pbg_server_submit_bubble": (ctypes.c_int, [_vp, ctypes.c_int, _dp, ctypes.c_double, ctypes.c_double,
                                                ctypes.c_ulonglong, ctypes.POINTER(_ll)]),
    "pbg_server_wait": (ctypes.c_int, [_vp, _ll, ctypes.c_double, ctypes.POINTER(Result), _dp]),
    "pbg_server_get_x": (ctypes.c_int, [_vp, ctypes.c_int, _vp, ctypes.c_int]),
    "pbg_server_stats_get": (ctypes.c_int, [_vp, ctypes.POINTER(ServerStats)]),
})

_PP = ctypes.POINTER(ctypes.c_void_p)
_SIGS.update({
    "pbg_bck_name": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_char_p, ctypes.c_int]),
    "pbg_bck_write": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, _PP, ctypes.c_int, ctypes.c_int,
                                     ctypes.c_int, ctypes.c_int]),
    "pbg_bck_read": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, _PP, ctypes.c_int, ctypes.c_int,
                                    ctypes.c_int, ctypes.c_int]),
    "pbg_bck_write_compact": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, _PP, ctypes.c_int, ctypes.c_int,
                                             ctypes.c_int, ctypes.c_int]),
    "pbg_bck_read_compact": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, _PP, ctypes.c_int, ctypes.c_int,
                                            ctypes.c_int, ctypes.c_int]),
})

_lib = None


def lib():
    """Load the CUDA library (raises if it is missing: no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("psiboil_b200: %s not built (run __graft_entry__.build())" % LIB_PATH)
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _check(code):
    if code != PBG_OK:
        raise PbgError(code, lib().pbg_last_error().decode())


def _ptr(a, dtype="float64"):
    """(pointer, where) of a numpy array or a CUDA tensor of the given dtype,
    C-contiguous; anything else raises before it reaches the library."""
    if a is None:
        return None, HOST
    if hasattr(a, "data_ptr") and hasattr(a, "is_cuda"):
        if not a.is_cuda:
            raise TypeError("tensors must be CUDA tensors (use numpy arrays for host memory)")
        if str(a.dtype) != "torch." + dtype:
            raise TypeError("expected a torch.%s tensor, got %s" % (dtype, a.dtype))
        if not a.is_contiguous():
            raise ValueError("tensors must be contiguous")
        return a.data_ptr(), DEVICE
    if isinstance(a, np.ndarray):
        if not a.flags["C_CONTIGUOUS"]:
            raise ValueError("arrays must be C-contiguous")
        if a.dtype != np.dtype(dtype):
            raise TypeError("expected a %s array, got %s" % (dtype, a.dtype))
        return a.ctypes.data, HOST
    raise TypeError("expected a numpy array or a CUDA tensor, got %r" % type(a))


def _ptrn(a, n, dtype="float64"):
    """_ptr that also requires at least n elements (the compact layout)."""
    p = _ptr(a, dtype)
    if a is not None:
        size = a.numel() if hasattr(a, "numel") else a.size
        if size < n:
            raise ValueError("array holds %d elements, %d needed" % (size, n))
    return p


def default_params(solver):
    p = Params()
    lib().pbg_params_default(ctypes.byref(p), solver)
    return p


def dot_noalloc(x, y, dV, out, stream=None):
    """pbg_dot_noalloc on CUDA tensors: out (2 doubles, device) = (x.y,
    sum x*y/dV/dV / n / n); allocates nothing.

    x, y and out must be contiguous float64 CUDA tensors on the current
    device; anything else raises here instead of reaching the kernel."""
    import torch
    dev = torch.cuda.current_device()
    for name, t in (("x", x), ("y", y), ("out", out)):
        _ptr(t)
        if t.device.index != dev:
            raise ValueError("%s is on cuda:%s, the current device is cuda:%d" % (name, t.device.index, dev))
    n = x.numel()
    if y.numel() != n or out.numel() < 2:
        raise ValueError("x and y must have the same length, out at least 2")
    h = stream.cuda_stream if stream is not None else None
    _check(lib().pbg_dot_noalloc(x.data_ptr(), y.data_ptr(), n, dV, out.data_ptr(), h))
    return out


def launch_count():
    return int(lib().pbg_launch_count())


def device_count():
    n = ctypes.c_int(0)
    rc = lib().pbg_device_count(ctypes.byref(n))
    return n.value if rc == PBG_OK else 0


def _first_cuda_tensor(values):
    for a in values:
        if isinstance(a, dict):
            t = _first_cuda_tensor(a.values())
            if t is not None:
                return t
        elif getattr(a, "is_cuda", False) and hasattr(a, "data_ptr"):
            return a
    return None


def _stream_ordered(fn):
    """For Session methods that take CUDA tensors. torch wrote those tensors
    on its current stream; the library works on the session's own
    (non-blocking) stream. So the session's stream first waits for torch's
    current stream, and torch's current stream then waits for the session's:
    the call sees the tensors' values, and later torch work sees its
    results. Nothing is done when the session's stream is the current one
    (work issued inside `torch.cuda.stream(ExternalStream(stream_handle()))`)."""
    @functools.wraps(fn)
    def wrap(self, *args, **kw):
        t = _first_cuda_tensor(list(args) + list(kw.values()))
        if t is None:
            return fn(self, *args, **kw)
        import torch
        cur = torch.cuda.current_stream(t.device)
        h = self.stream_handle()
        if cur.cuda_stream == h:
            return fn(self, *args, **kw)
        own = torch.cuda.ExternalStream(h, device=t.device)
        own.wait_stream(cur)
        out = fn(self, *args, **kw)
        cur.wait_stream(own)
        return out
    return wrap


def _inputs_ready(fn):
    """For batch and server calls that take CUDA tensors: those copy or read
    device inputs on the library's own streams, which torch's stream does
    not order; the host first waits for the work torch has queued, so the
    tensors hold their values when the library reads them."""
    @functools.wraps(fn)
    def wrap(self, *args, **kw):
        t = _first_cuda_tensor(list(args) + list(kw.values()))
        if t is not None:
            import torch
            torch.cuda.current_stream(t.device).synchronize()
        return fn(self, *args, **kw)
    return wrap


class Session:
    """One grid, its matrix, hierarchies and scratch on one GPU.

    Stands in for the reference's Centered/Pressure equation object that owns
    A, phi, fnew and aflag (Src/Equation/Centered/centered.h:62-200).
    """

    def __init__(self, nx, ny, nz, h, bc=None, device=0):
        if bc is None:
            bc = [NEUMANN] * 6
            bc[5 if nz > 1 else 3] = DIRICHLET
        self.dims = (int(nx), int(ny), int(nz))
        self.h = float(h)
        self.bc = list(bc)
        self.device = device
        arr = (ctypes.c_int * 6)(*bc)
        hnd = _vp()
        _check(lib().pbg_session_create(nx, ny, nz, h, arr, device, ctypes.byref(hnd)))
        self._h = hnd

    @property
    def ncell(self):
        return self.dims[0] * self.dims[1] * self.dims[2]

    def close(self):
        if getattr(self, "_h", None):
            lib().pbg_session_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- matrix -----------------------------------------------------------
    @_stream_ordered
    def upload_matrix(self, A, strides=None, offset=0):
        """A: mapping with c, w, e, s, n, b, t (the reference's Matrix)."""
        ptrs = [_ptr(A[k]) for k in "cwesnbt"]
        where = ptrs[0][1]
        nx, ny, nz = self.dims
        si, sj, sk = strides if strides else (ny * nz, nz, 1)
        _check(lib().pbg_matrix_upload(self._h, *[p for p, _ in ptrs], si, sj, sk, offset, where))

    def download_matrix(self):
        out = {k: np.zeros(self.ncell) for k in "cwesnbt"}
        _check(lib().pbg_matrix_download(self._h, *[out[k].ctypes.data for k in "cwesnbt"], HOST))
        return out

    @_stream_ordered
    def upload_active(self, aflag, strides=None, offset=0):
        a = np.ascontiguousarray(aflag, dtype=np.int32)
        nx, ny, nz = self.dims
        si, sj, sk = strides if strides else (ny * nz, nz, 1)
        _check(lib().pbg_active_upload(self._h, a.ctypes.data, si, sj, sk, offset, HOST))

    @_stream_ordered
    def upload_ci(self, ci, strides=None, offset=0):
        """The matrix's stored inverse central coefficient A.ci, read by Jacobi
        and Gauss-Seidel (1/c until it is uploaded, and after every matrix change)."""
        p, where = _ptr(ci)
        nx, ny, nz = self.dims
        si, sj, sk = strides if strides else (ny * nz, nz, 1)
        _check(lib().pbg_ci_upload(self._h, p, si, sj, sk, offset, where))

    @_stream_ordered
    def assemble_pressure(self, rho, solid):
        """Pressure::discretize on the device (harmonic face density)."""
        pr, where = _ptr(rho)
        ps, where2 = _ptr(solid, "uint8")
        if where != where2:
            raise ValueError("rho and solid must live in the same memory")
        _check(lib().pbg_assemble_pressure(self._h, pr, ps, where))

    @_stream_ordered
    def assemble_mix(self, col, rho_a, rho_b=1.0, solid=None):
        """Pressure::discretize of a two-phase mixture on the device
        (arithmetic face density from the colour; col None: one fluid)."""
        pc, where = _ptr(col)
        ps, where2 = _ptr(solid, "uint8")
        if col is not None and solid is not None and where != where2:
            raise ValueError("col and solid must live in the same memory")
        if col is None:
            where = where2
        _check(lib().pbg_assemble_mix(self._h, pc, rho_a, rho_b, ps, where))

    @_stream_ordered
    def divergence(self, u, v, w, dt, rhs, solid=None):
        """Pressure::update_rhs: rhs from the face velocities (solid: a
        voxel body, the immersed-body branch)."""
        pu, where = _ptr(u)
        _check(lib().pbg_divergence(self._h, pu, _ptr(v)[0], _ptr(w)[0], _ptr(solid, "uint8")[0], dt,
                                    _ptr(rhs)[0], where))
        return rhs

    @_stream_ordered
    def project(self, p, col, rho_a, rho_b, dt, u, v, w, solid=None):
        """Momentum::project: u, v, w updated in place."""
        pp, where = _ptr(p)
        _check(lib().pbg_project(self._h, pp, _ptr(col)[0], rho_a, rho_b, _ptr(solid, "uint8")[0], dt,
                                 _ptr(u)[0], _ptr(v)[0], _ptr(w)[0], where))
        return u, v, w

    @_stream_ordered
    def upload_body(self, fV, fS):
        """A cut immersed body for the flow functions (the reference's Body:
        fV per cell, fS the six face fractions per cell, planes w e s n b t);
        fV None removes it. With a body the flow functions take solid=None."""
        if fV is None:
            _check(lib().pbg_body_upload(self._h, None, None, HOST))
            return
        pv, where = _ptr(fV)
        if where == HOST:
            fV = np.ascontiguousarray(fV, dtype=np.float64)
            fS = np.ascontiguousarray(fS, dtype=np.float64)
            pv = fV.ctypes.data
        ps, where2 = _ptr(fS)
        if where2 != where:
            raise ValueError("fV and fS must live in the same memory")
        _check(lib().pbg_body_upload(self._h, pv, ps, where))

    @_stream_ordered
    def pressure_step(self, col, rho_a, rho_b, dt, u, v, w, p, params, solid=None):
        """Assemble, divergence, solve and project in one call; u, v, w and
        p updated in place. Returns the solver's Result."""
        pp, where = _ptr(p)
        res = Result()
        _check(lib().pbg_pressure_step(self._h, _ptr(col)[0], rho_a, rho_b, _ptr(solid, "uint8")[0], dt,
                                       _ptr(u)[0], _ptr(v)[0], _ptr(w)[0], pp, where,
                                       ctypes.byref(params), ctypes.byref(res)))
        return res

    def symmetric(self):
        sym = ctypes.c_int(0)
        _check(lib().pbg_session_info(self._h, None, ctypes.byref(sym), None))
        return bool(sym.value)

    # -- operators ---------------------------------------------------------
    @_stream_ordered
    def spmv(self, x, y):
        px, w = _ptrn(x, self.ncell)
        py, _ = _ptrn(y, self.ncell)
        _check(lib().pbg_spmv(self._h, px, py, w))
        return y

    @_stream_ordered
    def residual(self, x, b, r):
        px, w = _ptrn(x, self.ncell)
        _check(lib().pbg_residual(self._h, px, _ptrn(b, self.ncell)[0], _ptrn(r, self.ncell)[0], w))
        return r

    @_stream_ordered
    def dot(self, x, y):
        out = (ctypes.c_double * 2)()
        px, w = _ptrn(x, self.ncell)
        _check(lib().pbg_dot(self._h, px, _ptrn(y, self.ncell)[0], w, out))
        return out[0], out[1]

    @_stream_ordered
    def seq_sum(self, a, b=None):
        """Sequential sums in index order (pbg_seq_sum): the rounded
        left-to-right sum of a (and of b)."""
        out = (ctypes.c_double * 2)()
        pa, w = _ptr(a)
        pb = None
        if b is not None:
            pb, w2 = _ptr(b)
            if w2 != w or len(b) != len(a):
                raise ValueError("a and b must have the same length and memory")
        _check(lib().pbg_seq_sum(self._h, pa, pb, len(a), w, out))
        return out[0], out[1]

    def levels(self, kind=0):
        cnt = ctypes.c_int(0)
        dims = (ctypes.c_int * (3 * 64))()
        _check(lib().pbg_levels(self._h, kind, ctypes.byref(cnt), dims, 64))
        return [tuple(dims[3 * q:3 * q + 3]) for q in range(cnt.value)]

    def ac_level_matrix(self, level):
        nx, ny, nz = self.levels(0)[level]
        n = nx * ny * nz
        out = np.zeros(7 * n)
        _check(lib().pbg_ac_level_matrix(self._h, level, out.ctypes.data, HOST))
        return {k: out[q * n:(q + 1) * n] for q, k in enumerate("cwesnbt")}

    # -- solve -------------------------------------------------------------
    @_stream_ordered
    def solve(self, x, b, params, strides=None, offset=0):
        need = self.ncell if strides is None else 0
        px, where = _ptrn(x, need)
        pb, where2 = _ptrn(b, need)
        if where != where2:
            raise ValueError("x and b must live in the same memory")
        res = Result()
        if strides is None:
            _check(lib().pbg_solve(self._h, px, pb, where, ctypes.byref(params), ctypes.byref(res)))
        else:
            si, sj, sk = strides
            _check(lib().pbg_solve_strided(self._h, px, pb, si, sj, sk, offset, where,
                                           ctypes.byref(params), ctypes.byref(res)))
        return res

    def stream_handle(self):
        h = _vp()
        _check(lib().pbg_session_stream(self._h, ctypes.byref(h)))
        return h.value or 0

    def bench_kernel(self, which, precision=FP64, reps=20):
        """(ms per launch, algorithmic bytes per launch) of a hot kernel timed alone."""
        ms, by = ctypes.c_double(0), ctypes.c_double(0)
        _check(lib().pbg_bench_kernel(self._h, which, precision, reps, ctypes.byref(ms), ctypes.byref(by)))
        return ms.value, by.value

    def history(self):
        n = ctypes.c_int(0)
        _check(lib().pbg_history(self._h, None, 0, ctypes.byref(n)))
        out = np.zeros(max(n.value, 1))
        _check(lib().pbg_history(self._h, out.ctypes.data_as(_dp), n.value, ctypes.byref(n)))
        return out[:n.value]


# ---------------------------------------------------------------- solvers
class _Krylov:
    solver = SOLVER_CG

    PREC = {"di": 0, "diagonal": 0, "ic0": 1, "ic2": 2, "ic3": 3}

    def __init__(self, session, prec="di", exact_sums=False):
        if prec not in self.PREC:
            raise ValueError("prec must be one of %s (Prec::di/ic0/ic2/ic3)" % sorted(self.PREC))
        self.prec = self.PREC[prec]
        self.session = session
        self.exact_sums = exact_sums
        self.last = None

    def solve(self, x, b, min_iter=1, max_iter=20, name=None, res_rat=0.01, res_tol=1.0e-15,
              scale=1.0, stalecount=-1):
        """Linear::solve(A, x, b, MinIter, MaxIter, name, ResRat, ResTol, scale,
        stalecount): updates x in place, returns the converged flag."""
        p = default_params(self.solver)
        p.min_iter, p.max_iter = int(min_iter), int(max_iter)
        p.res_rat, p.res_tol, p.scale, p.stalecount = res_rat, res_tol, scale, int(stalecount)
        p.exact_sums = int(self.exact_sums)
        p.prec = self.prec
        self.last = self.session.solve(x, b, p)
        if name is not None:
            r = self.last
            print("%s, residual = %.17g, ratio = %.17g, iterations = %d" %
                  (name, r.res, r.res / r.res0 if r.res0 else 0.0, r.iterations))
        return bool(self.last.converged)


class CG(_Krylov):
    """CG with the diagonal preconditioner (Src/Solver/Linear/Krylov/cg.cpp)."""
    solver = SOLVER_CG


class BiCGS(_Krylov):
    """BiCGStab (Krylov/bicgs.cpp), diagonal or IC preconditioner."""
    solver = SOLVER_BICGS


class CGS(_Krylov):
    """Conjugate gradient squared (Krylov/cgs.cpp), diagonal or IC preconditioner."""
    solver = SOLVER_CGS


class Jacobi(_Krylov):
    """Jacobi (Src/Solver/Linear/Iterative/jacobi.cpp): x = ci (r + c x) per sweep;
    res and res0 are sqrt(r.r). Reads the session's A.ci (Session.upload_ci)."""
    solver = SOLVER_JACOBI

    def __init__(self, session, exact_sums=False):
        super().__init__(session, "di", exact_sums)


class GaussSeidel(_Krylov):
    """Gauss-Seidel (Iterative/gaussseidel.cpp), lexicographic sweeps run as one
    launch per hyperplane i + j + k (the sequential sweep's values)."""
    solver = SOLVER_GAUSS_SEIDEL

    def __init__(self, session, exact_sums=False):
        super().__init__(session, "di", exact_sums)


class AC:
    """Additive-correction multigrid (Src/Solver/Additive). smoother: the
    Linear solver every level uses ("cg", "bicgs", "cgs" with prec, or
    "jacobi", "gs"), as the Centered object's solver is in the reference."""

    SMOOTHERS = {"cg": SOLVER_CG, "bicgs": SOLVER_BICGS, "cgs": SOLVER_CGS, "jacobi": SOLVER_JACOBI,
                 "gs": SOLVER_GAUSS_SEIDEL}

    def __init__(self, session, exact_sums=False, smoother="cg", prec="di", solver=None, solver_prec="di"):
        """solver: AC's own solver for post-smoothing and the coarsest level,
        AC(cen, sol) (additive.cpp:8-48); None: the smoother."""
        if smoother not in self.SMOOTHERS or (solver is not None and solver not in self.SMOOTHERS):
            raise ValueError("smoother and solver must be one of %s" % sorted(self.SMOOTHERS))
        self.session = session
        self.exact_sums = exact_sums
        self.smoother = self.SMOOTHERS[smoother]
        self.prec = _Krylov.PREC[prec]
        self.solver = -1 if solver is None else self.SMOOTHERS[solver]
        self.solver_prec = _Krylov.PREC[solver_prec]
        self._resrat, self._restol, self._linf = 1.0e-18, 1.0e-18, False
        self.flex_visits = 1000000
        self._max_cyc, self._min_cyc = 20, 0
        self._stop_if_div, self._prio = True, True
        self.mv = [20, 20, 20]
        self.ms = [-1, -1, -1]
        self.last = None

    # setters of additive.h:97-142
    def max_cycles(self, mc=None):
        if mc is None:
            return self._max_cyc
        self._max_cyc = int(mc)

    def min_cycles(self, mc=None):
        if mc is None:
            return self._min_cyc
        self._min_cyc = int(mc)

    def stop_if_diverging(self, s=None):
        if s is None:
            return self._stop_if_div
        self._stop_if_div = bool(s)

    def priority_min_cycle(self, s=None):
        if s is None:
            return self._prio
        self._prio = bool(s)

    def max_iter_array(self, mv):
        self.mv = list(mv)

    def stale_iter_array(self, ms):
        self.ms = list(ms)

    def resrat(self, rr=None):
        """AC::resrat: the ResRat of the level solvers (default 1e-18)."""
        if rr is None:
            return self._resrat
        self._resrat = float(rr)

    def restol(self, rt=None):
        """AC::restol: the ResTol of the level solvers (default 1e-18)."""
        if rt is None:
            return self._restol
        self._restol = float(rt)

    def use_linf_error(self, s=None):
        """AC::use_linf_error: the cycle's tests on max |r/dV|."""
        if s is None:
            return self._linf
        self._linf = bool(s)

    def cycle(self, x, b, init=CYCLE_NONE, loop=CYCLE_V, toler=-1.0, factor=-1.0, mv=None, ms=None):
        """AC::cycle(init, loop, ResTol, ResRat, mv, ms, &ncyc) -> (bool, ncyc)."""
        p = default_params(SOLVER_AC)
        p.init_cycle, p.loop_cycle = init, loop
        p.toler, p.factor = toler, factor
        p.max_cycles, p.min_cycles = self._max_cyc, self._min_cyc
        p.stop_if_div, p.priority_min_cyc = int(self._stop_if_div), int(self._prio)
        for q in range(3):
            p.mv[q] = (mv or self.mv)[q]
            p.ms[q] = (ms or self.ms)[q]
        p.exact_sums = int(self.exact_sums)
        p.ac_smoother, p.prec = self.smoother, self.prec
        p.ac_solver, p.ac_solver_prec = self.solver, self.solver_prec
        p.ac_resrat, p.ac_restol, p.use_linf = self._resrat, self._restol, int(self._linf)
        p.flex_visits = int(self.flex_visits)
        self.last = self.session.solve(x, b, p)
        return bool(self.last.converged), self.last.cycles

    def vcycle(self, x, b, factor=-1.0, toler=-1.0):
        return self.cycle(x, b, CYCLE_NONE, CYCLE_V, toler, factor)

    def fcycle(self, x, b, factor=-1.0, toler=-1.0):
        return self.cycle(x, b, CYCLE_NONE, CYCLE_F, toler, factor)

    def wcycle(self, x, b, factor=-1.0, toler=-1.0):
        return self.cycle(x, b, CYCLE_NONE, CYCLE_W, toler, factor)

    def fullcycle(self, x, b, loop=CYCLE_V, factor=-1.0, toler=-1.0):
        return self.cycle(x, b, CYCLE_V, loop, toler, factor)

    def flexcycle(self, x, b, factor=-1.0, toler=-1.0):
        """AC::flexcycle: ends when level 0's smoother reaches resrat()."""
        return self.cycle(x, b, CYCLE_NONE, CYCLE_FLEX, toler, factor)


class Engine:
    """Flexible CG + AC K-cycle; FP64 or mixed (FP32 inner, FP64 refinement).
    A non-symmetric matrix (a cut body's) is solved by FP64 refinement around
    its symmetric part; a sweep that does not reduce the residual is undone
    and the result says DIVERGED."""

    def __init__(self, session):
        self.session = session
        self.last = None

    def solve(self, x, b, tol=1.0e-8, precision=FP64, inner_tol=1.0e-3, max_iter=500,
              max_sweeps=8, coarse_max=0, x0_zero=False):
        """x0_zero: start from zero (x is output only and is not uploaded)."""
        p = default_params(SOLVER_ENGINE)
        p.precision, p.tol, p.inner_tol = precision, tol, inner_tol
        p.max_iter, p.max_sweeps, p.coarse_max = max_iter, max_sweeps, coarse_max
        p.x0_zero = 1 if x0_zero else 0
        self.last = self.session.solve(x, b, p)
        return bool(self.last.converged)


def generate(kind, seed, n=16, nb=0, rmin=4.0, rmax=16.0, rc=0.0, ratio=1000.0, index=0, n2d=0,
             s2=(64, 512), s3=(32, 96), stream=0):
    """Seeded workload (psiboil_b200/csrc/problem_gen.h): returns
    (dims, h, rho, solid, b)."""
    params = (ctypes.c_double * 13)(n, nb, rmin, rmax, rc, ratio, index, n2d, s2[0], s2[1],
                                    s3[0], s3[1], stream)
    dims = (ctypes.c_int * 3)()
    h = ctypes.c_double(0.0)
    _check(lib().pbg_generate(kind, params, seed, dims, ctypes.byref(h), None, None, None))
    N = dims[0] * dims[1] * dims[2]
    rho = np.zeros(N)
    solid = np.zeros(N, dtype=np.uint8)
    b = np.zeros(N)
    _check(lib().pbg_generate(kind, params, seed, dims, ctypes.byref(h), rho.ctypes.data_as(_dp),
                              solid.ctypes.data, b.ctypes.data))
    return tuple(dims), h.value, rho, solid, b


def generate_flow(kind, seed, n=16, nb=0, rmin=4.0, rmax=16.0, rc=0.0, ratio=1000.0, index=0, n2d=0,
                  s2=(64, 512), s3=(32, 96), stream=0):
    """Flow state of one pressure-correction step (problem_gen.h
    pbg_gen_flow): (col, u, v, w, rho_liquid, rho_vapour), face arrays
    shaped (nx+1,ny,nz), (nx,ny+1,nz), (nx,ny,nz+1)."""
    (nx, ny, nz), _, _, _, _ = generate(kind, seed, n, nb, rmin, rmax, rc, ratio, index, n2d, s2, s3,
                                        stream)
    params = (ctypes.c_double * 13)(n, nb, rmin, rmax, rc, ratio, index, n2d, s2[0], s2[1],
                                    s3[0], s3[1], stream)
    col = np.zeros((nx, ny, nz))
    u = np.zeros((nx + 1, ny, nz))
    v = np.zeros((nx, ny + 1, nz))
    w = np.zeros((nx, ny, nz + 1))
    rho = (ctypes.c_double * 2)()
    _check(lib().pbg_generate_flow(kind, params, seed, col.ctypes.data, u.ctypes.data, v.ctypes.data,
                                   w.ctypes.data, rho))
    return col, u, v, w, rho[0], rho[1]


KIND_SINGLE, KIND_CYL, KIND_BATCH = 0, 1, 2


def batch_config(precision=MIXED, slots=64, **shape):
    c = BatchConfig()
    lib().pbg_batch_config_default(ctypes.byref(c))
    c.precision, c.slots = precision, slots
    for k, v in shape.items():
        setattr(c, k, v)
    return c


class Batch:
    """Many independent pressure problems solved together (pbg_batch_*).

    Each problem keeps its matrix, hierarchy and solution on the device;
    solve() starts from the stored solution (warm start) unless reset."""

    def __init__(self, precision=MIXED, slots=64, device=0, **shape):
        self.config = batch_config(precision, slots, **shape)
        h = _vp()
        _check(lib().pbg_batch_create(ctypes.byref(self.config), device, ctypes.byref(h)))
        self._h = h
        self.dims = {}

    def close(self):
        if self._h:
            lib().pbg_batch_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def problem_bytes(self, nx, ny, nz):
        v = _ll(0)
        _check(lib().pbg_batch_problem_bytes(self._h, nx, ny, nz, ctypes.byref(v)))
        return v.value

    @_inputs_ready
    def add(self, dims, h, rho=None, solid=None, b=None, x=None, bc=None):
        """A new problem; returns its id."""
        if bc is None:  # Dirichlet top: kmax in 3-D, jmax in 2-D (as Session)
            bc = [NEUMANN] * 6
            bc[5 if dims[2] > 1 else 3] = DIRICHLET
        cbc = (ctypes.c_int * 6)(*bc)
        pid = ctypes.c_int(-1)
        _check(lib().pbg_batch_add(self._h, dims[0], dims[1], dims[2], h, cbc, ctypes.byref(pid)))
        i = pid.value
        self.dims[i] = tuple(dims)
        if rho is not None:
            self.set_fields(i, rho, solid)
        if b is not None:
            self.set_rhs(i, b)
        self.set_x(i, x)
        return i

    def remove(self, i):
        _check(lib().pbg_batch_remove(self._h, i))
        self.dims.pop(i, None)

    @_inputs_ready
    def set_fields(self, i, rho, solid):
        pr, wr = _ptr(rho)
        ps, ws = _ptr(solid, "uint8")
        if wr != ws:
            raise ValueError("rho and solid must live on the same side")
        _check(lib().pbg_batch_set_fields(self._h, i, pr, ps, wr))

    @_inputs_ready
    def set_rhs(self, i, b):
        pb_, w = _ptr(b)
        _check(lib().pbg_batch_set_rhs(self._h, i, pb_, w))

    @_inputs_ready
    def set_x(self, i, x=None):
        px, w = _ptr(x)
        _check(lib().pbg_batch_set_x(self._h, i, px, w))

    def get_x(self, i, out=None):
        if out is None:
            d = self.dims[i]
            out = np.zeros(d[0] * d[1] * d[2])
        p, w = _ptr(out)
        _check(lib().pbg_batch_get_x(self._h, i, p, w))
        return out

    @staticmethod
    def _params(tol, inner_tol, max_iter, max_sweeps):
        p = default_params(SOLVER_ENGINE)
        p.tol, p.inner_tol, p.max_iter, p.max_sweeps = tol, inner_tol, max_iter, max_sweeps
        return p

    def solve(self, ids, tol=1.0e-8, inner_tol=1.0e-3, max_iter=500, max_sweeps=8):
        """Solve the problems `ids`; returns a list of Result (seconds = time
        from the start of the call until that problem finished)."""
        ids = list(ids)
        arr = (ctypes.c_int * len(ids))(*ids)
        res = (Result * len(ids))()
        p = self._params(tol, inner_tol, max_iter, max_sweeps)
        _check(lib().pbg_batch_solve(self._h, arr, len(ids), ctypes.byref(p), res))
        return list(res)

    def autotune(self, ids, cache=None, tol=1.0e-8, inner_tol=1.0e-3, max_iter=500, max_sweeps=8):
        ids = list(ids)
        arr = (ctypes.c_int * len(ids))(*ids)
        p = self._params(tol, inner_tol, max_iter, max_sweeps)
        best = BatchConfig()
        _check(lib().pbg_batch_autotune(self._h, arr, len(ids), ctypes.byref(p),
                                        cache.encode() if cache else None, ctypes.byref(best)))
        self.config = best
        return best


class Server:
    """The serving loop (pbg_server_*): resident sessions, a request queue
    and a worker thread that batches requests continuously on one GPU."""

    def __init__(self, precision=MIXED, slots=64, hbm_budget=0, device=0, **kw):
        c = ServerConfig()
        lib().pbg_server_config_default(ctypes.byref(c))
        c.precision, c.slots, c.hbm_budget = precision, slots, hbm_budget
        for k, v in kw.items():
            setattr(c, k, v)
        self.config = c
        h = _vp()
        _check(lib().pbg_server_create(ctypes.byref(c), device, ctypes.byref(h)))
        self._h = h
        self.dims = {}

    def close(self):
        if self._h:
            lib().pbg_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def open_session(self, dims, h, bc=None):
        if bc is None:
            bc = [NEUMANN] * 6
            bc[5 if dims[2] > 1 else 3] = DIRICHLET
        sid = ctypes.c_int(-1)
        _check(lib().pbg_server_open_session(self._h, dims[0], dims[1], dims[2], h,
                                             (ctypes.c_int * 6)(*bc), ctypes.byref(sid)))
        self.dims[sid.value] = tuple(dims)
        return sid.value

    def close_session(self, sid):
        _check(lib().pbg_server_close_session(self._h, sid))
        self.dims.pop(sid, None)

    @_inputs_ready
    def submit(self, sid, rhs, rho=None, solid=None):
        pb_, w = _ptr(rhs)
        pr, _ = _ptr(rho)
        ps, _ = _ptr(solid, "uint8")
        rid = _ll(-1)
        _check(lib().pbg_server_submit(self._h, sid, pr, ps, pb_, w, ctypes.byref(rid)))
        return rid.value

    def submit_bubble(self, sid, center, radius, ratio, seed):
        c = (ctypes.c_double * 3)(*center)
        rid = _ll(-1)
        _check(lib().pbg_server_submit_bubble(self._h, sid, c, radius, ratio, seed, ctypes.byref(rid)))
        return rid.value

    def wait(self, rid, timeout=-1.0):
        """(Result, latency seconds) of a request."""
        r = Result()
        lat = ctypes.c_double(0.0)
        _check(lib().pbg_server_wait(self._h, rid, timeout, ctypes.byref(r), ctypes.byref(lat)))
        return r, lat.value

    def get_x(self, sid, out=None):
        if out is None:
            d = self.dims[sid]
            out = np.zeros(d[0] * d[1] * d[2])
        p, w = _ptr(out)
        _check(lib().pbg_server_get_x(self._h, sid, p, w))
        return out

    def stats(self):
        st = ServerStats()
        _check(lib().pbg_server_stats_get(self._h, ctypes.byref(st)))
        return st.as_dict()


# ---------------------------------------------------------------- .bck checkpoints
BW = 3  # the reference's halo width


def bck_name(base, step=-1, cpu=-1):
    """name_file(base, ".bck", step, cpu) of the reference."""
    buf = ctypes.create_string_buffer(len(base) + 64)
    _check(lib().pbg_bck_name(base.encode(), step, cpu, buf, len(buf)))
    return buf.value.decode()


def _field_ptrs(fields):
    ps, where = [], None
    for f in fields:
        p, w = _ptr(f)
        if where is not None and w != where:
            raise ValueError("fields must all be host or all device arrays")
        ps.append(p)
        where = w
    return (ctypes.c_void_p * len(ps))(*ps), where


def bck_write(path, fields, dims, compact=True):
    """Write fields (phi, cold, ...) to a .bck file. compact: interior
    arrays of an nx x ny x nz grid (dims); else full halo blocks (dims =
    block extents)."""
    arr, where = _field_ptrs(fields)
    fn = lib().pbg_bck_write_compact if compact else lib().pbg_bck_write
    _check(fn(path.encode(), len(fields), arr, dims[0], dims[1], dims[2], where))


def bck_read(path, nfields, dims, compact=True, out=None):
    """Read nfields fields from a .bck file (see bck_write); host arrays."""
    if out is None:
        n = dims[0] * dims[1] * dims[2] if compact else dims[0] * dims[1] * dims[2]
        out = [np.zeros(n) for _ in range(nfields)]
    arr, where = _field_ptrs(out)
    fn = lib().pbg_bck_read_compact if compact else lib().pbg_bck_read
    _check(fn(path.encode(), nfields, arr, dims[0], dims[1], dims[2], where))
    return out

