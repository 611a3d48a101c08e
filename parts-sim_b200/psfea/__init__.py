"""psfea — Python binding (ctypes) of the C ABI in include/ps_fea.h.

Mirrors the reference's solver class, ``ps::VoxelFEA`` (native/src/fea/voxel_fea.hpp:130-189):
same constructor arguments, ``solve`` with ``SolveOptions`` fields (tol, max_iter, x0, cancel),
``precondition``, ``apply``, ``stresses``, ``reactions``. Invalid inputs raise ``ValueError``
where the reference throws ``std::invalid_argument``. There is no CPU fallback: if the compiled
library is missing, importing this module fails.
"""
import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpsfea.so")

PS_OK, PS_NOT_CONVERGED, PS_BREAKDOWN, PS_CANCELLED, PS_TIMEOUT, PS_PENDING = 0, 1, 2, 3, 4, 5
PS_EINVAL, PS_ENONFINITE, PS_EOOM, PS_ECUDA, PS_ENODEV = 10, 11, 12, 13, 14
PREC = {"fp64": 0, "mixed": 1, "fp32": 2, "half": 3}
CUDA_STREAM_LEGACY = 1  # cudaStreamLegacy: the legacy default stream (PyTorch's default stream, reported as 0)
STATUS_NAMES = {0: "OK", 1: "NOT_CONVERGED", 2: "BREAKDOWN", 3: "CANCELLED", 4: "TIMEOUT", 5: "PENDING", 10: "EINVAL", 11: "ENONFINITE",
                12: "EOOM", 13: "ECUDA", 14: "ENODEV"}


class SolveOpts(C.Structure):
    _fields_ = [("tol", C.c_double), ("max_iter", C.c_int32), ("precision", C.c_int32), ("x0", C.c_void_p),
                ("cancel", C.c_void_p), ("time_limit_s", C.c_double), ("smoother_degree", C.c_int32)]


class SolveResultC(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("converged", C.c_int32), ("status", C.c_int32), ("folds", C.c_int32),
                ("residual", C.c_double), ("seconds", C.c_double), ("kernels", C.c_int64)]


class PsRequest(C.Structure):
    _fields_ = [("dims", C.c_int32 * 3), ("density", C.c_void_p), ("nu", C.c_double), ("bc", C.c_void_p), ("f", C.c_void_p),
                ("coarsest_max_dof", C.c_int64), ("tol", C.c_double), ("max_iter", C.c_int32), ("precision", C.c_int32),
                ("smoother_degree", C.c_int32)]


class PsRequestResult(C.Structure):
    _fields_ = [("id", C.c_int64), ("status", C.c_int32), ("iterations", C.c_int32), ("converged", C.c_int32), ("residual", C.c_double),
                ("n_dof", C.c_int64), ("u", C.c_void_p), ("build_s", C.c_double), ("wait_s", C.c_double), ("solve_s", C.c_double),
                ("total_s", C.c_double)]


class TopologyOpts(C.Structure):
    _fields_ = [("vol_frac", C.c_double), ("penal", C.c_double), ("rmin", C.c_double), ("move", C.c_double), ("tol", C.c_double),
                ("max_iter", C.c_int32), ("solve_tol", C.c_double), ("precision", C.c_int32)]


class TopologyStepC(C.Structure):
    _fields_ = [("it", C.c_int32), ("solve_iterations", C.c_int32), ("solve_status", C.c_int32), ("compliance", C.c_double),
                ("volume", C.c_double), ("change", C.c_double), ("seconds", C.c_double)]


class BreakStepC(C.Structure):
    _fields_ = [("step", C.c_int32), ("voxels", C.c_int32), ("solve_iterations", C.c_int32), ("cracked", C.c_int32), ("detached", C.c_int32),
                ("lambda_", C.c_double), ("max_disp", C.c_double), ("seconds", C.c_double)]


BREAK_REASONS = {0: "step limit", 1: "separated", 2: "unsupported load", 3: "solver did not converge", 4: "no stress"}


class TuneResultC(C.Structure):
    _fields_ = [("smoother_degree", C.c_int32), ("inner64", C.c_int32), ("split_levels", C.c_int64), ("coarsest_max_dof", C.c_int64),
                ("trials", C.c_int32), ("cached", C.c_int32), ("best_seconds", C.c_double), ("default_seconds", C.c_double)]


PS_TUNE_FORCE = 1


class PsServerStats(C.Structure):
    _fields_ = [("queued", C.c_int64), ("active", C.c_int64), ("completed", C.c_int64), ("device_bytes_in_use", C.c_int64),
                ("peak_device_bytes", C.c_int64), ("budget_bytes", C.c_int64), ("peak_active", C.c_int64)]


if not os.path.exists(LIB_PATH):
    raise ImportError(f"{LIB_PATH} is not built: run `make -C parts-sim_b200/csrc` (or __graft_entry__.build())")
lib = C.CDLL(LIB_PATH)

_P = C.c_void_p
_F64P = np.ctypeslib.ndpointer(np.float64, flags="C")
_F32P = np.ctypeslib.ndpointer(np.float32, flags="C")
_U8P = np.ctypeslib.ndpointer(np.uint8, flags="C")
_I32P = np.ctypeslib.ndpointer(np.int32, flags="C")
_I64P = np.ctypeslib.ndpointer(np.int64, flags="C")


def _sig(name, res, *args):
    f = getattr(lib, name)
    f.restype = res
    f.argtypes = list(args)
    return f


_create = _sig("ps_fea_create", C.c_int, _I32P, _F32P, C.c_double, _U8P, C.c_int64, C.c_void_p, C.POINTER(C.c_void_p))
_destroy = _sig("ps_fea_destroy", None, _P)
_solve = _sig("ps_fea_solve", C.c_int, _P, _F64P, C.POINTER(SolveOpts), _F64P, C.POINTER(SolveResultC))
_solve_dev = _sig("ps_fea_solve_dev", C.c_int, _P, C.c_void_p, C.POINTER(SolveOpts), C.c_void_p, C.POINTER(SolveResultC))
_solve_batch = _sig("ps_fea_solve_batch", C.c_int, _P, C.c_int32, _F64P, C.POINTER(SolveOpts), _F64P, C.c_void_p)
_precondition = _sig("ps_fea_precondition", C.c_int, _P, _F64P, _F64P)
_precondition_block = _sig("ps_fea_precondition_block", C.c_int, _P, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p)
_apply = _sig("ps_fea_apply", C.c_int, _P, C.c_int32, _F64P, _F64P, C.c_int32)
_stresses = _sig("ps_fea_stresses", C.c_int, _P, _F64P, C.c_double, C.c_double, C.c_int32, _F32P, C.c_void_p, C.c_void_p)
_reactions = _sig("ps_fea_reactions", C.c_int, _P, _F64P, C.c_void_p, _F64P)
_ndof = _sig("ps_fea_ndof", C.c_int64, _P)
_nlev = _sig("ps_fea_num_levels", C.c_int32, _P)
_level_info = _sig("ps_fea_level_info", C.c_int, _P, C.c_int32, _I64P)
_level_fixed = _sig("ps_fea_level_fixed", C.c_int, _P, C.c_int32, _U8P)
_level_lmax = _sig("ps_fea_level_lmax", C.c_double, _P, C.c_int32)
_dev_bytes = _sig("ps_fea_device_bytes", C.c_int64, _P)
_set_stream = _sig("ps_fea_set_stream", C.c_int, _P, C.c_void_p)
_time_kernel = _sig("ps_fea_time_kernel", C.c_int, _P, C.c_int32, C.c_int32, C.POINTER(C.c_double))
_launches = _sig("ps_fea_kernel_launches", C.c_int64, _P)
_srv_create = _sig("ps_server_create", C.c_int, C.c_int64, C.c_int32, C.c_int32, C.POINTER(C.c_void_p))
_srv_submit = _sig("ps_server_submit", C.c_int, _P, C.POINTER(PsRequest), C.POINTER(C.c_int64))
_srv_poll = _sig("ps_server_poll", C.c_int, _P, C.c_int64, C.POINTER(PsRequestResult))
_srv_wait = _sig("ps_server_wait", C.c_int, _P, C.c_int64, C.POINTER(PsRequestResult))
_srv_release = _sig("ps_server_release", C.c_int, _P, C.c_int64)
_srv_stats = _sig("ps_server_get_stats", C.c_int, _P, C.POINTER(PsServerStats))
_srv_destroy = _sig("ps_server_destroy", None, _P)
_apply_dot_noalloc = _sig("ps_fea_apply_dot_noalloc", C.c_int, _P, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p)
_element = _sig("ps_element_matrix", C.c_int, C.c_double, _F64P, C.c_void_p)
_autotune = _sig("ps_fea_autotune", C.c_int, _P, _F64P, C.POINTER(SolveOpts), C.c_int32, C.POINTER(TuneResultC))
_create_tuned = _sig("ps_fea_create_tuned", C.c_int, _I32P, _F32P, C.c_double, _U8P, C.c_void_p, _F64P, C.POINTER(SolveOpts), C.c_int32,
                     C.POINTER(TuneResultC), C.POINTER(C.c_void_p))
_topo_default = _sig("ps_topology_opts_default", None, C.POINTER(TopologyOpts))
_topo_run = _sig("ps_topology_run", C.c_int, _I32P, _F32P, C.c_void_p, C.c_double, _U8P, _F64P, C.POINTER(TopologyOpts), _F32P, C.c_void_p,
                 C.POINTER(C.c_int32))
_break_test = _sig("ps_break_test", C.c_int, _I32P, _F32P, C.c_double, _U8P, _F64P, C.c_double, C.c_double, C.c_double, C.c_int32, C.c_int32,
                   C.c_void_p, C.POINTER(C.c_int32), C.c_void_p, C.c_int64, _F32P, C.POINTER(C.c_double), C.POINTER(C.c_int32))
_prune = _sig("ps_prune_floating", C.c_int, _I32P, _F32P, _U8P, _F32P, C.POINTER(C.c_int32))
_prune_dev = _sig("ps_prune_floating_dev", C.c_int, _I32P, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_int32), C.c_void_p)
_last_error = _sig("ps_last_error", C.c_char_p)
_opts_default = _sig("ps_solve_opts_default", None, C.POINTER(SolveOpts))
_h_create = _sig("ps_hierarchy_create", C.c_int, _I32P, _F32P, C.c_double, _U8P, C.c_int64, C.c_void_p, C.POINTER(C.c_void_p))
_h_create_dev = _sig("ps_hierarchy_create_dev", C.c_int, _I32P, _F32P, C.c_double, _U8P, C.c_int64, C.c_void_p, C.POINTER(C.c_void_p))
_h_nlev = _sig("ps_hierarchy_num_levels", C.c_int32, _P)
_h_info = _sig("ps_hierarchy_level_info", C.c_int, _P, C.c_int32, _I64P)
_h_fixed = _sig("ps_hierarchy_level_fixed", C.c_int, _P, C.c_int32, _U8P)
_h_own = _sig("ps_hierarchy_level_own", C.c_int, _P, C.c_int32, _F32P)
_h_kb = _sig("ps_hierarchy_level_kb", C.c_int, _P, C.c_int32, _F64P)
_h_destroy = _sig("ps_hierarchy_destroy", None, _P)

#: every symbol include/ps_fea.h declares
EXPORTS = ("ps_solve_opts_default", "ps_fea_create", "ps_fea_solve", "ps_fea_solve_dev", "ps_fea_solve_batch", "ps_fea_precondition",
           "ps_fea_apply", "ps_fea_stresses", "ps_fea_reactions", "ps_fea_ndof", "ps_fea_num_levels", "ps_fea_level_info",
           "ps_fea_level_fixed", "ps_fea_level_lmax", "ps_fea_device_bytes", "ps_fea_destroy", "ps_element_matrix",
           "ps_prune_floating", "ps_last_error", "ps_hierarchy_create", "ps_hierarchy_create_dev", "ps_hierarchy_num_levels", "ps_hierarchy_level_info",
           "ps_hierarchy_level_fixed", "ps_hierarchy_level_own", "ps_hierarchy_level_kb", "ps_hierarchy_destroy",
           "ps_fea_set_stream", "ps_fea_time_kernel", "ps_fea_kernel_launches", "ps_fea_apply_dot_noalloc", "ps_fea_precondition_block",
           "ps_topology_opts_default", "ps_topology_run", "ps_break_test", "ps_fea_autotune", "ps_fea_create_tuned",
           "ps_prune_floating_dev",
           "ps_server_create", "ps_server_submit", "ps_server_poll", "ps_server_wait", "ps_server_release", "ps_server_get_stats",
           "ps_server_destroy")


class SolverError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


def _raise(status):
    msg = (_last_error() or b"").decode()
    if status in (PS_EINVAL, PS_ENONFINITE):
        raise ValueError(msg)
    if status == PS_EOOM:
        raise MemoryError(msg)
    raise SolverError(status, msg)


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


@dataclass
class SolveResult:
    """voxel_fea.hpp:119-124 plus the status code, FP64 fold count (mixed) and wall time."""
    u: np.ndarray
    iterations: int
    residual: float
    converged: bool
    status: int
    folds: int = 0
    seconds: float = 0.0
    kernels: int = 0

    @property
    def cancelled(self):
        return self.status == PS_CANCELLED


def make_opts(tol=1e-6, max_iter=500, precision="fp64", x0=None, cancel=None, time_limit_s=0.0, smoother_degree=0):
    o = SolveOpts()
    _opts_default(C.byref(o))
    o.tol = float(tol)
    o.max_iter = int(max_iter)
    o.precision = PREC[precision] if isinstance(precision, str) else int(precision)
    o.x0 = x0
    o.cancel = cancel
    o.time_limit_s = float(time_limit_s)
    o.smoother_degree = int(smoother_degree)
    return o


class VoxelFEA:
    """Device-resident solver for one voxel model (``ps::VoxelFEA`` + ``ps::GpuFeaSolver`` in one)."""

    def __init__(self, dims, density, nu, bc, coarsest_max_dof=1100, diag_add=None):
        self.dims = np.ascontiguousarray(dims, np.int32)
        nx, ny, nz = (int(v) for v in self.dims)
        density = np.ascontiguousarray(density, np.float32).ravel()
        bc = np.ascontiguousarray(bc, np.uint8).ravel()
        if nx >= 1 and ny >= 1 and nz >= 1 and (density.size != nx * ny * nz or bc.size != 3 * (nx + 1) * (ny + 1) * (nz + 1)):
            raise ValueError("Structural grid, density and fixture sizes do not match.")
        self._diag = None if diag_add is None else np.ascontiguousarray(diag_add, np.float64).ravel()
        if self._diag is not None and self._diag.size != 3 * (nx + 1) * (ny + 1) * (nz + 1):
            raise ValueError("Diagonal shift size does not match.")
        h = C.c_void_p()
        st = _create(self.dims, density, float(nu), bc, int(coarsest_max_dof), _ptr(self._diag), C.byref(h))
        if st != PS_OK:
            _raise(st)
        self.h = h
        self.nu = nu

    def close(self):
        if getattr(self, "h", None):
            _destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def n_dof(self):
        return int(_ndof(self.h))

    @property
    def n_nodes(self):
        return self.n_dof // 3

    @property
    def n_levels(self):
        return int(_nlev(self.h))

    @property
    def device_bytes(self):
        return int(_dev_bytes(self.h))

    def level_info(self, l):
        out = np.zeros(9, np.int64)
        st = _level_info(self.h, l, out)
        if st != PS_OK:
            _raise(st)
        keys = ("nx", "ny", "nz", "nNodes", "nDof", "freeDof", "nElems", "nOwn", "coarse_m")
        return dict(zip(keys, (int(v) for v in out)))

    def fixed(self, l=0):
        out = np.zeros(self.level_info(l)["nDof"], np.uint8)
        st = _level_fixed(self.h, l, out)
        if st != PS_OK:
            _raise(st)
        return out

    def lmax(self, l):
        return float(_level_lmax(self.h, l))

    def _check_vec(self, v, name):
        v = np.ascontiguousarray(v, np.float64).ravel()
        if v.size != self.n_dof:
            raise ValueError("Force or displacement vector has the wrong size.")
        return v

    def solve(self, f, tol=1e-6, max_iter=500, x0=None, precision="fp64", cancel=None, time_limit_s=0.0, smoother_degree=0,
              out=None):
        """K u = f; returns a SolveResult (u in normalised units: u_phys = u / (E h)). out: a
        C-contiguous float64 array of n_dof values that receives u and is returned as the result's
        u (for instance in pinned host memory, which the device writes at full speed); else a new
        array."""
        f = self._check_vec(f, "f")
        x0a = None if x0 is None else self._check_vec(x0, "x0")
        o = make_opts(tol, max_iter, precision, _ptr(x0a), None if cancel is None else C.addressof(cancel), time_limit_s, smoother_degree)
        if out is None:
            u = np.zeros(self.n_dof, np.float64)
        elif isinstance(out, np.ndarray) and out.dtype == np.float64 and out.flags.c_contiguous and out.size == self.n_dof:
            u = out.reshape(-1)
        else:
            raise ValueError("out must be a C-contiguous float64 array of n_dof values.")
        r = SolveResultC()
        st = _solve(self.h, f, C.byref(o), u, C.byref(r))
        if st >= PS_EINVAL:
            _raise(st)
        return SolveResult(u if out is None else out, r.iterations, r.residual, bool(r.converged), st, r.folds, r.seconds, r.kernels)

    def solve_dev(self, f_ptr, u_ptr, tol=1e-6, max_iter=500, precision="fp64", x0_ptr=None, smoother_degree=0):
        """The solve on device pointers (e.g. ``tensor.data_ptr()`` of CUDA float64 tensors)."""
        o = make_opts(tol, max_iter, precision, x0_ptr, smoother_degree=smoother_degree)
        r = SolveResultC()
        st = _solve_dev(self.h, C.c_void_p(f_ptr), C.byref(o), C.c_void_p(u_ptr), C.byref(r))
        if st >= PS_EINVAL:
            _raise(st)
        return SolveResult(None, r.iterations, r.residual, bool(r.converged), st, r.folds, r.seconds, r.kernels)

    def solve_batch(self, F, tol=1e-6, max_iter=500, precision="fp64", X0=None):
        F = np.ascontiguousarray(F, np.float64)
        nrhs = F.shape[0]
        if F.shape[1] != self.n_dof:
            raise ValueError("Force or displacement vector has the wrong size.")
        X0 = None if X0 is None else np.ascontiguousarray(X0, np.float64)
        o = make_opts(tol, max_iter, precision, _ptr(X0))
        U = np.zeros_like(F)
        res = (SolveResultC * nrhs)()
        st = _solve_batch(self.h, nrhs, F.ravel(), C.byref(o), U.ravel(), C.cast(res, C.c_void_p))
        if st >= PS_EINVAL:
            _raise(st)
        return [SolveResult(U[q], res[q].iterations, res[q].residual, bool(res[q].converged), res[q].status, res[q].folds,
                            res[q].seconds, res[q].kernels) for q in range(nrhs)]

    def set_stream(self, stream_ptr):
        """Route the handle's work to a CUDA stream (e.g. ``torch.cuda.Stream().cuda_stream``)."""
        st = _set_stream(self.h, C.c_void_p(stream_ptr) if stream_ptr else None)
        if st != PS_OK:
            _raise(st)

    def time_kernel(self, which=0, reps=20):
        """Mean ms of the finest level's operator kernel (0: FP32 smoothing step, 1: FP64 product)."""
        ms = C.c_double()
        st = _time_kernel(self.h, which, reps, C.byref(ms))
        if st != PS_OK:
            _raise(st)
        return ms.value

    def apply_dot_noalloc(self, x_ptr, y_ptr, dot_ptr, stream_ptr=None):
        """y = K x and x.y on device pointers without allocating (see ps_fea_apply_dot_noalloc);
        stream-ordered, returns before the GPU has finished. stream_ptr is a CUDA stream handle
        such as ``torch.cuda.current_stream().cuda_stream``: 0 is the legacy default stream (what
        PyTorch reports for its default stream) and None the handle's own stream."""
        if stream_ptr is None:
            stream = None
        elif stream_ptr == 0:
            stream = C.c_void_p(CUDA_STREAM_LEGACY)
        else:
            stream = C.c_void_p(stream_ptr)
        st = _apply_dot_noalloc(self.h, C.c_void_p(x_ptr), C.c_void_p(y_ptr), C.c_void_p(dot_ptr), stream)
        if st != PS_OK:
            _raise(st)

    @property
    def kernel_launches(self):
        return int(_launches(self.h))

    def precondition(self, r):
        r = self._check_vec(r, "r")
        z = np.zeros_like(r)
        st = _precondition(self.h, r, z)
        if st != PS_OK:
            _raise(st)
        return z

    def autotune(self, f, tol=1e-8, max_iter=5000, precision="fp64", force=False):
        """Times solves of f over smoother degrees and tile paths, keeps the fastest on this handle
        (see ps_fea_autotune); returns the choice as a dict."""
        f = self._check_vec(f, "f")
        o = make_opts(tol, max_iter, precision)
        t = TuneResultC()
        st = _autotune(self.h, f, C.byref(o), PS_TUNE_FORCE if force else 0, C.byref(t))
        if st != PS_OK:
            _raise(st)
        return {k: getattr(t, k) for k, _ in TuneResultC._fields_}

    @classmethod
    def create_tuned(cls, dims, density, nu, bc, f, tol=1e-8, max_iter=5000, precision="fp64", force=False, diag_add=None):
        """A handle built for the fastest of several coarsening depths, each autotuned on f (see
        ps_fea_create_tuned); returns (handle, choice)."""
        self = cls.__new__(cls)
        self.dims = np.ascontiguousarray(dims, np.int32)
        density = np.ascontiguousarray(density, np.float32).ravel()
        bc = np.ascontiguousarray(bc, np.uint8).ravel()
        f = np.ascontiguousarray(f, np.float64).ravel()
        self._diag = None if diag_add is None else np.ascontiguousarray(diag_add, np.float64).ravel()
        o = make_opts(tol, max_iter, precision)
        t = TuneResultC()
        h = C.c_void_p()
        st = _create_tuned(self.dims, density, float(nu), bc, _ptr(self._diag), f, C.byref(o), PS_TUNE_FORCE if force else 0, C.byref(t),
                           C.byref(h))
        if st != PS_OK:
            _raise(st)
        self.h = h
        self.nu = nu
        return self, {k: getattr(t, k) for k, _ in TuneResultC._fields_}

    def precondition_block(self, nvec, r_ptr, z_ptr, stream_ptr=None):
        """z_k = V-cycle preconditioner of r_k for nvec consecutive device vectors (pointers, e.g.
        ``tensor.data_ptr()``); stream-ordered on stream_ptr (0: the legacy default stream, None:
        the handle's stream), returns before the GPU has finished."""
        if stream_ptr is None:
            stream = None
        elif stream_ptr == 0:
            stream = C.c_void_p(CUDA_STREAM_LEGACY)
        else:
            stream = C.c_void_p(stream_ptr)
        st = _precondition_block(self.h, int(nvec), C.c_void_p(r_ptr), C.c_void_p(z_ptr), stream)
        if st != PS_OK:
            _raise(st)

    def apply(self, x, level=0, raw=False):
        x = np.ascontiguousarray(x, np.float64).ravel()
        if x.size != self.level_info(level)["nDof"]:
            raise ValueError("vector has the wrong size")
        y = np.zeros_like(x)
        st = _apply(self.h, level, x, y, int(raw))
        if st != PS_OK:
            _raise(st)
        return y

    def stresses(self, u, E, h, principals=True):
        u = self._check_vec(u, "u")
        nn = self.n_nodes
        vm = np.zeros(nn, np.float32)
        p1 = np.zeros(nn, np.float32) if principals else None
        p3 = np.zeros(nn, np.float32) if principals else None
        st = _stresses(self.h, u, float(E), float(h), int(principals), vm, _ptr(p1), _ptr(p3))
        if st != PS_OK:
            _raise(st)
        return vm, p1, p3

    def reactions(self, u, f=None):
        u = self._check_vec(u, "u")
        f = None if f is None else self._check_vec(f, "f")
        R = np.zeros(3, np.float64)
        st = _reactions(self.h, u, _ptr(f), R)
        if st != PS_OK:
            _raise(st)
        return R


class Hierarchy:
    """The host-side multigrid hierarchy alone, for inspection and tests. device=False: built on the
    host threads (no GPU needed); device=True: the Galerkin coarse matrices of graded levels are
    computed on the current CUDA device (the build ``VoxelFEA`` handles use), bitwise the same."""

    def __init__(self, dims, density, nu, bc, coarsest_max_dof=1100, diag_add=None, device=False):
        dims = np.ascontiguousarray(dims, np.int32)
        density = np.ascontiguousarray(density, np.float32).ravel()
        bc = np.ascontiguousarray(bc, np.uint8).ravel()
        nx, ny, nz = (int(v) for v in dims)
        if nx >= 1 and ny >= 1 and nz >= 1 and (density.size != nx * ny * nz or bc.size != 3 * (nx + 1) * (ny + 1) * (nz + 1)):
            raise ValueError("Structural grid, density and fixture sizes do not match.")
        self._diag = None if diag_add is None else np.ascontiguousarray(diag_add, np.float64).ravel()
        h = C.c_void_p()
        st = (_h_create_dev if device else _h_create)(dims, density, float(nu), bc, int(coarsest_max_dof), _ptr(self._diag), C.byref(h))
        if st != PS_OK:
            _raise(st)
        self.h = h

    def __del__(self):
        if getattr(self, "h", None):
            _h_destroy(self.h)
            self.h = None

    @property
    def n_levels(self):
        return int(_h_nlev(self.h))

    def level_info(self, l):
        out = np.zeros(9, np.int64)
        if _h_info(self.h, l, out) != PS_OK:
            _raise(PS_EINVAL)
        keys = ("nx", "ny", "nz", "nNodes", "nDof", "freeDof", "nElems", "nOwn", "coarse_m")
        return dict(zip(keys, (int(v) for v in out)))

    def fixed(self, l=0):
        out = np.zeros(self.level_info(l)["nDof"], np.uint8)
        _h_fixed(self.h, l, out)
        return out

    def own(self, l):
        n = self.level_info(l)["nOwn"]
        out = np.zeros(max(n, 1) * 576, np.float32)
        _h_own(self.h, l, out)
        return out[: n * 576].reshape(n, 24, 24)

    def kb(self, l):
        out = np.zeros(576, np.float64)
        _h_kb(self.h, l, out)
        return out.reshape(24, 24)


def element_matrix(nu):
    """(K 24x24, corner stress 8x6x24) of the unit-cube element, E = 1."""
    K = np.zeros(576, np.float64)
    cs = np.zeros(8 * 144, np.float64)
    st = _element(float(nu), K, _ptr(cs))
    if st != PS_OK:
        _raise(st)
    return K.reshape(24, 24), cs.reshape(8, 6, 24)


def prune_floating(dims, density, held_node):
    dims = np.ascontiguousarray(dims, np.int32)
    density = np.ascontiguousarray(density, np.float32).ravel()
    out = np.zeros_like(density)
    removed = C.c_int32()
    st = _prune(dims, density, np.ascontiguousarray(held_node, np.uint8).ravel(), out, C.byref(removed))
    if st != PS_OK:
        _raise(st)
    return out, int(removed.value)


def prune_floating_dev(dims, density_ptr, held_ptr, out_ptr, stream_ptr=None):
    """pruneFloating on device arrays (pointers); returns the number of voxels removed."""
    removed = C.c_int32()
    st = _prune_dev(np.ascontiguousarray(dims, np.int32), C.c_void_p(density_ptr), C.c_void_p(held_ptr), C.c_void_p(out_ptr),
                    C.byref(removed), C.c_void_p(stream_ptr) if stream_ptr else None)
    if st != PS_OK:
        _raise(st)
    return int(removed.value)


def topology_run(dims, fill, nu, bc, f, keep=None, vol_frac=0.4, penal=3.0, rmin=1.5, move=0.2, tol=0.01, max_iter=40, solve_tol=1e-5,
                 precision="fp64"):
    """SIMP topology optimisation on the device (the reference's optimizeTopology,
    native/src/fea/topology.cpp:103-183). Returns (density, history): the final physical density per
    voxel and one dict per iteration (it, compliance, volume, change, solve_iterations, seconds)."""
    dims = np.ascontiguousarray(dims, np.int32)
    fill = np.ascontiguousarray(fill, np.float32).ravel()
    bc = np.ascontiguousarray(bc, np.uint8).ravel()
    f = np.ascontiguousarray(f, np.float64).ravel()
    keep = None if keep is None else np.ascontiguousarray(keep, np.uint8).ravel()
    o = TopologyOpts()
    _topo_default(C.byref(o))
    o.vol_frac, o.penal, o.rmin, o.move, o.tol = float(vol_frac), float(penal), float(rmin), float(move), float(tol)
    o.max_iter, o.solve_tol = int(max_iter), float(solve_tol)
    o.precision = PREC[precision] if isinstance(precision, str) else int(precision)
    out = np.zeros(fill.size, np.float32)
    hist = (TopologyStepC * max(1, int(max_iter)))()
    n = C.c_int32()
    st = _topo_run(dims, fill, _ptr(keep), float(nu), bc, f, C.byref(o), out, C.cast(hist, C.c_void_p), C.byref(n))
    if st != PS_OK:
        _raise(st)
    return out, [{k: getattr(hist[q], k) for k, _ in TopologyStepC._fields_} for q in range(n.value)]


def break_test(dims, density, nu, bc, f, E, h, strength, principal=False, max_steps=10, cracked_cap=1 << 20):
    """Progressive failure on the device (the reference's breakTest, native/src/fea/static_study.cpp:
    199-279). Returns a dict: steps (one dict each), cracked (voxel lists per step), density left,
    peak load factor and the stop reason."""
    dims = np.ascontiguousarray(dims, np.int32)
    density = np.ascontiguousarray(density, np.float32).ravel()
    bc = np.ascontiguousarray(bc, np.uint8).ravel()
    f = np.ascontiguousarray(f, np.float64).ravel()
    steps = (BreakStepC * max(1, int(max_steps)))()
    n = C.c_int32()
    cracked = np.zeros(int(cracked_cap), np.int32)
    out = np.zeros_like(density)
    peak = C.c_double()
    reason = C.c_int32()
    st = _break_test(dims, density, float(nu), bc, f, float(E), float(h), float(strength), int(bool(principal)), int(max_steps),
                     C.cast(steps, C.c_void_p), C.byref(n), cracked.ctypes.data_as(C.c_void_p), int(cracked_cap), out, C.byref(peak),
                     C.byref(reason))
    if st != PS_OK:
        _raise(st)
    rows, lists, at = [], [], 0
    for q in range(n.value):
        s = steps[q]
        rows.append({"step": s.step, "voxels": s.voxels, "solve_iterations": s.solve_iterations, "cracked": s.cracked, "detached": s.detached,
                     "lambda": s.lambda_, "max_disp": s.max_disp, "seconds": s.seconds})
        lists.append(cracked[at:at + s.cracked].copy())
        at += s.cracked
    return {"steps": rows, "cracked": lists, "density": out, "peak": peak.value, "reason": BREAK_REASONS.get(reason.value, str(reason.value))}


class Server:
    """Continuous-batching request loop (ps_server_*): submit solves at any time, each is built on
    host threads, admitted to the GPU by memory footprint and run concurrently with the others."""

    def __init__(self, budget_bytes=0, max_active=0, build_threads=0):
        h = C.c_void_p()
        st = _srv_create(int(budget_bytes), int(max_active), int(build_threads), C.byref(h))
        if st != PS_OK:
            _raise(st)
        self.h = h

    def submit(self, dims, density, nu, bc, f, tol=1e-8, max_iter=5000, precision="mixed", coarsest_max_dof=300, smoother_degree=0):
        density = np.ascontiguousarray(density, np.float32).ravel()
        bc = np.ascontiguousarray(bc, np.uint8).ravel()
        f = np.ascontiguousarray(f, np.float64).ravel()
        q = PsRequest()
        q.dims[:] = [int(v) for v in dims]
        q.density, q.bc, q.f = _ptr(density), _ptr(bc), _ptr(f)
        q.nu = float(nu)
        q.coarsest_max_dof = int(coarsest_max_dof)
        q.tol = float(tol)
        q.max_iter = int(max_iter)
        q.precision = PREC[precision] if isinstance(precision, str) else int(precision)
        q.smoother_degree = int(smoother_degree)
        rid = C.c_int64()
        st = _srv_submit(self.h, C.byref(q), C.byref(rid))
        if st != PS_OK:
            _raise(st)
        return int(rid.value)

    @staticmethod
    def _result(r, keep_u=True):
        u = None
        if keep_u and r.u:
            u = np.ctypeslib.as_array(C.cast(r.u, C.POINTER(C.c_double)), shape=(r.n_dof,)).copy()
        return {"id": r.id, "status": r.status, "iterations": r.iterations, "converged": bool(r.converged), "residual": r.residual,
                "n_dof": r.n_dof, "u": u, "build_s": r.build_s, "wait_s": r.wait_s, "solve_s": r.solve_s, "total_s": r.total_s}

    def wait(self, rid, keep_u=True, release=True):
        r = PsRequestResult()
        st = _srv_wait(self.h, int(rid), C.byref(r))
        if st != PS_OK:
            _raise(st)
        out = self._result(r, keep_u)
        if release:
            _srv_release(self.h, int(rid))
        return out

    def poll(self, rid, keep_u=True, release=True):
        r = PsRequestResult()
        st = _srv_poll(self.h, int(rid), C.byref(r))
        if st == PS_PENDING:
            return None
        if st != PS_OK:
            _raise(st)
        out = self._result(r, keep_u)
        if release:
            _srv_release(self.h, int(rid))
        return out

    def stats(self):
        s = PsServerStats()
        _srv_stats(self.h, C.byref(s))
        return {k: getattr(s, k) for k, _ in PsServerStats._fields_}

    def close(self):
        if getattr(self, "h", None):
            _srv_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
