"""ORACLE — test infrastructure only (tests/, the smoke check and bench.py's CPU-baseline leg).

ctypes loaders for the two CPU oracles of the voxel solve:

* ``Oracle("port")``: the restatement in ``oracle/psoracle.cpp`` (always built from this repo);
* ``Oracle("reference")``: the reference's own ``ps::VoxelFEA`` (native/src/fea/voxel_fea.hpp:130-189)
  compiled from its sources into ``oracle/_ref/libpsref.so`` by ``oracle/Makefile``.

Both expose the same calls, so a test can run either one, or both side by side.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIBS = {"port": (os.path.join(HERE, "libpsoracle.so"), "orc_"),
         "reference": (os.path.join(HERE, "_ref", "libpsref.so"), "ref_")}
_loaded = {}

_P = C.c_void_p
_I64P = np.ctypeslib.ndpointer(np.int64, flags="C")
_F64P = np.ctypeslib.ndpointer(np.float64, flags="C")
_F32P = np.ctypeslib.ndpointer(np.float32, flags="C")
_U8P = np.ctypeslib.ndpointer(np.uint8, flags="C")
_I32P = np.ctypeslib.ndpointer(np.int32, flags="C")


def available(kind):
    return os.path.exists(_LIBS[kind][0])


def build():
    """Compile the oracle libraries (the reference one only where its sources are present)."""
    import subprocess
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def _lib(kind):
    if kind in _loaded:
        return _loaded[kind]
    path, pre = _LIBS[kind]
    if not os.path.exists(path):
        raise FileNotFoundError(f"oracle library {path} is not built (make -C oracle)")
    lib = C.CDLL(path)

    def fn(name, res, *args):
        f = getattr(lib, pre + name)
        f.restype = res
        f.argtypes = list(args)
        return f

    ns = {
        "create": fn("create", _P, _I32P, _F32P, C.c_double, _U8P, C.c_int64, C.c_void_p, C.c_char_p, C.c_int),
        "destroy": fn("destroy", None, _P),
        "num_levels": fn("num_levels", C.c_int, _P),
        "level_info": fn("level_info", None, _P, C.c_int, _I64P),
        "level_fixed": fn("level_fixed", None, _P, C.c_int, _U8P),
        "level_active": fn("level_active", None, _P, C.c_int, _U8P),
        "level_kb": fn("level_kb", None, _P, C.c_int, _F64P),
        "level_elems": fn("level_elems", None, _P, C.c_int, _I32P),
        "level_kidx": fn("level_kidx", None, _P, C.c_int, _I32P),
        "level_rho": fn("level_rho", None, _P, C.c_int, _F64P),
        "level_own": fn("level_own", None, _P, C.c_int, _F32P),
        "level_invdiag": fn("level_invdiag", None, _P, C.c_int, _F64P),
        "prepare": fn("prepare", None, _P),
        "level_lmax": fn("level_lmax", C.c_double, _P, C.c_int),
        "set_lmax": fn("set_lmax", None, _P, C.c_int, C.c_double),
        "apply": fn("apply", None, _P, C.c_int, _F64P, _F64P, C.c_int),
        "precondition": fn("precondition", None, _P, _F64P, _F64P),
        "vcycle32": fn("vcycle32", None, _P, C.c_int, _F32P, _F32P),
        "coarse_factor": fn("coarse_factor", None, _P, _F64P),
        "solve": fn("solve", C.c_int, _P, _F64P, C.c_double, C.c_int, C.c_void_p, _F64P, C.POINTER(C.c_int32),
                    C.POINTER(C.c_double), C.POINTER(C.c_int32), C.c_char_p, C.c_int),
        "stresses": fn("stresses", None, _P, _F64P, C.c_double, C.c_double, C.c_int, _F32P, C.c_void_p, C.c_void_p),
        "reactions": fn("reactions", None, _P, _F64P, C.c_void_p, _F64P),
        "element": fn("element", C.c_int, C.c_double, C.c_int, _F64P, C.c_void_p, C.c_void_p, C.c_char_p, C.c_int),
        "prune": fn("prune", C.c_int, _I32P, _F32P, _U8P, _F32P),
    }
    if kind == "port":
        ns["apply32"] = fn("apply32", None, _P, C.c_int, _F32P, _F32P)
    _loaded[kind] = ns
    return ns


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class OracleModel:
    """One voxel model on a CPU oracle: ``OracleModel(kind, dims, density, nu, bc, coarsest, diag_add)``."""

    def __init__(self, kind, dims, density, nu, bc, coarsest_max_dof=1100, diag_add=None):
        self.kind = kind
        self.L = _lib(kind)
        self.dims = np.ascontiguousarray(dims, dtype=np.int32)
        self.density = np.ascontiguousarray(density, dtype=np.float32).ravel()
        self.bc = np.ascontiguousarray(bc, dtype=np.uint8).ravel()
        self.diag_add = None if diag_add is None else np.ascontiguousarray(diag_add, dtype=np.float64).ravel()
        err = C.create_string_buffer(512)
        self.h = self.L["create"](self.dims, self.density, float(nu), self.bc, int(coarsest_max_dof), _ptr(self.diag_add), err, 512)
        if not self.h:
            raise ValueError(err.value.decode())

    def close(self):
        if self.h:
            self.L["destroy"](self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def n_levels(self):
        return self.L["num_levels"](self.h)

    def level_info(self, l):
        out = np.zeros(9, np.int64)
        self.L["level_info"](self.h, l, out)
        keys = ("nx", "ny", "nz", "nNodes", "nDof", "freeDof", "nElems", "nOwn", "coarse_m")
        return dict(zip(keys, (int(v) for v in out)))

    @property
    def n_dof(self):
        return self.level_info(0)["nDof"]

    def fixed(self, l=0):
        out = np.zeros(self.level_info(l)["nDof"], np.uint8)
        self.L["level_fixed"](self.h, l, out)
        return out

    def active(self, l=0):
        out = np.zeros(self.level_info(l)["nNodes"], np.uint8)
        self.L["level_active"](self.h, l, out)
        return out

    def kb(self, l=0):
        out = np.zeros(576, np.float64)
        self.L["level_kb"](self.h, l, out)
        return out.reshape(24, 24)

    def elems(self, l):
        out = np.zeros(self.level_info(l)["nElems"], np.int32)
        self.L["level_elems"](self.h, l, out)
        return out

    def kidx(self, l):
        out = np.zeros(self.level_info(l)["nElems"], np.int32)
        self.L["level_kidx"](self.h, l, out)
        return out

    def rho(self, l):
        out = np.zeros(self.level_info(l)["nElems"], np.float64)
        self.L["level_rho"](self.h, l, out)
        return out

    def own(self, l):
        n = self.level_info(l)["nOwn"]
        out = np.zeros(max(n, 1) * 576, np.float32)
        self.L["level_own"](self.h, l, out)
        return out[: n * 576].reshape(n, 24, 24)

    def invdiag(self, l):
        out = np.zeros(self.level_info(l)["nDof"], np.float64)
        self.L["level_invdiag"](self.h, l, out)
        return out

    def prepare(self):
        self.L["prepare"](self.h)

    def lmax(self, l):
        return self.L["level_lmax"](self.h, l)

    def set_lmax(self, l, v):
        self.L["set_lmax"](self.h, l, float(v))

    def apply(self, x, level=0, raw=False):
        x = np.ascontiguousarray(x, np.float64)
        y = np.zeros_like(x)
        self.L["apply"](self.h, level, x, y, int(raw))
        return y

    def apply32(self, x, level=0):
        x = np.ascontiguousarray(x, np.float32)
        y = np.zeros_like(x)
        self.L["apply32"](self.h, level, x, y)
        return y

    def precondition(self, r):
        r = np.ascontiguousarray(r, np.float64)
        z = np.zeros_like(r)
        self.L["precondition"](self.h, r, z)
        return z

    def vcycle32(self, r, level=0):
        r = np.ascontiguousarray(r, np.float32)
        z = np.zeros_like(r)
        self.L["vcycle32"](self.h, level, r, z)
        return z

    def coarse_factor(self):
        m = self.level_info(self.n_levels - 1)["coarse_m"]
        out = np.zeros(max(m * m, 1), np.float64)
        self.L["coarse_factor"](self.h, out)
        return out[: m * m].reshape(m, m)

    def solve(self, f, tol=1e-6, max_iter=500, x0=None):
        f = np.ascontiguousarray(f, np.float64)
        u = np.zeros_like(f)
        it, res, conv = C.c_int32(), C.c_double(), C.c_int32()
        x0 = None if x0 is None else np.ascontiguousarray(x0, np.float64)
        err = C.create_string_buffer(512)
        rc = self.L["solve"](self.h, f, float(tol), int(max_iter), _ptr(x0), u, C.byref(it), C.byref(res), C.byref(conv), err, 512)
        if rc:
            raise ValueError(err.value.decode())
        return u, int(it.value), float(res.value), bool(conv.value)

    def stresses(self, u, E, h, principals=True):
        u = np.ascontiguousarray(u, np.float64)
        nn = self.level_info(0)["nNodes"]
        vm = np.zeros(nn, np.float32)
        p1 = np.zeros(nn, np.float32) if principals else None
        p3 = np.zeros(nn, np.float32) if principals else None
        self.L["stresses"](self.h, u, float(E), float(h), int(principals), vm, _ptr(p1), _ptr(p3))
        return vm, p1, p3

    def reactions(self, u, f=None):
        u = np.ascontiguousarray(u, np.float64)
        f = None if f is None else np.ascontiguousarray(f, np.float64)
        R = np.zeros(3, np.float64)
        self.L["reactions"](self.h, u, _ptr(f), R)
        return R


def element(kind, nu, modes=True):
    """(K 24x24, cornerStress 8x6x24, gaussB 8x6x24) of the unit-cube element for E = 1."""
    L = _lib(kind)
    K = np.zeros(576, np.float64)
    cs = np.zeros(8 * 144, np.float64)
    gb = np.zeros(8 * 144, np.float64)
    err = C.create_string_buffer(512)
    if L["element"](float(nu), int(modes), K, _ptr(cs), _ptr(gb), err, 512):
        raise ValueError(err.value.decode())
    return K.reshape(24, 24), cs.reshape(8, 6, 24), gb.reshape(8, 6, 24)


def topology(dims, fill, nu, bc, f, keep=None, vol_frac=0.4, penal=3.0, rmin=1.5, move=0.2, tol=0.01, max_iter=40, solve_tol=1e-5):
    """The reference's own optimizeTopology (native/src/fea/topology.cpp:103-183) with runTopology's
    solve (study_runner.cpp:403-419): (final density, [(it, compliance, volume, change), ...])."""
    path, _ = _LIBS["reference"]
    if not os.path.exists(path):
        raise FileNotFoundError(f"oracle library {path} is not built (make -C oracle REF=...)")
    lib = C.CDLL(path)
    fn = lib.ref_topology
    fn.restype = C.c_int
    fn.argtypes = [_I32P, _F32P, C.c_void_p, C.c_double, _U8P, _F64P, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int,
                   C.c_double, _F32P, _F64P, C.POINTER(C.c_int), C.c_char_p, C.c_int]
    fill = np.ascontiguousarray(fill, np.float32).ravel()
    keep = None if keep is None else np.ascontiguousarray(keep, np.uint8).ravel()
    out = np.zeros_like(fill)
    hist = np.zeros(4 * max(1, max_iter), np.float64)
    n = C.c_int()
    err = C.create_string_buffer(512)
    rc = fn(np.asarray(dims, np.int32), fill, _ptr(keep), float(nu), np.ascontiguousarray(bc, np.uint8).ravel(),
            np.ascontiguousarray(f, np.float64).ravel(), vol_frac, penal, rmin, move, tol, int(max_iter), solve_tol, out, hist, C.byref(n), err, 512)
    if rc:
        raise ValueError(err.value.decode())
    return out, [tuple(hist[4 * k:4 * k + 4]) for k in range(n.value)]


def prune(kind, dims, density, held_node):
    L = _lib(kind)
    density = np.ascontiguousarray(density, np.float32).ravel()
    out = np.zeros_like(density)
    removed = L["prune"](np.asarray(dims, np.int32), density, np.ascontiguousarray(held_node, np.uint8).ravel(), out)
    return out, int(removed)
