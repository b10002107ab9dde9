"""ctypes binding of the CPU oracle (test infrastructure only).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module, as the checker.  It builds ``oracle/_build/liboracle.so`` from
``castro_oracle.c`` with the Makefile beside it when the library is missing.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")
# the two builds of oracle/Makefile: "parity" (non-contracting, the checker) and
# "fast" (-O3 -march=native with FMA contraction: the timed CPU baseline, and an
# independent rounding of the same algorithm for the noise classification)
# and "count" (the parity build with every floating-point operation counted, op_count.cpp)
LIB_PATHS = {"parity": LIB_PATH, "fast": os.path.join(HERE, "_build", "liboracle_fast.so"),
             "count": os.path.join(HERE, "_build", "liboracle_count.so")}
OP_CLASSES = ("add", "mul", "div", "sqrt", "transcendental", "compare", "sign")

MAX_SPEC = 13
EOS_INPUT_RT, EOS_INPUT_RE, EOS_INPUT_RP = 1, 2, 3

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class EosT(C.Structure):
    _fields_ = [(n, C.c_double) for n in (
        "rho T p e h s abar zbar dpdT dpdr dedT dedr dhdT dhdr dsdT dsdr dpde dpdr_e "
        "cv cp xne xnp eta pele ppos mu mu_e y_e gam1 cs dpdA dpdZ dedA dedZ").split()]


class ProbT(C.Structure):
    _fields_ = [
        ("ambient_from_T", C.c_int),
        ("dens_ambient", C.c_double),
        ("p_ambient", C.c_double),
        ("T_ambient", C.c_double),
        ("exp_energy", C.c_double),
        ("r_init", C.c_double),
        ("nsub", C.c_int),
        ("X", C.c_double * MAX_SPEC),
        ("T_init", C.c_double),
        ("pert", _dp),
        ("pert_lo", C.c_int * 3),
        ("pert_hi", C.c_int * 3),
        ("pert_amp", C.c_double),
    ]


def build(force: bool = False) -> str:
    srcs = [os.path.join(HERE, f) for f in ("castro_oracle.c", "castro_oracle.h", "op_count.cpp")]
    newest = max(os.path.getmtime(f) for f in srcs)
    stale = [p for p in LIB_PATHS.values() if not os.path.exists(p) or os.path.getmtime(p) < newest]
    if force or stale:
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


_lib = None
_variants: dict = {}


def lib(variant: str = "parity"):
    """The oracle library: the parity build (default) or the "fast" timing build."""
    global _lib
    if variant != "parity":
        if variant not in _variants:
            build()
            _variants[variant] = _bind(C.CDLL(LIB_PATHS[variant]))
        return _variants[variant]
    if _lib is None:
        build()
        _lib = _bind(C.CDLL(LIB_PATH))
    return _lib


def _bind(L):
    """Argument and result types of the entry points the bindings call."""
    L.oracle_network_init.argtypes = [C.c_int, _dp, _dp]
    L.oracle_eos_init.argtypes = [C.c_char_p]
    L.oracle_eos.argtypes = [C.c_int, C.POINTER(EosT)]
    L.oracle_set_problem.argtypes = [C.POINTER(ProbT)]
    L.oracle_set_momentum_flux_pressure.argtypes = [C.c_int]
    L.oracle_set_coulomb_corrections.restype = None
    L.oracle_set_coulomb_corrections.argtypes = [C.c_int]
    L.oracle_level_create.restype = C.c_void_p
    L.oracle_level_create.argtypes = [C.c_int, _ip, _ip, _ip, _ip, _dp, _dp, C.c_int]
    L.oracle_level_destroy.argtypes = [C.c_void_p]
    L.oracle_level_state.restype = _dp
    L.oracle_level_state.argtypes = [C.c_void_p, C.c_int]
    L.oracle_level_set_threads.argtypes = [C.c_void_p, C.c_int]
    L.oracle_level_init_data.argtypes = [C.c_void_p]
    L.oracle_level_est_time_step.restype = C.c_double
    L.oracle_level_est_time_step.argtypes = [C.c_void_p]
    L.oracle_level_clean_state.argtypes = [C.c_void_p]
    L.oracle_level_advance.argtypes = [C.c_void_p, C.c_double]
    L.oracle_level_coarse_step.restype = C.c_double
    L.oracle_level_coarse_step.argtypes = [C.c_void_p, C.c_double]
    L.oracle_level_time.restype = C.c_double
    L.oracle_level_time.argtypes = [C.c_void_p]
    L.oracle_level_dt.restype = C.c_double
    L.oracle_level_dt.argtypes = [C.c_void_p]
    L.oracle_level_steps.restype = C.c_int
    L.oracle_level_steps.argtypes = [C.c_void_p]
    L.oracle_level_blast_radius.restype = C.c_double
    L.oracle_level_blast_radius.argtypes = [C.c_void_p, _dp]
    if hasattr(L, "oracle_op_counts"):
        L.oracle_op_counts.restype = None
        L.oracle_op_counts.argtypes = [C.POINTER(C.c_ulonglong)]
        L.oracle_op_counts_reset.restype = None
        L.oracle_op_counts_reset.argtypes = []
    return L


def op_counts_reset():
    """Zero the counting build's operation counters."""
    lib("count").oracle_op_counts_reset()


def op_counts() -> dict:
    """Floating-point operations the counting build has executed since the last
    reset, summed over threads, by class (OP_CLASSES)."""
    out = (C.c_ulonglong * len(OP_CLASSES))()
    lib("count").oracle_op_counts(out)
    return dict(zip(OP_CLASSES, (int(v) for v in out)))


def ptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["F_CONTIGUOUS"] or a.ndim <= 1
    return a.ctypes.data_as(_dp)


def ivec(v):
    return (C.c_int * 3)(*[int(x) for x in v])


def dvec(v):
    return (C.c_double * len(v))(*[float(x) for x in v])


def network_init(aion, zion, variant: str = "parity"):
    a = np.ascontiguousarray(aion, dtype=np.float64)
    z = np.ascontiguousarray(zion, dtype=np.float64)
    assert lib(variant).oracle_network_init(len(a), ptr(a), ptr(z)) == 0


def set_momentum_flux_pressure(on: bool, variant: str = "parity"):
    """The interface pressure in the normal momentum flux (off, as in the reference)."""
    lib(variant).oracle_set_momentum_flux_pressure(1 if on else 0)


def set_coulomb_corrections(on: bool, variant: str = "parity"):
    """Coulomb corrections in the EOS (off, as in the reference's eos.F90)."""
    lib(variant).oracle_set_coulomb_corrections(1 if on else 0)


def eos_init(path: str, variant: str = "parity"):
    rc = lib(variant).oracle_eos_init(path.encode())
    if rc != 0:
        raise RuntimeError(f"oracle_eos_init({path}) failed: {rc}")


def eos(mode: int, variant: str = "parity", **fields) -> EosT:
    st = EosT()
    for k, v in fields.items():
        setattr(st, k, float(v))
    lib(variant).oracle_eos(mode, C.byref(st))
    return st


def fab(lo, hi, ncomp):
    """An uninitialised-looking (NaN) FAB in Fortran order, shape (nx, ny, nz, ncomp)."""
    shape = tuple(h - l + 1 for l, h in zip(lo, hi)) + (ncomp,)
    return np.full(shape, np.nan, dtype=np.float64, order="F")


def call(name, *args):
    """Call an oracle_<name> entry point with numpy / list arguments."""
    f = getattr(lib(), "oracle_" + name)
    cargs = []
    for a in args:
        if isinstance(a, np.ndarray):
            if a.dtype == np.float64:
                cargs.append(a.ctypes.data_as(_dp))
            elif a.dtype == np.int8:
                cargs.append(a.ctypes.data_as(C.POINTER(C.c_byte)))
            else:
                raise TypeError(a.dtype)
        elif isinstance(a, (list, tuple)) and len(a) == 3 and all(isinstance(x, (int, np.integer)) for x in a):
            cargs.append(ivec(a))
        elif isinstance(a, (list, tuple)):
            cargs.append(dvec(a))
        elif isinstance(a, float):
            cargs.append(C.c_double(a))
        elif isinstance(a, (int, np.integer)):
            cargs.append(C.c_int(int(a)))
        elif isinstance(a, C.Array) or isinstance(a, C._Pointer):
            cargs.append(a)
        else:
            raise TypeError(type(a))
    return f(*cargs)


class Problem:
    """Problem constants passed to oracle_set_problem (keeps the perturbation alive)."""

    def __init__(self, *, ambient_from_T, dens_ambient, exp_energy, r_init, X,
                 p_ambient=1e21, T_ambient=1e6, nsub=10, T_init=1e9, pert=None, pert_lo=(0, 0, 0),
                 pert_amp=0.0):
        self.s = ProbT()
        self.s.ambient_from_T = int(ambient_from_T)
        self.s.dens_ambient = dens_ambient
        self.s.p_ambient = p_ambient
        self.s.T_ambient = T_ambient
        self.s.exp_energy = exp_energy
        self.s.r_init = r_init
        self.s.nsub = nsub
        for n, x in enumerate(X):
            self.s.X[n] = x
        self.s.T_init = T_init
        self.pert = None
        if pert is not None:
            self.pert = np.asfortranarray(pert, dtype=np.float64)
            self.s.pert = self.pert.ctypes.data_as(_dp)
            for d in range(3):
                self.s.pert_lo[d] = pert_lo[d]
                self.s.pert_hi[d] = pert_lo[d] + self.pert.shape[d] - 1
            self.s.pert_amp = pert_amp

    def install(self, variant: str = "parity"):
        lib(variant).oracle_set_problem(C.byref(self.s))


class Level:
    """A single AMR level (BoxArray + state) advanced by the oracle."""

    def __init__(self, boxes, dom_lo, dom_hi, problo, probhi, bc, nvar, variant: str = "parity"):
        self.boxes = [(tuple(l), tuple(h)) for l, h in boxes]
        los = np.array([b[0] for b in self.boxes], dtype=np.int32).reshape(-1)
        his = np.array([b[1] for b in self.boxes], dtype=np.int32).reshape(-1)
        self.nvar = nvar
        self.L = lib(variant)
        self.h = self.L.oracle_level_create(len(self.boxes), los.ctypes.data_as(_ip), his.ctypes.data_as(_ip),
                                           ivec(dom_lo), ivec(dom_hi), dvec(problo), dvec(probhi), int(bc))

    def __del__(self):
        if getattr(self, "h", None) and getattr(self, "L", None) is not None:
            self.L.oracle_level_destroy(self.h)
            self.h = None

    def state(self, b) -> np.ndarray:
        lo, hi = self.boxes[b]
        shape = tuple(h - l + 1 for l, h in zip(lo, hi)) + (self.nvar,)
        n = int(np.prod(shape))
        p = self.L.oracle_level_state(self.h, b)
        return np.ctypeslib.as_array(p, shape=(n,)).reshape(shape, order="F")

    def set_threads(self, n):
        self.L.oracle_level_set_threads(self.h, n)

    def init_data(self):
        self.L.oracle_level_init_data(self.h)

    def est_time_step(self):
        return self.L.oracle_level_est_time_step(self.h)

    def clean_state(self):
        self.L.oracle_level_clean_state(self.h)

    def advance(self, dt):
        self.L.oracle_level_advance(self.h, dt)

    def coarse_step(self, stop_time=-1.0):
        return self.L.oracle_level_coarse_step(self.h, stop_time)

    @property
    def time(self):
        return self.L.oracle_level_time(self.h)

    @property
    def dt(self):
        return self.L.oracle_level_dt(self.h)

    @property
    def steps(self):
        return self.L.oracle_level_steps(self.h)

    def blast_radius(self):
        m = C.c_double()
        r = self.L.oracle_level_blast_radius(self.h, C.byref(m))
        return r, m.value


def level_from_instance(inst: dict, nvar: int, variant: str = "parity") -> tuple["Level", "Problem"]:
    """An oracle Level + Problem for one instance of a workload description
    (on the given build of the oracle; its network and table must be initialised)."""
    p = dict(inst["problem"])
    prob = Problem(ambient_from_T=p["ambient_from_T"], dens_ambient=p["dens_ambient"], p_ambient=p["p_ambient"],
                   T_ambient=p["T_ambient"], exp_energy=p["exp_energy"], r_init=p["r_init"], X=p["X"],
                   nsub=p["nsub"], T_init=p["T_init"], pert=p.get("pert"), pert_lo=inst["dom_lo"],
                   pert_amp=p.get("pert_amp", 0.0))
    prob.install(variant)
    L = Level(inst["boxes"], inst["dom_lo"], inst["dom_hi"], inst["problo"], inst["probhi"], inst["bc"], nvar,
              variant)
    L.init_data()
    return L, prob


def assemble(L: "Level", inst: dict) -> np.ndarray:
    lo, hi = inst["dom_lo"], inst["dom_hi"]
    G = np.zeros(tuple(h - l + 1 for l, h in zip(lo, hi)) + (L.nvar,), order="F")
    for b, (blo, bhi) in enumerate(L.boxes):
        G[blo[0] - lo[0]:bhi[0] - lo[0] + 1, blo[1] - lo[1]:bhi[1] - lo[1] + 1,
          blo[2] - lo[2]:bhi[2] - lo[2] + 1] = L.state(b)
    return G
