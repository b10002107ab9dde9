"""ctypes binding of libcastro_b200.so (the C-ABI declared in include/castro_b200.h).

The library is the product: every computation goes through its CUDA kernels.
Loading fails loudly when the shared library has not been built; there is no
CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBDIR = os.path.join(HERE, "lib")
MAX_SPEC = 13

BC_PERIODIC, BC_OUTFLOW = 0, 1
MODE_PLAIN, MODE_BATCHED, MODE_PLAIN_BOX, MODE_PERSISTENT = 0, 1, 2, 3

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class Problem(C.Structure):
    """castro_problem: the Sedov constants of Source/Prob.F90 plus the config knobs."""

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
        ("pert", C.c_void_p),
        ("pert_lo", C.c_int * 3),
        ("pert_hi", C.c_int * 3),
        ("pert_amp", C.c_double),
    ]


class InstanceDesc(C.Structure):
    _fields_ = [
        ("dom_lo", C.c_int * 3),
        ("dom_hi", C.c_int * 3),
        ("problo", C.c_double * 3),
        ("probhi", C.c_double * 3),
        ("bc", C.c_int),
        ("nbox", C.c_int),
        ("box_lo", _ip),
        ("box_hi", _ip),
        ("prob", Problem),
        ("stop_time", C.c_double),
    ]


_libs: dict[bool, C.CDLL] = {}

# every extern "C" symbol of include/castro_b200.h
ABI_SYMBOLS = [
    "castro_last_error", "castro_clear_error", "castro_error_string", "castro_version", "castro_set_stream",
    "castro_get_stream", "castro_exact_build", "network_init", "network_finalize", "castro_network_init",
    "castro_nspec", "eos_init", "eos_finalize", "castro_eos_init_path", "ctoprim", "enforce_minimum_density",
    "normalize_species", "reset_internal_e", "compute_temp", "castro_clean_state", "estdt", "store_flux", "fill_hydro_source",
    "normalize_species_fluxes", "apply_av", "trans1", "trans2", "compute_flux", "divu", "trace_ppm", "initdata",
    "denerror", "calculate_blast_radius", "castro_problem_defaults", "castro_set_problem",
    "castro_construct_hydro_source_box", "castro_sim_create", "castro_sim_destroy", "castro_sim_nbox",
    "castro_sim_box_size", "castro_sim_box_state", "castro_sim_init_data", "castro_sim_upload",
    "castro_sim_download", "castro_sim_total_size", "castro_sim_step", "castro_sim_run", "castro_sim_run_host",
    "castro_sim_sync", "castro_sim_time", "castro_sim_dt", "castro_sim_steps", "castro_sim_est_time_step",
    "castro_sim_blast_radius", "castro_sim_launches_per_step", "castro_sim_eos_failures", "castro_main",
    "castro_sim_stream", "castro_sim_profile_step", "castro_measure_fp64_tflops",
    "castro_construct_hydro_source_box_noalloc",
    "ctoprim_adj", "clean_state_adj", "divu_adj", "trace_ppm_adj", "compute_flux_adj", "trans1_adj", "trans2_adj",
    "apply_av_adj", "normalize_species_fluxes_adj", "fill_hydro_source_adj", "castro_adj_create",
    "castro_adj_destroy", "castro_adj_set_problem", "castro_adj_set_shell", "castro_adj_forward",
    "castro_adj_backward", "castro_adj_dt", "castro_adj_final_state", "castro_adj_initial_adjoint",
    "castro_adj_time_ms", "castro_adj_device_bytes", "castro_sim_write_plotfile",
    "castro_sim_write_checkpoint", "castro_sim_read_checkpoint", "castro_set_table_l2_window",
    "castro_set_momentum_flux_pressure", "castro_momentum_flux_pressure",
    "castro_set_coulomb_corrections", "castro_coulomb_corrections",
    "castro_set_column_tiles", "castro_column_tiles",
    "castro_flux_register_crse_init", "castro_flux_register_fine_add", "castro_flux_register_reflux",
    "castro_average_down",
    "castro_sim_set_wait_limit", "castro_saxpy", "castro_adj_create_window",
]


def lib_path(exact: bool = False) -> str:
    """Path of the library; CASTRO_B200_LIB / CASTRO_B200_EXACT_LIB override it."""
    env = os.environ.get("CASTRO_B200_EXACT_LIB" if exact else "CASTRO_B200_LIB")
    if env:
        return env
    return os.path.join(LIBDIR, "libcastro_b200_exact.so" if exact else "libcastro_b200.so")


def load(exact: bool = False) -> C.CDLL:
    """Load the CUDA library (production or CASTRO_EXACT build)."""
    if exact in _libs:
        return _libs[exact]
    path = lib_path(exact)
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing: build it with `python mini-castro_b200/build.py` "
                           "(the CTU advance has no CPU fallback)")
    L = C.CDLL(path)
    L.castro_error_string.restype = C.c_char_p
    L.castro_network_init.argtypes = [C.c_int, _dp, _dp]
    L.castro_eos_init_path.argtypes = [C.c_char_p]
    L.castro_set_stream.argtypes = [C.c_void_p]
    L.castro_get_stream.restype = C.c_void_p
    L.castro_problem_defaults.argtypes = [C.POINTER(Problem)]
    L.castro_set_problem.argtypes = [C.POINTER(Problem)]
    L.castro_sim_create.restype = C.c_void_p
    L.castro_sim_create.argtypes = [C.c_int, C.POINTER(InstanceDesc), C.c_int]
    L.castro_sim_destroy.argtypes = [C.c_void_p]
    L.castro_sim_nbox.argtypes = [C.c_void_p, C.c_int]
    L.castro_sim_box_size.restype = C.c_size_t
    L.castro_sim_box_size.argtypes = [C.c_void_p, C.c_int, C.c_int]
    L.castro_sim_box_state.restype = C.c_void_p
    L.castro_sim_box_state.argtypes = [C.c_void_p, C.c_int, C.c_int]
    L.castro_sim_init_data.argtypes = [C.c_void_p]
    L.castro_sim_upload.argtypes = [C.c_void_p, C.c_void_p]
    L.castro_sim_download.argtypes = [C.c_void_p, C.c_void_p]
    L.castro_sim_total_size.restype = C.c_size_t
    L.castro_sim_total_size.argtypes = [C.c_void_p]
    L.castro_sim_step.argtypes = [C.c_void_p]
    L.castro_sim_run.argtypes = [C.c_void_p, C.c_int]
    L.castro_sim_run_host.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]
    L.castro_sim_sync.argtypes = [C.c_void_p]
    for f in ("castro_sim_time", "castro_sim_dt", "castro_sim_est_time_step"):
        getattr(L, f).restype = C.c_double
        getattr(L, f).argtypes = [C.c_void_p, C.c_int]
    L.castro_sim_steps.argtypes = [C.c_void_p, C.c_int]
    L.castro_sim_blast_radius.restype = C.c_double
    L.castro_sim_blast_radius.argtypes = [C.c_void_p, C.c_int, _dp]
    L.castro_sim_launches_per_step.argtypes = [C.c_void_p]
    L.castro_sim_stream.restype = C.c_void_p
    L.castro_sim_stream.argtypes = [C.c_void_p]
    L.castro_sim_profile_step.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_char_p)]
    L.castro_measure_fp64_tflops.restype = C.c_double
    L.castro_sim_eos_failures.restype = C.c_longlong
    L.castro_sim_eos_failures.argtypes = [C.c_void_p]
    L.castro_sim_write_plotfile.argtypes = [C.c_void_p, C.c_int, C.c_char_p]
    L.castro_set_table_l2_window.argtypes = [C.c_int]
    L.castro_set_momentum_flux_pressure.argtypes = [C.c_int]
    L.castro_momentum_flux_pressure.restype = C.c_int
    L.castro_set_coulomb_corrections.argtypes = [C.c_int]
    L.castro_set_column_tiles.argtypes = [C.c_int]
    L.castro_column_tiles.restype = C.c_int
    L.castro_coulomb_corrections.restype = C.c_int
    L.castro_saxpy.argtypes = [C.c_void_p, C.c_void_p, C.c_longlong, C.c_double]
    L.castro_sim_set_wait_limit.argtypes = [C.c_void_p, C.c_longlong, C.c_int, C.c_int]
    L.castro_sim_write_checkpoint.argtypes = [C.c_void_p, C.c_char_p]
    L.castro_sim_read_checkpoint.argtypes = [C.c_void_p, C.c_char_p]
    L.castro_adj_create.restype = C.c_void_p
    L.castro_adj_create.argtypes = [C.POINTER(InstanceDesc), C.c_int, C.c_int]
    L.castro_adj_create_window.restype = C.c_void_p
    L.castro_adj_create_window.argtypes = [C.POINTER(InstanceDesc), C.c_int, C.c_int, C.c_int, C.c_int]
    L.castro_adj_destroy.argtypes = [C.c_void_p]
    L.castro_adj_set_problem.argtypes = [C.c_void_p, C.POINTER(Problem)]
    L.castro_adj_set_shell.argtypes = [C.c_void_p, C.c_double, C.c_double]
    L.castro_adj_forward.argtypes = [C.c_void_p, _dp]
    L.castro_adj_backward.argtypes = [C.c_void_p, _dp, _dp, C.c_void_p]
    L.castro_adj_dt.restype = C.c_double
    L.castro_adj_dt.argtypes = [C.c_void_p, C.c_int]
    L.castro_adj_final_state.argtypes = [C.c_void_p, C.c_void_p]
    L.castro_adj_initial_adjoint.argtypes = [C.c_void_p, C.c_void_p]
    L.castro_adj_time_ms.restype = C.c_double
    L.castro_adj_time_ms.argtypes = [C.c_void_p, C.c_int]
    L.castro_adj_device_bytes.restype = C.c_size_t
    L.castro_adj_device_bytes.argtypes = [C.c_void_p]
    _libs[exact] = L
    return L


class CastroError(RuntimeError):
    pass


def check(L: C.CDLL, what: str = "") -> None:
    code = L.castro_last_error()
    if code:
        msg = L.castro_error_string().decode()
        L.castro_clear_error()
        raise CastroError(f"{what}: castro error {code}: {msg}")


def init(aion: Sequence[float], zion: Sequence[float], table: str, exact: bool = False) -> C.CDLL:
    """network_init + eos_init for the given species network and table file."""
    L = load(exact)
    a = np.ascontiguousarray(aion, dtype=np.float64)
    z = np.ascontiguousarray(zion, dtype=np.float64)
    L.castro_network_init(len(a), a.ctypes.data_as(_dp), z.ctypes.data_as(_dp))
    check(L, "castro_network_init")
    L.castro_eos_init_path(table.encode())
    check(L, "eos_init")
    return L


def make_problem(L: C.CDLL, **kw) -> Problem:
    p = Problem()
    L.castro_problem_defaults(C.byref(p))
    for k, v in kw.items():
        if k == "X":
            for n, x in enumerate(v):
                p.X[n] = x
            for n in range(len(v), MAX_SPEC):
                p.X[n] = 0.0
        elif k in ("pert_lo", "pert_hi"):
            for d in range(3):
                getattr(p, k)[d] = int(v[d])
        else:
            setattr(p, k, v)
    return p


def ivec(v):
    return (C.c_int * 3)(*[int(x) for x in v])


def dvec(v):
    return (C.c_double * len(v))(*[float(x) for x in v])


def dev_ptr(t) -> int:
    """Device pointer of a torch CUDA tensor (or an int pointer passed through)."""
    if isinstance(t, int):
        return t
    assert t.is_cuda and t.is_contiguous(), "expected a contiguous CUDA tensor"
    return t.data_ptr()


def call(L: C.CDLL, name: str, *args) -> None:
    """Call a Castro_F.H entry point: torch tensors become device pointers,
    3-int sequences become int[3] host arrays, 3-float sequences become double[3]."""
    cargs = []
    for a in args:
        if hasattr(a, "data_ptr"):
            cargs.append(C.c_void_p(dev_ptr(a)))
        elif isinstance(a, (list, tuple)) and all(isinstance(x, (int, np.integer)) for x in a):
            cargs.append(ivec(a))
        elif isinstance(a, (list, tuple)):
            cargs.append(dvec(a))
        elif isinstance(a, float):
            cargs.append(C.c_double(a))
        elif isinstance(a, (int, np.integer)):
            cargs.append(C.c_int(int(a)))
        elif a is None:
            cargs.append(C.c_void_p(0))
        else:
            cargs.append(a)
    getattr(L, name)(*cargs)
    check(L, name)


class Sim:
    """castro_sim: single-level Sedov instances advanced on the GPU."""

    def __init__(self, L: C.CDLL, instances: list[dict], mode: int = MODE_BATCHED):
        self.L = L
        self.instances = instances
        descs = (InstanceDesc * len(instances))()
        self._keep = []
        for n, inst in enumerate(instances):
            d = descs[n]
            for k in range(3):
                d.dom_lo[k] = inst["dom_lo"][k]
                d.dom_hi[k] = inst["dom_hi"][k]
                d.problo[k] = inst["problo"][k]
                d.probhi[k] = inst["probhi"][k]
            d.bc = inst["bc"]
            los = np.ascontiguousarray(np.array([b[0] for b in inst["boxes"]], dtype=np.int32).reshape(-1))
            his = np.ascontiguousarray(np.array([b[1] for b in inst["boxes"]], dtype=np.int32).reshape(-1))
            self._keep += [los, his]
            d.nbox = len(inst["boxes"])
            d.box_lo = los.ctypes.data_as(_ip)
            d.box_hi = his.ctypes.data_as(_ip)
            d.prob = inst["problem"]
            d.stop_time = inst.get("stop_time", -1.0)
        self.h = L.castro_sim_create(len(instances), descs, mode)
        check(L, "castro_sim_create")
        if not self.h:
            raise CastroError("castro_sim_create returned NULL")
        self.mode = mode

    def close(self):
        if getattr(self, "h", None):
            self.L.castro_sim_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def init_data(self):
        self.L.castro_sim_init_data(self.h)
        check(self.L, "castro_sim_init_data")

    def step(self, n: int = 1):
        self.L.castro_sim_run(self.h, n)
        check(self.L, "castro_sim_run")

    def sync(self):
        self.L.castro_sim_sync(self.h)
        check(self.L, "castro_sim_sync")

    @property
    def total_size(self) -> int:
        return int(self.L.castro_sim_total_size(self.h))

    def download(self) -> np.ndarray:
        out = np.empty(self.total_size, dtype=np.float64)
        self.L.castro_sim_download(self.h, out.ctypes.data_as(C.c_void_p))
        self.sync()
        return out

    def upload(self, host: np.ndarray):
        host = np.ascontiguousarray(host, dtype=np.float64)
        assert host.size == self.total_size
        self.L.castro_sim_upload(self.h, host.ctypes.data_as(C.c_void_p))
        self.sync()

    def box_states(self, flat: np.ndarray | None = None) -> list[list[np.ndarray]]:
        """Per instance, per box: (nx, ny, nz, NVAR) Fortran-order views of a downloaded state."""
        flat = self.download() if flat is None else flat
        nvar = 7 + int(self.L.castro_nspec())
        out, off = [], 0
        for inst in self.instances:
            boxes = []
            for lo, hi in inst["boxes"]:
                shape = tuple(h - l + 1 for l, h in zip(lo, hi)) + (nvar,)
                n = int(np.prod(shape))
                boxes.append(flat[off:off + n].reshape(shape, order="F"))
                off += n
            out.append(boxes)
        return out

    def time(self, inst: int = 0) -> float:
        return self.L.castro_sim_time(self.h, inst)

    def dt(self, inst: int = 0) -> float:
        return self.L.castro_sim_dt(self.h, inst)

    def steps(self, inst: int = 0) -> int:
        return self.L.castro_sim_steps(self.h, inst)

    def est_time_step(self, inst: int = 0) -> float:
        return self.L.castro_sim_est_time_step(self.h, inst)

    def write_plotfile(self, path: str, inst: int = 0):
        """AMReX plotfile of instance inst (castro_sim_write_plotfile)."""
        self.L.castro_sim_write_plotfile(self.h, inst, path.encode())
        check(self.L, "castro_sim_write_plotfile")

    def write_checkpoint(self, path: str):
        """Checkpoint of every instance (castro_sim_write_checkpoint)."""
        self.L.castro_sim_write_checkpoint(self.h, path.encode())
        check(self.L, "castro_sim_write_checkpoint")

    def read_checkpoint(self, path: str):
        """Restart from a checkpoint of a sim with the same instances (castro_sim_read_checkpoint)."""
        self.L.castro_sim_read_checkpoint(self.h, path.encode())
        check(self.L, "castro_sim_read_checkpoint")

    def blast_radius(self, inst: int = 0):
        m = C.c_double()
        r = self.L.castro_sim_blast_radius(self.h, inst, C.byref(m))
        check(self.L, "blast_radius")
        return r, m.value

    def stream(self) -> int:
        return int(self.L.castro_sim_stream(self.h))

    def profile_step(self) -> dict:
        """One batched step with an event around each fused kernel: {name: ms}."""
        ms = (C.c_double * 16)()
        names = (C.c_char_p * 16)()
        n = self.L.castro_sim_profile_step(self.h, ms, names)
        check(self.L, "castro_sim_profile_step")
        return {names[k].decode(): ms[k] for k in range(n)}

    def launches_per_step(self) -> int:
        return self.L.castro_sim_launches_per_step(self.h)

    def eos_failures(self) -> int:
        return int(self.L.castro_sim_eos_failures(self.h))


def assemble(instance: dict, boxes: list[np.ndarray]) -> np.ndarray:
    """Gather per-box states of one instance into a domain array (nx, ny, nz, NVAR)."""
    lo = instance["dom_lo"]
    hi = instance["dom_hi"]
    nvar = boxes[0].shape[3]
    G = np.zeros(tuple(h - l + 1 for l, h in zip(lo, hi)) + (nvar,), order="F")
    for (blo, bhi), U in zip(instance["boxes"], boxes):
        G[blo[0] - lo[0]:bhi[0] - lo[0] + 1, blo[1] - lo[1]:bhi[1] - lo[1] + 1, blo[2] - lo[2]:bhi[2] - lo[2] + 1] = U
    return G
